"""CPU statement (numpy, test infrastructure) of the pool gradient at theta = 0 through
transition densities, the computation bsim_poolplan_classify plans for.

With l~ = eps l and r~ = eps r (eps(a, b) = (-1)^popc(b & K(a)), K(a) = XOR over alpha
electrons i of (1 << i) - 1: the interleaved -> alpha-first determinant sign) every pool
component's gradient <r| G |l> (op/batchgrad.hpp:529-540 at theta = 0) is a difference of
two entries of five tables, each a GEMM over strings with holes:

  D1a[p][q]       = sum_{k (n-1 electrons), b} (k+p | b)  (k+q | b)
  Tab[p][q][r][s] = sum_{kA, kB (n-1 each)}   (kA+p | kB+r) (kA+q | kB+s)
  Gaa[p][q][r][s] = sum_{k (n-2 electrons), b} (k+p+q | b) (k+s+r | b)   (a+_p a+_q a_r a_s)

where (k+p | b) is the l~ (left factor) or r~ (right factor) element of the string
a+_p |k> with that creation sign; D1b and Gbb are the same on the beta strings.
Single symmetry block only.
"""
import itertools

import numpy as np


def _popc(x):
    return bin(int(x)).count("1")


def eps_frame(astr, bstr):
    """eps[a, b] = (-1)^popc(b & K(a)) over the strings of one block."""
    K = []
    for a in astr:
        k = 0
        for i in range(64):
            if (int(a) >> i) & 1:
                k ^= (1 << i) - 1
        K.append(k)
    return np.array([[1.0 - 2.0 * (_popc(int(b) & k) & 1) for b in bstr] for k in K])


def _create(s, orbs):
    """(sign, string) of a+_{orbs[0]} a+_{orbs[1]} ... |s> (rightmost applied first), or (0, None)."""
    sg = 1
    for o in reversed(orbs):
        if (s >> o) & 1:
            return 0, None
        if _popc(s & ((1 << o) - 1)) & 1:
            sg = -sg
        s |= 1 << o
    return sg, s


def hole_table(strs, k, norb):
    """For the strings with k holes (k electrons removed from any string of strs):
    idx[h, t] (string index of a+_{t0} .. a+_{t(k-1)} |h>, 0 where it vanishes) and
    sgn[h, t] (its sign, 0 where it vanishes), t over ordered k-tuples of orbitals."""
    where = {int(s): i for i, s in enumerate(strs)}
    holes = sorted({int(s) ^ sum(1 << o for o in c) for s in strs
                    for c in itertools.combinations([o for o in range(norb) if (int(s) >> o) & 1], k)})
    tups = list(itertools.product(range(norb), repeat=k))
    idx = np.zeros((len(holes), len(tups)), np.int64)
    sgn = np.zeros((len(holes), len(tups)))
    for h, hs in enumerate(holes):
        for t, tup in enumerate(tups):
            sg, s = _create(hs, list(tup))
            if sg and s in where:
                idx[h, t], sgn[h, t] = where[s], sg
    return idx, sgn


def tables(astr, bstr, l, r, norb):
    """The five transition-density tables of l and r (interleaved-frame vectors of one
    block, alpha-major), as dense numpy arrays indexed by orbitals."""
    n = norb
    E = eps_frame(astr, bstr)
    L = E * np.asarray(l, float).reshape(len(astr), len(bstr))
    R = E * np.asarray(r, float).reshape(len(astr), len(bstr))
    out = {}
    # one hole: D1 (rows (hole, other-spin string), columns p) and Tab
    ia, sa = hole_table(astr, 1, n)
    ib, sb = hole_table(bstr, 1, n)

    def one(M, i1, s1):              # [(h, col), p]
        return (s1[:, :, None] * M[i1]).transpose(0, 2, 1).reshape(-1, n)
    out["d1a"] = one(L, ia, sa).T @ one(R, ia, sa)
    out["d1b"] = one(L.T, ib, sb).T @ one(R.T, ib, sb)

    def two(M):                      # [(hA, hB), (p, r)]
        g = M[ia[:, None, :, None], ib[None, :, None, :]] * (sa[:, None, :, None] * sb[None, :, None, :])
        return g.reshape(-1, n * n)
    T = (two(L).T @ two(R)).reshape(n, n, n, n)          # [p, r, q, s]
    out["tab"] = T.transpose(0, 2, 1, 3)                 # [p, q, r, s]
    # two holes, same spin
    for key, M, N, strs in (("gaa", L, R, astr), ("gbb", L.T, R.T, bstr)):
        i2, s2 = hole_table(strs, 2, n)
        lg = (s2[:, :, None] * M[i2]).transpose(0, 2, 1).reshape(-1, n * n)
        rg = (s2[:, :, None] * N[i2]).transpose(0, 2, 1).reshape(-1, n * n)
        # <a'| a+_p a+_q |h> <h| a_r a_s |a> with <h| a_r a_s |a> = <a| a+_s a+_r |h>
        G = (lg.T @ rg).reshape(n, n, n, n)              # [p, q, s, r]
        out[key] = G.transpose(0, 1, 3, 2)
    return out


_DAGGER = {1: (1, 0), 2: (1, 0), 3: (1, 0, 3, 2), 4: (3, 2, 1, 0), 5: (3, 2, 1, 0)}
_NAME = {1: "d1a", 2: "d1b", 3: "tab", 4: "gaa", 5: "gbb"}


def grads_from_plan(tab, kind, idx, coef):
    """grad_g = coef_g (X[dagger(idx_g)] - X[idx_g]) for every planned group (kind >= 1),
    0 for kind 0, NaN for kind -1 (general groups)."""
    g = np.full(len(kind), np.nan)
    for i, (k, ix, c) in enumerate(zip(kind, idx, coef)):
        if k == 0:
            g[i] = 0.0
        elif k > 0:
            X = tab[_NAME[int(k)]]
            m = len(_DAGGER[int(k)])
            fwd = tuple(int(v) for v in ix[:m])
            dag = tuple(fwd[j] for j in _DAGGER[int(k)])
            g[i] = c * (X[dag] - X[fwd])
    return g


def emulate_device(astr, bstr, l, r, norb, kind, idx, coef, hole_table, tables_out=None):
    """The arithmetic of the library's density kernels (pooldensity.cu), restated in numpy
    on the library's own hole tables (hole_table(strs, norb, holes) -> (nh, table) with
    entries (index << 1) | sign or -1): Tab as C[p n + r][q n + s], the same-spin tables
    as C2[pq][rs] = <a+_p a+_q a_s a_r> (p > q, r > s), D1 from Tab's traces, then
    grads = coef (X[dagger] - X[idx]) with 0 for kind 0 and NaN for kind -1.  tables_out
    (a dict), when given, receives lt, rt, C, C2a, C2b."""
    n = norb
    nA, nB = len(astr), len(bstr)
    E = eps_frame(astr, bstr)
    lt = E * np.asarray(l, float).reshape(nA, nB)
    rt = E * np.asarray(r, float).reshape(nA, nB)
    _, tA = hole_table(astr, n, 1)
    _, tB = hole_table(bstr, n, 1)

    def dec(t):
        return np.where(t >= 0, t >> 1, 0), np.where(t >= 0, 1.0 - 2.0 * (t & 1), 0.0)
    ia, sa = dec(tA)
    ib, sb = dec(tB)

    def gat(M):   # [(hA, hB), (p, r)]
        g = M[ia[:, None, :, None], ib[None, :, None, :]] * (sa[:, None, :, None] * sb[None, :, None, :])
        return g.reshape(-1, n * n)
    C = gat(lt).T @ gat(rt)
    npair = n * (n - 1) // 2
    C2 = {}
    for spin, (strs, Ml, Mr) in enumerate(((astr, lt, rt), (bstr, lt.T, rt.T))):
        nel = bin(int(strs[0])).count("1")
        if nel < 2:
            C2[spin] = None
            continue
        _, t2 = hole_table(strs, n, 2)
        i2, s2 = dec(t2)
        A = (s2[:, :, None] * Ml[i2]).transpose(0, 2, 1).reshape(-1, npair)
        B = (s2[:, :, None] * Mr[i2]).transpose(0, 2, 1).reshape(-1, npair)
        C2[spin] = A.T @ B
    if tables_out is not None:
        tables_out.update(lt=lt, rt=rt, C=C, C2a=C2[0], C2b=C2[1])
    na_el, nb_el = bin(int(astr[0])).count("1"), bin(int(bstr[0])).count("1")
    D1a = np.array([[sum(C[x * n + k, y * n + k] for k in range(n)) / nb_el for y in range(n)] for x in range(n)])
    D1b = np.array([[sum(C[k * n + x, k * n + y] for k in range(n)) / na_el for y in range(n)] for x in range(n)])

    def g2(M, p, q, r_, s):
        if M is None or p == q or r_ == s:
            return 0.0
        sg = -1.0
        if p < q:
            p, q, sg = q, p, -sg
        if r_ < s:
            r_, s, sg = s, r_, -sg
        return sg * M[p * (p - 1) // 2 + q, r_ * (r_ - 1) // 2 + s]

    def at(k, i0, i1, i2, i3):
        if k == 1:
            return D1a[i0, i1]
        if k == 2:
            return D1b[i0, i1]
        if k == 3:
            return C[i0 * n + i2, i1 * n + i3]
        return g2(C2[0] if k == 4 else C2[1], i0, i1, i2, i3)
    out = np.empty(len(kind))
    for g, (k, i, c) in enumerate(zip(kind, idx, coef)):
        k = int(k)
        if k <= 0:
            out[g] = 0.0 if k == 0 else np.nan
            continue
        i0, i1, i2, i3 = (int(v) for v in i)
        fwd = at(k, i0, i1, i2, i3)
        dag = at(k, i1, i0, 0, 0) if k in (1, 2) else (at(k, i1, i0, i3, i2) if k == 3 else at(k, i3, i2, i1, i0))
        out[g] = c * (dag - fwd)
    return out


def embed_blocks(B, v):
    """A vector of a symmetry-blocked oracle basis as a dense [all alpha strings x all beta
    strings] array (zeros where the determinant is not in the basis), with the union string
    lists in increasing order: the layout the density kernels use for blocked bases."""
    A = np.unique(np.concatenate([B.strings(k, 0) for k in range(B.num_blocks)]))
    Bs = np.unique(np.concatenate([B.strings(k, 1) for k in range(B.num_blocks)]))
    ia = {int(s): i for i, s in enumerate(A)}
    ib = {int(s): i for i, s in enumerate(Bs)}
    M = np.zeros((len(A), len(Bs)))
    v = np.asarray(v, float)
    for k in range(B.num_blocks):
        na, nb, off = int(B.blocks[k, 2]), int(B.blocks[k, 3]), int(B.blocks[k, 4])
        ra = [ia[int(s)] for s in B.strings(k, 0)]
        rb = [ib[int(s)] for s in B.strings(k, 1)]
        M[np.ix_(ra, rb)] = v[off:off + na * nb].reshape(na, nb)
    return A, Bs, M
