"""Host-side construction of the inputs of the on-the-fly (OTF) operator path.

The CUDA library consumes an *OTF network*: a list of groups, each holding an
alpha X-mask ``ax``, a beta X-mask ``bx`` and a low-rank factorisation of the
Z-mask coefficient matrix of all Pauli strings sharing ``(ax, bx)``::

    <a ^ ax, b ^ bx | H_g | a, b> = sum_r PA_r(a) * PB_r(b)
    PA_r(a) = sum_k (-1)^popc(a & za[k]) * wa[k, r]        (PB likewise)

This module builds such networks from second-quantised operators:

* ``synthetic_integrals`` -- the seeded integral generator the benchmarks use
  (symmetric ``h``, PSD ERIs from a rank-24 Cholesky-like factor).
* ``jw_hamiltonian_terms`` -- Jordan-Wigner transform over interleaved spin
  orbitals (alpha = 2p, beta = 2p+1), restating the operator of the reference's
  ``src/include/ham/ham.hpp:402-450`` (H = h_pq a+_ps a_qs +
  1/2 g_pqrs a+_ps a+_qt a_rt a_ss) and its term order ``ham.hpp:18-31``
  (sort by x, then z).  The Pauli convention is ``P(x, z)|s> =
  (-1)^popc(s & z) |s ^ x>``, products obey ``(x1,z1)(x2,z2) =
  (-1)^popc(z1 & x2) (x1^x2, z1^z2)`` (the reference's multiply rule,
  ``jl/binqubitaabb.jl:313-374``).
* ``split_aabb`` -- even/odd bit de-interleave (``ham.hpp:520-551``).
* ``compress_groups`` -- per-(ax, bx) SVD compression restating
  ``jl/network.jl:158-246`` (rank = #singular values > tol, wa = U sqrt(S),
  wb = V sqrt(S), entries below 1e-12 zeroed).
* ``ucc_pool`` -- spin-orbital UCC generators ``t - t^dagger`` (one X group
  each, as ``jl/network.jl:248-301`` requires) and spin-adapted generators as
  ordered products of their spin-orbital components.

Everything here is setup work done once per molecule; none of it is on the
timed path.
"""
from __future__ import annotations

import dataclasses
import itertools
import math
from typing import List, Sequence, Tuple

import numpy as np

U64 = np.uint64


# ---------------------------------------------------------------------------
# bit helpers
# ---------------------------------------------------------------------------

def popcount_u64(x: np.ndarray) -> np.ndarray:
    """Vectorised popcount of a uint64 array."""
    x = x.astype(np.uint64, copy=True)
    m1, m2, m4 = U64(0x5555555555555555), U64(0x3333333333333333), U64(0x0F0F0F0F0F0F0F0F)
    x = x - ((x >> U64(1)) & m1)
    x = (x & m2) + ((x >> U64(2)) & m2)
    x = (x + (x >> U64(4))) & m4
    return ((x * U64(0x0101010101010101)) >> U64(56)).astype(np.int64)


def _deinterleave(mask, nbits: int, odd: bool) -> np.ndarray:
    """Take every second bit (even positions, or odd ones) and pack them; mask is a
    uint64 array or a list of uint64 words (bit 64w + i in word w)."""
    words = mask if isinstance(mask, list) else [mask]
    out = np.zeros_like(words[0], dtype=np.uint64)
    off = 1 if odd else 0
    for p in range(nbits):
        bit = 2 * p + off
        out |= ((words[bit // 64] >> U64(bit % 64)) & U64(1)) << U64(p)
    return out


# ---------------------------------------------------------------------------
# integrals
# ---------------------------------------------------------------------------

def synthetic_integrals(norb: int, seed: int = 0, nchol: int = 24):
    """Seeded synthetic real integrals.

    h_pq symmetric with off-diagonal N(0, 0.1^2) and diagonal sorted ascending
    in U[-2, 0]; (pq|rs) = sum_k L^k_pq L^k_rs with L^k symmetric, entries
    N(0, 0.05^2), k = 1..nchol (8-fold symmetric and positive semidefinite).

    Returns ``(h, g, e_nuc)`` with ``g[p,q,r,s] = (ps|qr)`` -- the index order
    the reference's generator reads (``py/mole_pbc_int.py:10``) -- so that
    H = sum h_pq a+_p a_q + 1/2 sum g_pqrs a+_p a+_q a_r a_s.
    """
    rng = np.random.default_rng(seed)
    h = np.triu(rng.normal(0.0, 0.1, (norb, norb)), 1)
    h = h + h.T
    np.fill_diagonal(h, np.sort(rng.uniform(-2.0, 0.0, norb)))
    L = np.triu(rng.normal(0.0, 0.05, (nchol, norb, norb)))
    L = L + np.triu(L, 1).transpose(0, 2, 1)
    eri = np.einsum("kpq,krs->pqrs", L, L)          # chemists' (pq|rs)
    g = np.ascontiguousarray(eri.transpose(0, 2, 3, 1))  # g[p,q,r,s] = (ps|qr)
    return h, g, 0.0


# ---------------------------------------------------------------------------
# Jordan-Wigner over interleaved spin orbitals
# ---------------------------------------------------------------------------

def _ladder_components(modes: np.ndarray, dagger: Sequence[bool], words: int = 1):
    """Pauli expansion of a product of ladder operators, vectorised over rows.

    ``modes`` is (n_terms, k) spin-orbital indices; ``dagger[i]`` tells whether
    factor i is a creation operator.  Each factor is
    ``1/2 X_j Z^{below j} (+/-) 1/2 X_j Z^{below j | j}`` (+ for creation).
    Returns (x, z, sign) arrays of shape (n_terms, 2**k); the common factor
    2**-k is left to the caller.  With ``words`` > 1 the masks span
    64 * words spin orbitals (the reference's UInt128 interleaved masks for
    more than 32 spatial orbitals) and x, z are lists of per-word arrays,
    word w holding spin orbitals 64w..64w+63.
    """
    n, k = modes.shape
    if words == 1:
        x = np.zeros((n, 1), dtype=np.uint64)
        z = np.zeros((n, 1), dtype=np.uint64)
        s = np.ones((n, 1), dtype=np.int64)
        for i in range(k):
            j = modes[:, i].astype(np.uint64)
            e = (U64(1) << j)[:, None]
            m = e - U64(1)
            comps = [(m, 1), (m | e, 1 if dagger[i] else -1)]
            xs, zs, ss = [], [], []
            for zc, sc in comps:
                # (x, z) * (e, zc): sign (-1)^popc(z & e)
                flip = 1 - 2 * (popcount_u64(z & e) & 1)
                xs.append(x ^ e)
                zs.append(z ^ zc)
                ss.append(s * flip * sc)
            x = np.concatenate(xs, axis=1)
            z = np.concatenate(zs, axis=1)
            s = np.concatenate(ss, axis=1)
        return x, z, s
    x = [np.zeros((n, 1), dtype=np.uint64) for _ in range(words)]
    z = [np.zeros((n, 1), dtype=np.uint64) for _ in range(words)]
    s = np.ones((n, 1), dtype=np.int64)
    full = U64(0xFFFFFFFFFFFFFFFF)
    for i in range(k):
        j = modes[:, i].astype(np.int64)
        wj, bj = j // 64, (j % 64).astype(np.uint64)
        e = [np.where(wj == w, U64(1) << bj, U64(0))[:, None] for w in range(words)]
        m = [np.where(w < wj, full, np.where(wj == w, (U64(1) << bj) - U64(1), U64(0)))[:, None]
             for w in range(words)]
        comps = [(m, 1), ([m[w] | e[w] for w in range(words)], 1 if dagger[i] else -1)]
        xs, zs, ss = [[] for _ in range(words)], [[] for _ in range(words)], []
        for zc, sc in comps:
            bit = np.zeros_like(s)
            for w in range(words):
                bit = bit + ((z[w] & e[w]) != 0)
            flip = 1 - 2 * (bit & 1)
            for w in range(words):
                xs[w].append(x[w] ^ e[w])
                zs[w].append(z[w] ^ zc[w])
            ss.append(s * flip * sc)
        x = [np.concatenate(xs[w], axis=1) for w in range(words)]
        z = [np.concatenate(zs[w], axis=1) for w in range(words)]
        s = np.concatenate(ss, axis=1)
    return x, z, s


def _combine_terms(x, z, c, tol):
    """Sum coefficients of equal (x, z) and drop |c| <= tol; sorted by (x, z).
    x, z are uint64 arrays, or lists of per-word arrays (highest word most
    significant) for masks wider than 64 spin orbitals."""
    if isinstance(x, list):
        keys = tuple(z) + tuple(x)          # lexsort: last key primary -> x high word first
        order = np.lexsort(keys)
        x = [w[order] for w in x]
        z = [w[order] for w in z]
        c = c[order]
        diff = np.zeros(max(len(c) - 1, 0), dtype=bool)
        for w in x + z:
            diff |= np.diff(w) != 0
        brk = np.flatnonzero(diff) + 1
        starts = np.r_[0, brk].astype(np.int64)
        cs = np.add.reduceat(c, starts) if len(c) else c
        keep = np.abs(cs) > tol
        return [w[starts][keep] for w in x], [w[starts][keep] for w in z], cs[keep]
    order = np.lexsort((z, x))
    x, z, c = x[order], z[order], c[order]
    brk = np.flatnonzero((np.diff(x) != 0) | (np.diff(z) != 0)) + 1
    starts = np.r_[0, brk]
    cs = np.add.reduceat(c, starts) if len(c) else c
    xs, zs = x[starts], z[starts]
    keep = np.abs(cs) > tol
    return xs[keep], zs[keep], cs[keep]


def jw_hamiltonian_terms(h, g, e_nuc: float = 0.0, tol: float = 1e-12):
    """Jordan-Wigner Pauli terms (x, z, c) of the spin-orbital Hamiltonian.

    Spin orbitals are interleaved (alpha p -> 2p, beta p -> 2p+1), restating
    the operator of the reference's ham.hpp:402-450; terms are summed, filtered
    at ``tol`` and sorted by (x, z) as the reference does (``ham.hpp:18-31``,
    stage 4 sort).  Up to 32 spatial orbitals x and z are uint64 arrays; above
    that (the reference's UInt128 masks, ham_real.cpp:4) they are lists of two
    uint64 word arrays, and the two-body terms are combined chunk by chunk.
    """
    norb = h.shape[0]
    if 2 * norb > 128:
        raise ValueError("jw_hamiltonian_terms supports at most 64 spatial orbitals")
    words = 1 if 2 * norb <= 64 else 2
    xs, zs, cs = [], [], []

    def add(x, z, c):
        if words == 1:
            xs.append(x.ravel()); zs.append(z.ravel()); cs.append(c.ravel())
        else:   # combine each chunk at once to bound memory
            cx, cz, cc = _combine_terms([w.ravel() for w in x], [w.ravel() for w in z], c.ravel(), 0.0)
            xs.append(cx); zs.append(cz); cs.append(cc)
    # one-body: h_pq a+_{p s} a_{q s}
    p, q = np.nonzero(np.abs(h) > tol)
    for sp in (0, 1):
        modes = np.stack([2 * p + sp, 2 * q + sp], axis=1)
        x, z, sgn = _ladder_components(modes, (True, False), words)
        add(x, z, sgn * (h[p, q] * 0.25)[:, None])
    # two-body: 1/2 g_pqrs a+_{p s} a+_{q t} a_{r t} a_{s s}
    idx = np.nonzero(np.abs(g) > tol)
    vals = g[idx] * 0.5
    P, Q, R, S = idx
    for s1, s2 in ((0, 0), (1, 1), (0, 1), (1, 0)):
        modes = np.stack([2 * P + s1, 2 * Q + s2, 2 * R + s2, 2 * S + s1], axis=1)
        # chunk to bound memory
        for lo in range(0, len(vals), 1 << 18):
            hi = min(len(vals), lo + (1 << 18))
            x, z, sgn = _ladder_components(modes[lo:hi], (True, True, False, False), words)
            add(x, z, sgn * (vals[lo:hi] * 0.0625)[:, None])
    if abs(e_nuc) > tol:
        if words == 1:
            xs.append(np.zeros(1, np.uint64)); zs.append(np.zeros(1, np.uint64))
        else:
            xs.append([np.zeros(1, np.uint64)] * 2); zs.append([np.zeros(1, np.uint64)] * 2)
        cs.append(np.array([e_nuc]))
    if words == 1:
        x = np.concatenate(xs); z = np.concatenate(zs); c = np.concatenate(cs).astype(np.float64)
        return _combine_terms(x, z, c, tol)
    x = [np.concatenate([t[w] for t in xs]) for w in range(2)]
    z = [np.concatenate([t[w] for t in zs]) for w in range(2)]
    return _combine_terms(x, z, np.concatenate(cs).astype(np.float64), tol)


def split_aabb(x, z, norb):
    """De-interleave Pauli masks into alpha and beta halves (``ham.hpp:520-551``);
    x, z may be uint64 arrays or lists of words (spin orbital 64w + i in word w)."""
    return (_deinterleave(x, norb, False), _deinterleave(z, norb, False),
            _deinterleave(x, norb, True), _deinterleave(z, norb, True))


# ---------------------------------------------------------------------------
# network container + SVD compression
# ---------------------------------------------------------------------------

@dataclasses.dataclass
class OTFNetwork:
    """Flat-array OTF network, the argument list of ``build_network_otf_f64``
    (reference ``src/include/op/declare.hpp:25-35``)."""

    norb: int
    orbsym: np.ndarray   # int64 [norb]
    axs: np.ndarray      # uint64 [ngs]
    bxs: np.ndarray      # uint64 [ngs]
    ranks: np.ndarray    # int64 [ngs]
    num_zas: np.ndarray  # int64 [ngs]
    num_zbs: np.ndarray  # int64 [ngs]
    flat_zas: np.ndarray  # uint64
    flat_zbs: np.ndarray  # uint64
    flat_wa: np.ndarray   # float64, per group column-major [num_za x rank]
    flat_wb: np.ndarray   # float64

    @property
    def ngs(self) -> int:
        return int(len(self.axs))

    def group(self, g: int):
        """(ax, bx, rank, za, zb, wa[num_za, rank], wb[num_zb, rank]) of group g."""
        za0 = int(self.num_zas[:g].sum()); zb0 = int(self.num_zbs[:g].sum())
        wa0 = int((self.num_zas[:g] * self.ranks[:g]).sum())
        wb0 = int((self.num_zbs[:g] * self.ranks[:g]).sum())
        na, nb, r = int(self.num_zas[g]), int(self.num_zbs[g]), int(self.ranks[g])
        wa = self.flat_wa[wa0:wa0 + na * r].reshape(r, na).T
        wb = self.flat_wb[wb0:wb0 + nb * r].reshape(r, nb).T
        return (int(self.axs[g]), int(self.bxs[g]), r, self.flat_zas[za0:za0 + na],
                self.flat_zbs[zb0:zb0 + nb], wa, wb)

    def type_codes(self) -> np.ndarray:
        """0 diagonal, 1 pure alpha, 2 pure beta, 3 mixed (``otf.hpp:289-296``)."""
        ax = self.axs != 0
        bx = self.bxs != 0
        return np.where(~ax & ~bx, 0, np.where(ax & ~bx, 1, np.where(~ax & bx, 2, 3))).astype(np.int64)

    def as_uint32(self):
        """Masks narrowed to uint32 (the reference's UInt32 string type)."""
        if self.norb > 32:
            raise ValueError("uint32 strings need norb <= 32")
        return dict(axs=self.axs.astype(np.uint32), bxs=self.bxs.astype(np.uint32),
                    flat_zas=self.flat_zas.astype(np.uint32), flat_zbs=self.flat_zbs.astype(np.uint32))


def compress_groups(ax, az, bx, bz, c, norb, tol=1e-12, orbsym=None) -> OTFNetwork:
    """Group terms by (ax, bx) (terms must be sorted so groups are contiguous)
    and compress each group's Z coefficient matrix by SVD (``jl/network.jl:158-246``)."""
    n = len(c)
    key_change = np.flatnonzero((np.diff(ax) != 0) | (np.diff(bx) != 0)) + 1
    starts = np.r_[0, key_change].astype(np.int64) if n else np.zeros(0, np.int64)
    ends = np.r_[key_change, n].astype(np.int64) if n else np.zeros(0, np.int64)
    return _compress_runs(ax, az, bx, bz, c, starts, ends, norb, tol, orbsym)


def _compress_runs(ax, az, bx, bz, c, starts, ends, norb, tol=1e-12, orbsym=None) -> OTFNetwork:
    """One group per run [starts[i], ends[i]) of terms: the run's Z coefficient
    matrix M[za, zb] compressed by SVD (rank = singular values > tol, wa = U sqrt(S),
    wb = V sqrt(S), entries below 1e-12 zeroed), SVDs batched by matrix shape."""
    ngs = len(starts)
    groups = [None] * ngs
    shapes = {}
    for gi, (i, j) in enumerate(zip(starts, ends)):
        ua = np.unique(az[i:j]); ub = np.unique(bz[i:j])
        M = np.zeros((len(ua), len(ub)))
        np.add.at(M, (np.searchsorted(ua, az[i:j]), np.searchsorted(ub, bz[i:j])), c[i:j])
        groups[gi] = (int(ax[i]), int(bx[i]), ua, ub, M)
        shapes.setdefault(M.shape, []).append(gi)
    result = [None] * ngs
    for shp, gl in shapes.items():
        Ms = np.stack([groups[gi][4] for gi in gl])
        U, S, Vt = np.linalg.svd(Ms, full_matrices=False)
        for t, gi in enumerate(gl):
            keep = np.flatnonzero(np.abs(S[t]) > tol)
            sq = np.sqrt(S[t][keep])
            wa = U[t][:, keep] * sq
            wb = Vt[t][keep, :].T * sq
            wa[np.abs(wa) < 1e-12] = 0.0
            wb[np.abs(wb) < 1e-12] = 0.0
            result[gi] = (groups[gi][0], groups[gi][1], len(keep), groups[gi][2], groups[gi][3], wa, wb)
    return _pack(result, norb, orbsym)


def _pack(groups, norb, orbsym=None) -> OTFNetwork:
    orbsym = np.zeros(norb, np.int64) if orbsym is None else np.asarray(orbsym, np.int64)
    A = lambda v, t: np.ascontiguousarray(np.asarray(v, dtype=t))
    cat = lambda parts, t: A(np.concatenate(parts) if parts else np.zeros(0), t)
    return OTFNetwork(
        norb=norb, orbsym=orbsym,
        axs=A([g[0] for g in groups], np.uint64), bxs=A([g[1] for g in groups], np.uint64),
        ranks=A([g[2] for g in groups], np.int64),
        num_zas=A([len(g[3]) for g in groups], np.int64), num_zbs=A([len(g[4]) for g in groups], np.int64),
        flat_zas=cat([g[3] for g in groups], np.uint64), flat_zbs=cat([g[4] for g in groups], np.uint64),
        flat_wa=cat([g[5].ravel(order="F") for g in groups], np.float64),
        flat_wb=cat([g[6].ravel(order="F") for g in groups], np.float64),
    )


def group_range(net: OTFNetwork, lo: int, hi: int) -> OTFNetwork:
    """The network's groups [lo, hi) as a network of their own (the flat arrays sliced;
    a rank's share of a pool when the pool gradient is split over ranks)."""
    if not 0 <= lo <= hi <= net.ngs:
        raise ValueError(f"group range [{lo}, {hi}) outside [0, {net.ngs})")
    nza, nzb = np.asarray(net.num_zas, np.int64), np.asarray(net.num_zbs, np.int64)
    rk = np.asarray(net.ranks, np.int64)
    za0, zb0 = int(nza[:lo].sum()), int(nzb[:lo].sum())
    za1, zb1 = int(nza[:hi].sum()), int(nzb[:hi].sum())
    wa0, wb0 = int((nza[:lo] * rk[:lo]).sum()), int((nzb[:lo] * rk[:lo]).sum())
    wa1, wb1 = int((nza[:hi] * rk[:hi]).sum()), int((nzb[:hi] * rk[:hi]).sum())
    c = lambda a: np.ascontiguousarray(a)
    return OTFNetwork(norb=net.norb, orbsym=c(net.orbsym), axs=c(net.axs[lo:hi]), bxs=c(net.bxs[lo:hi]),
                      ranks=c(rk[lo:hi]), num_zas=c(nza[lo:hi]), num_zbs=c(nzb[lo:hi]),
                      flat_zas=c(net.flat_zas[za0:za1]), flat_zbs=c(net.flat_zbs[zb0:zb1]),
                      flat_wa=c(net.flat_wa[wa0:wa1]), flat_wb=c(net.flat_wb[wb0:wb1]))


def hamiltonian_network(norb: int, seed: int = 0, tol: float = 1e-12, e_nuc=None, native: bool = False,
                        device: bool = False) -> OTFNetwork:
    """OTF network of the seeded synthetic Hamiltonian on ``norb`` orbitals.  native:
    group and compress with the library's builder (bsim_netbuild_*, host threads);
    device: the same with every group's SVD on the current GPU."""
    h, g, e0 = synthetic_integrals(norb, seed)
    x, z, c = jw_hamiltonian_terms(h, g, e0 if e_nuc is None else e_nuc, tol)
    ax, az, bx, bz = split_aabb(x, z, norb)
    if native or device:
        from binsim_b200 import cuotf
        return cuotf.compress_groups_native(ax, az, bx, bz, c, norb, tol, device=device)
    return compress_groups(ax, az, bx, bz, c, norb, tol)


# ---------------------------------------------------------------------------
# UCC generator pools
# ---------------------------------------------------------------------------

def _generator_terms(cre: Sequence[int], ann: Sequence[int]):
    """Pauli terms of t - t^dagger with t = a+_{cre...} a_{ann...} (spin orbitals).
    Returns combined (x, z, c) or None when the generator vanishes."""
    k = len(cre) + len(ann)
    modes = np.array([list(cre) + list(ann)], dtype=np.int64)
    x, z, s = _ladder_components(modes, [True] * len(cre) + [False] * len(ann))
    # t^dagger = a+_{ann reversed} a_{cre reversed}
    modes_d = np.array([list(reversed(ann)) + list(reversed(cre))], dtype=np.int64)
    xd, zd, sd = _ladder_components(modes_d, [True] * len(ann) + [False] * len(cre))
    scale = 0.5 ** k
    X = np.concatenate([x.ravel(), xd.ravel()])
    Z = np.concatenate([z.ravel(), zd.ravel()])
    C = np.concatenate([s.ravel() * scale, -sd.ravel() * scale]).astype(np.float64)
    X, Z, C = _combine_terms(X, Z, C, 1e-14)
    if len(C) == 0:
        return None
    if len(np.unique(X)) != 1:
        raise AssertionError("a generator t - t^dagger must have a single X mask")
    return X, Z, C


@dataclasses.dataclass
class Pool:
    """Spin-orbital generator network plus the spin-adapted grouping.

    ``network`` holds one group per spin-orbital component (original index =
    component index).  ``components[i]`` lists the component indices whose
    ordered product, sharing one angle, forms spin-adapted generator ``i``.
    ``excitations[g]`` is the (creators, annihilators) spin-orbital tuple of
    group g: the group is t - t^dagger with t = a+_{cre...} a_{ann...}."""

    network: OTFNetwork
    components: List[List[int]]
    labels: List[Tuple]
    excitations: List[Tuple[Tuple[int, ...], Tuple[int, ...]]] = dataclasses.field(default_factory=list)


def _component(cre, ann, norb):
    t = _generator_terms(cre, ann)
    if t is None:
        return None
    X, Z, C = t
    ax, az, bx, bz = split_aabb(X, Z, norb)
    return ax, az, bx, bz, C


def ucc_pool(norb: int, singles=True, doubles=True, generalized=True, nelec=None, native: bool = False,
             device: bool = False) -> Pool:
    """Spin-adapted generalised singles and doubles as ordered products of
    spin-orbital generators (alpha = 2p, beta = 2p+1).

    singles  (p > q):          a+_{p s} a_{q s} - h.c.,  s = alpha, beta
    doubles  (p >= q, r >= s,
              (p,q) > (r,s)):  a+_{p s} a+_{q t} a_{s t} a_{r s} - h.c. over the
                               spin pairs (s,t) in aa, bb, ab, ba with p,q
                               distinct for equal spins.
    Vanishing components (t = t^dagger) are dropped.  A spin-adapted generator
    applies its components in list order with a shared angle.
    """
    keys = []            # unique (cre, ann) spin-orbital components, first appearance order
    key_index = {}
    gens, labels = [], []

    def comp_id(cre, ann):
        key = (tuple(cre), tuple(ann))
        if key not in key_index:
            key_index[key] = len(keys)
            keys.append(key)
        return key_index[key]

    orbs = range(norb)
    if singles:
        for p in orbs:
            for q in orbs:
                if p <= q:
                    continue
                gens.append([comp_id([2 * p + s], [2 * q + s]) for s in (0, 1)]); labels.append(("s", p, q))
    if doubles:
        pairs = [(p, q) for p in orbs for q in orbs if p >= q]
        for (p, q), (r, s_) in itertools.combinations(pairs, 2):
            ids = []
            for s1, s2 in ((0, 0), (1, 1), (0, 1), (1, 0)):
                a1, a2 = 2 * p + s1, 2 * q + s2
                b1, b2 = 2 * r + s1, 2 * s_ + s2
                if a1 == a2 or b1 == b2:
                    continue
                i = comp_id([a1, a2], [b2, b1])
                if i not in ids:
                    ids.append(i)
            gens.append(ids); labels.append(("d", p, q, r, s_))
    # Pauli terms of every component, vectorised over components of one shape
    terms = [None] * len(keys)
    by_shape = {}
    for i, (cr, an) in enumerate(keys):
        by_shape.setdefault((len(cr), len(an)), []).append(i)
    for shp, idx in by_shape.items():
        for lo in range(0, len(idx), 1 << 15):
            chunk = idx[lo:lo + (1 << 15)]
            for i, t in zip(chunk, _components_batch([keys[i] for i in chunk], norb)):
                terms[i] = t
    # drop vanishing components (t = t^dagger) and renumber
    new_id = {}
    groups, excitations = [], []
    for i, t in enumerate(terms):
        if t is None:
            continue
        new_id[i] = len(groups)
        groups.append(t)
        excitations.append(keys[i])
    gens2, labels2 = [], []
    for ids, lab in zip(gens, labels):
        ids = [new_id[i] for i in ids if i in new_id]
        if ids:
            gens2.append(ids); labels2.append(lab)
    if not groups:
        raise ValueError("empty pool")
    AX = np.concatenate([g[0] for g in groups]); AZ = np.concatenate([g[1] for g in groups])
    BX = np.concatenate([g[2] for g in groups]); BZ = np.concatenate([g[3] for g in groups])
    CC = np.concatenate([g[4] for g in groups])
    sizes = [len(g[4]) for g in groups]
    if native or device:   # the library's builder, one group per component run (device: SVDs on the GPU)
        from binsim_b200 import cuotf
        net = cuotf.compress_groups_native(AX, AZ, BX, BZ, CC, norb, run_sizes=sizes, device=device)
    else:
        net = _compress_each(AX, AZ, BX, BZ, CC, sizes, norb)
    return Pool(network=net, components=gens2, labels=labels2, excitations=excitations)


def _compress_each(ax, az, bx, bz, c, sizes, norb, tol=1e-12) -> OTFNetwork:
    """SVD-compress consecutive runs of given sizes, one group per run
    (``jl/network.jl:248-301``)."""
    sizes = np.asarray(sizes, np.int64)
    ends = np.cumsum(sizes)
    starts = ends - sizes
    return _compress_runs(ax, az, bx, bz, c, starts, ends, norb, tol)


def _components_batch(keys, norb):
    """Pauli terms of t - t^dagger for many spin-orbital generators at once (all with
    the same numbers of creators and annihilators), de-interleaved to AABB form.

    Returns, per key, (ax, az, bx, bz, C) term arrays sorted by (x, z) or None when
    the generator vanishes (the per-generator path of ``_generator_terms``,
    vectorised over generators)."""
    words = 1 if 2 * norb <= 64 else 2
    n = len(keys)
    kc, ka = len(keys[0][0]), len(keys[0][1])
    modes = np.array([list(cr) + list(an) for cr, an in keys], dtype=np.int64)
    modes_d = np.array([list(reversed(an)) + list(reversed(cr)) for cr, an in keys], dtype=np.int64)
    x, z, sg = _ladder_components(modes, [True] * kc + [False] * ka, words)
    xd, zd, sd = _ladder_components(modes_d, [True] * ka + [False] * kc, words)
    scale = 0.5 ** (kc + ka)
    if words == 1:
        x, z, xd, zd = [x], [z], [xd], [zd]
    X = [np.concatenate([x[w], xd[w]], axis=1).ravel() for w in range(words)]
    Z = [np.concatenate([z[w], zd[w]], axis=1).ravel() for w in range(words)]
    C = np.concatenate([sg * scale, -sd * scale], axis=1).astype(np.float64).ravel()
    row = np.repeat(np.arange(n, dtype=np.int64), sg.shape[1] * 2)
    # sum equal (row, x, z) terms, drop |c| <= 1e-14 (as _combine_terms per generator)
    order = np.lexsort(tuple(Z) + tuple(X) + (row,))
    row, C = row[order], C[order]
    X = [w[order] for w in X]
    Z = [w[order] for w in Z]
    diff = np.diff(row) != 0
    for w in X + Z:
        diff |= np.diff(w) != 0
    starts = np.r_[0, np.flatnonzero(diff) + 1].astype(np.int64)
    cs = np.add.reduceat(C, starts)
    keep = np.abs(cs) > 1e-14
    starts = starts[keep]
    row, cs = row[starts], cs[keep]
    X = [w[starts] for w in X]
    Z = [w[starts] for w in Z]
    ax, az, bx, bz = split_aabb(X if words > 1 else X[0], Z if words > 1 else Z[0], norb)
    out = [None] * n
    bnd = np.r_[0, np.flatnonzero(np.diff(row) != 0) + 1, len(row)]
    for i in range(len(bnd) - 1):
        lo, hi = bnd[i], bnd[i + 1]
        r = int(row[lo])
        if np.any(ax[lo:hi] != ax[lo]) or np.any(bx[lo:hi] != bx[lo]):
            raise AssertionError("a generator t - t^dagger must have a single X mask")
        out[r] = (ax[lo:hi], az[lo:hi], bx[lo:hi], bz[lo:hi], cs[lo:hi])
    return out


def draw_generators(pool: Pool, n: int, seed: int = 0, amp_sigma: float = 0.05):
    """Seeded random sequence of ``n`` spin-adapted generators and amplitudes.

    Returns (op_idx, param_idx, thetas): the component sequence applied in
    order (indices into ``pool.network``), the parameter each component
    belongs to, and the ``n`` amplitudes ~ N(0, amp_sigma^2)."""
    rng = np.random.default_rng(seed)
    pick = rng.integers(0, len(pool.components), size=n)
    thetas = rng.normal(0.0, amp_sigma, size=n)
    op_idx, param_idx = [], []
    for i, gidx in enumerate(pick):
        for cidx in pool.components[gidx]:
            op_idx.append(cidx)
            param_idx.append(i)
    return np.asarray(op_idx, np.int64), np.asarray(param_idx, np.int64), thetas


def num_strings(norb: int, ne: int) -> int:
    return math.comb(norb, ne)
