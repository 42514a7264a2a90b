"""CPU emulation (test infrastructure) of the launch geometry and index arithmetic of the
density kernels in binsim_b200/csrc/pooldensity.cu: the host's grid and split choices,
each thread's shared-memory fill items, the per-lane fragments of mma.sync m8n8k4
(row.col, FP64: lane (g, t) = (lane / 4, lane % 4) supplies A[g][t] and B[t][g] and
receives D[g][2t], D[g][2t + 1]), and the addresses of the atomic flush.  Every buffer
index is bounds-checked, so running a case here checks the kernels' indexing against
their buffers before they run on a GPU."""
import numpy as np

TK, TM, TN, NT = 32, 64, 128, 512
LS, XS = TM + 4, TN + 4
SMS = 148

_lane = np.arange(32)
_g, _t = _lane >> 2, _lane & 3
_w = np.arange(16)
_rb, _ch = _w >> 1, _w & 1


def _check(i, n, what):
    i = np.asarray(i)
    if i.size and (i.min() < 0 or i.max() >= n):
        raise IndexError(f"{what}: index range [{i.min()}, {i.max()}] outside [0, {n})")


def _step(As, Bs, D):
    """One Acc::step: for kk in 0, 4, .., 28, every warp's eight m8n8k4 tiles."""
    for kk in range(0, TK, 4):
        a = As[kk + _t[None, :], _rb[:, None] * 8 + _g[None, :]]                        # [warp, lane]
        b = Bs[kk + _t[None, None, :], _ch[:, None, None] * 64 + _g[None, None, :]
               + 8 * np.arange(8)[None, :, None]]                                      # [warp, tile, lane]
        A = np.zeros((16, 8, 4))
        A[:, _g, _t] = a
        B = np.zeros((16, 8, 4, 8))
        B[:, :, _t, _g] = b
        D += np.einsum("wik,wjkl->wjil", A, B)


def _flush(D, C, m0, c0, mrows, ncols):
    """Acc::flush: lane (g, t) of warp w adds D[w, k, g, 2t + j] at row m0 + 8 rb + g,
    column c0 + 64 ch + 8 k + 2 t + j (rows < mrows, columns < ncols, nonzero only)."""
    for w in range(16):
        row = m0 + _rb[w] * 8 + _g
        for k in range(8):
            for j in range(2):
                col = c0 + _ch[w] * 64 + 8 * k + 2 * _t + j
                v = D[w, k, _g, 2 * _t + j]
                ok = (row < mrows) & (col < ncols) & (v != 0.0)
                _check(row[ok] * C.shape[1] + col[ok], C.size, "flush")
                np.add.at(C, (row[ok], col[ok]), v[ok])


def _signed(v, e, neg):
    _check(e, v.size, "vector gather")
    x = v.ravel()[e]
    return np.where(neg, -x, x)


def tab(n, nB, tA, tB, lt, rt, sms=SMS):
    """C [n^2 x n^2] as tab_kernel computes it, over the grid density_grad launches (for
    a GPU of `sms` multiprocessors: fewer make larger K splits per CTA)."""
    nHa, nHb = tA.shape[0], tB.shape[0]
    M = n * n
    C = np.zeros((M, M))
    tiles = -(-M // TM) * -(-M // TN)
    splits = max(1, min(nHa, -(-sms * 8 // tiles)))
    hsplit = -(-nHa // splits)
    grid = (-(-M // TM), -(-M // TN), -(-nHa // hsplit))
    tid = np.arange(NT)
    iA = tid[None, :] + np.arange(TK * TM // NT)[:, None] * NT
    iB = tid[None, :] + np.arange(TK * TN // NT)[:, None] * NT
    for bx in range(grid[0]):
        for by in range(grid[1]):
            m0, c0 = bx * TM, by * TN
            jA, jB = m0 + iA % TM, c0 + iB % TN
            ak, bk = iA // TM, iB // TN
            ap, ar = np.where(jA < M, jA // n, -1), np.where(jA < M, jA % n, 0)
            bp, br = np.where(jB < M, jB // n, -1), np.where(jB < M, jB % n, 0)
            for bz in range(grid[2]):
                hA0, hA1 = bz * hsplit, min(nHa, bz * hsplit + hsplit)
                D = np.zeros((16, 8, 8, 8))
                for hA in range(hA0, hA1):
                    _check(hA * n + ap[ap >= 0], tA.size, "idxA")
                    ia = np.where(ap >= 0, tA[hA, np.maximum(ap, 0)], -1)
                    ib = np.where(bp >= 0, tA[hA, np.maximum(bp, 0)], -1)
                    for hB0 in range(0, nHb, TK):
                        As, Bs = np.zeros((TK, LS)), np.zeros((TK, XS))
                        for (kk, ii, side, jj, src, sm, width) in (
                                (ak, ia, ar, iA, lt, As, TM), (bk, ib, br, iB, rt, Bs, TN)):
                            hB = hB0 + kk
                            live = (ii >= 0) & (hB < nHb)
                            _check((np.minimum(hB, nHb - 1) * n + side)[live], tB.size, "idxB")
                            jb = np.where(live, tB[np.minimum(hB, nHb - 1), side], -1)
                            ok = live & (jb >= 0)
                            e = np.where(ok, (ii >> 1) * nB + (jb >> 1), 0)
                            v = np.where(ok, _signed(src, e, ((ii ^ jb) & 1) == 1), 0.0)
                            _check(kk, TK, "slice row")
                            sm[kk, jj % width] = v
                        _step(As, Bs, D)
                _flush(D, C, m0, c0, M, M)
    return C


def pair2(n, nA, nB, t2, lt, rt, spin, sms=SMS, zcap=65535):
    """C2 [npair x npair] of one spin as pair2_kernel computes it: grid z capped at
    zcap, CTA z taking items z, z + zcap, ... (item = h2 * nos + o range)."""
    npair = n * (n - 1) // 2
    nH2 = t2.shape[0]
    nO = nB if spin == 0 else nA
    C2 = np.zeros((npair, npair))
    tiles = -(-npair // TM) * -(-npair // TN)
    want = max(1, -(-sms * 8 // (tiles * nH2)))
    osplit = max(TK, -(-(-(-nO // want)) // TK) * TK)
    nos = -(-nO // osplit)
    nitems = nH2 * nos
    grid = (-(-npair // TM), -(-npair // TN), min(nitems, zcap))
    tid = np.arange(NT)
    iA = tid[None, :] + np.arange(TK * TM // NT)[:, None] * NT
    iB = tid[None, :] + np.arange(TK * TN // NT)[:, None] * NT
    for bx in range(grid[0]):
        for by in range(grid[1]):
            m0, c0 = bx * TM, by * TN
            jA, jB = m0 + iA % TM, c0 + iB % TN
            for bz in range(grid[2]):
                D = np.zeros((16, 8, 8, 8))
                for item in range(bz, nitems, grid[2]):
                    h2, o0 = item // nos, (item % nos) * osplit
                    o1 = min(nO, o0 + osplit)
                    _check(h2 * npair + jA[jA < npair], t2.size, "idx2")
                    ia = np.where(jA < npair, t2[h2, np.minimum(jA, npair - 1)], -1)
                    ib = np.where(jB < npair, t2[h2, np.minimum(jB, npair - 1)], -1)
                    for s0 in range(o0, o1, TK):
                        As, Bs = np.zeros((TK, LS)), np.zeros((TK, XS))
                        for (ii, ii_flat, src, sm, width, step) in ((ia, iA, lt, As, TM, TM),
                                                                     (ib, iB, rt, Bs, TN, TN)):
                            kk = ii_flat // step
                            o = s0 + kk
                            ok = (ii >= 0) & (o < o1)
                            row = ii >> 1
                            e = np.where(ok, row * nB + o if spin == 0 else o * nB + row, 0)
                            v = np.where(ok, _signed(src, e, (ii & 1) == 1), 0.0)
                            sm[kk, ii_flat % width] = v
                        _step(As, Bs, D)
                _flush(D, C2, m0, c0, npair, npair)
    return C2
