// Pool gradient at theta = 0 through transition densities.  A symmetry-blocked
// basis is embedded in the dense [all alpha strings x all beta strings] arrays
// (zeros outside the basis), on which the single-block computation below is exact.
//
// For the groups that bsim_poolplan_classify recognises as coef * (t - t^dagger),
// t one excitation with at most two creators and two annihilators, the gradient
// of op/batchgrad.hpp:529-540 at theta = 0 is coef * (X[dagger(i)] - X[i]) for one
// of five tables of the frame vectors l~ = eps l, r~ = eps r
// (eps(a, b) = (-1)^popc(b & K(a)), K(a) = XOR over alpha electrons i of (1 << i) - 1):
//
//   Tab  C[p n + r][q n + s] = sum_{hA, hB} A[(hA, hB)][p n + r] B[(hA, hB)][q n + s]
//        A = sA(hA, p) sB(hB, r) l~[hA + p][hB + r],  B the same on r~
//        = <l~| a+_p a_q (alpha) a+_r a_s (beta) |r~>      (hA, hB: one-hole strings)
//   Gaa  C2a[pq][rs] = sum_{h2, b} s(h2, pq) l~[h2 + pq][b] s(h2, rs) r~[h2 + rs][b]
//        = <l~| a+_p a+_q a_s a_r |r~> for p > q, r > s     (h2: two-hole alpha strings,
//        h2 + pq = a+_p a+_q |h2> with its sign)
//   Gbb  the same on the beta index
//   D1a[p][q] = sum_r Tab[p][q][r][r] / n_beta,  D1b[r][s] = sum_p Tab[p][p][r][s] / n_alpha
//        (the beta number operator is n_beta on every determinant)
//
// Tab and Gaa/Gbb are GEMMs whose operands are gathered through the hole tables
// ((string index << 1) | creation sign, or -1) straight from l~ and r~; FP64 on
// the DMMA path (mma.sync m8n8k4, 16 warps, a 64 x 128 output tile per CTA,
// 32-row K slices in shared memory), split over K with FP64 atomics into the
// tables.  At 36 orbitals and 3 + 3 electrons Tab is 1296 x 396,900 x 1296.
#include "../../include/binsim_cuotf.h"
#include "ops.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace bsim {

namespace {

constexpr unsigned kPoolDensityMagic = 0xB5B1D7A1u;
constexpr int kTK = 32, kTM = 64, kTN = 128;     // K slice, output tile
constexpr int kLS = kTM + 4, kXS = kTN + 4;      // shared strides (4 mod 16 doubles: no bank conflicts)
constexpr int kNT = 512;
constexpr i64 kMaxGridZ = 65535;
constexpr size_t kSmem = sizeof(double) * kTK * (kLS + kXS);   // 51,200 bytes: dynamic shared memory

__device__ __forceinline__ void dmma884(double &c0, double &c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

template <typename Ti>
__device__ __forceinline__ u64 kmask(Ti a)
{
    u64 s = (u64)a, k = 0;
    while (s) {
        const int i = __ffsll((long long)s) - 1;
        k ^= (1ull << i) - 1ull;
        s &= s - 1;
    }
    return k;
}

// lt = eps l, rt = eps r; grid (nA, ceil(nB / 256))
template <typename Ti>
__global__ void frame_pair_kernel(int nB, const Ti *__restrict__ astr, const Ti *__restrict__ bstr,
                                  const double *__restrict__ l, const double *__restrict__ r, double *__restrict__ lt,
                                  double *__restrict__ rt, const int *__restrict__ flag)
{
    const int a = blockIdx.x, b = blockIdx.y * blockDim.x + threadIdx.x;
    if (b >= nB || (flag && *flag == 0)) return;
    const u64 k = kmask(astr[a]);
    const i64 i = (i64)a * nB + b;
    const bool neg = __popcll((u64)bstr[b] & k) & 1;
    lt[i] = neg ? -l[i] : l[i];
    rt[i] = neg ? -r[i] : r[i];
}

// Blocked bases: block k's part of l and r (its alpha and beta string lists, at
// offset off) scattered with the frame sign into the dense [all alpha strings x
// all beta strings] arrays lt, rt (zeroed before; determinants outside the basis
// stay zero).  gA, gB: each block-list string's index in the union lists.
// grid (nAk, ceil(nBk / 256))
template <typename Ti>
__global__ void embed_frame_kernel(int nBk, int nBall, const Ti *__restrict__ astr, const Ti *__restrict__ bstr,
                                   const int *__restrict__ gA, const int *__restrict__ gB,
                                   const double *__restrict__ l, const double *__restrict__ r, double *__restrict__ lt,
                                   double *__restrict__ rt, const int *__restrict__ flag)
{
    const int a = blockIdx.x, b = blockIdx.y * blockDim.x + threadIdx.x;
    if (b >= nBk || (flag && *flag == 0)) return;
    const u64 k = kmask(astr[a]);
    const i64 i = (i64)a * nBk + b, o = (i64)gA[a] * nBall + gB[b];
    const bool neg = __popcll((u64)bstr[b] & k) & 1;
    lt[o] = neg ? -l[i] : l[i];
    rt[o] = neg ? -r[i] : r[i];
}

// Accumulator of one 64 x 128 tile of C = A^T B: each step multiplies a 32-row K
// slice held in shared memory (As[k][row], Bs[k][col]).  DMMA fragment mapping of
// m8n8k4 row.col: lane (g, t) = (lane / 4, lane % 4) holds A[g][t], B[t][g] and
// C[g][2t .. 2t+1]; warp w computes rows 8 (w / 2) .. +7 and columns
// 64 (w % 2) .. +63 as eight 8 x 8 tiles.
struct Acc {
    double c[8][2];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int k = 0; k < 8; ++k) c[k][0] = c[k][1] = 0.0;
    }
    __device__ __forceinline__ void step(const double (*As)[kLS], const double (*Bs)[kXS])
    {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const int g = lane >> 2, t = lane & 3, rb = wid >> 1, ch = wid & 1;
#pragma unroll
        for (int kk = 0; kk < kTK; kk += 4) {
            const double a = As[kk + t][rb * 8 + g];
            double b[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) b[k] = Bs[kk + t][ch * 64 + g + 8 * k];
#pragma unroll
            for (int k = 0; k < 8; ++k) dmma884(c[k][0], c[k][1], a, b[k]);
        }
    }
    // C[(m0 + row) * ldc + c0 + col] += tile, rows < mrows, cols < ncols
    __device__ __forceinline__ void flush(double *C, i64 ldc, int m0, int c0, int mrows, int ncols) const
    {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const int g = lane >> 2, t = lane & 3, rb = wid >> 1, ch = wid & 1;
        const int row = m0 + rb * 8 + g;
        if (row >= mrows) return;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int col = c0 + ch * 64 + 8 * k + 2 * t;
            if (col < ncols && c[k][0] != 0.0) atomicAdd(C + (i64)row * ldc + col, c[k][0]);
            if (col + 1 < ncols && c[k][1] != 0.0) atomicAdd(C + (i64)row * ldc + col + 1, c[k][1]);
        }
    }
};

__device__ __forceinline__ double signed_at(const double *__restrict__ v, i64 i, int neg)
{
    const double x = __ldg(v + i);
    return neg ? -x : x;
}

struct TabArgs {
    int n, nB, nHa, nHb, M, hsplit;
    const int *idxA;   // [nHa][n]
    const int *idxB;   // [nHb][n]
    const double *lt, *rt;
    double *C;         // [M][M]
    const int *flag;   // the launch does nothing when *flag == 0 (null: always runs)
};

// grid (ceil(M / 64), ceil(M / 128), ceil(nHa / hsplit)); K = (hA, hB), hA in the
// CTA's split, hB in 32-row slices (the last one zero-padded).
__global__ void __launch_bounds__(kNT, 1) tab_kernel(const TabArgs P)
{
    if (P.flag && *P.flag == 0) return;
    extern __shared__ __align__(16) double smem_tab[];
    double(*As)[kLS] = reinterpret_cast<double(*)[kLS]>(smem_tab);
    double(*Bs)[kXS] = reinterpret_cast<double(*)[kXS]>(smem_tab + kTK * kLS);
    const int m0 = blockIdx.x * kTM, c0 = blockIdx.y * kTN;
    const int hA0 = blockIdx.z * P.hsplit, hA1 = min(P.nHa, hA0 + P.hsplit);
    constexpr int IA = kTK * kTM / kNT, IB = kTK * kTN / kNT;   // 4 and 8 fill items per thread
    // fixed per thread: the item's slice row k and output index (p, r) or (q, s)
    int ak[IA], ap[IA], ar[IA], bk[IB], bp[IB], br[IB];
#pragma unroll
    for (int it = 0; it < IA; ++it) {
        const int i = threadIdx.x + it * kNT, j = m0 + i % kTM;
        ak[it] = i / kTM;
        ap[it] = j < P.M ? j / P.n : -1;
        ar[it] = j < P.M ? j % P.n : 0;
    }
#pragma unroll
    for (int it = 0; it < IB; ++it) {
        const int i = threadIdx.x + it * kNT, j = c0 + i % kTN;
        bk[it] = i / kTN;
        bp[it] = j < P.M ? j / P.n : -1;
        br[it] = j < P.M ? j % P.n : 0;
    }
    Acc acc;
    acc.zero();
    for (int hA = hA0; hA < hA1; ++hA) {
        int ia[IA], ib[IB];   // alpha side of every item is fixed for this hA
#pragma unroll
        for (int it = 0; it < IA; ++it) ia[it] = ap[it] >= 0 ? __ldg(P.idxA + (i64)hA * P.n + ap[it]) : -1;
#pragma unroll
        for (int it = 0; it < IB; ++it) ib[it] = bp[it] >= 0 ? __ldg(P.idxA + (i64)hA * P.n + bp[it]) : -1;
        for (int hB0 = 0; hB0 < P.nHb; hB0 += kTK) {
#pragma unroll
            for (int it = 0; it < IA; ++it) {
                const int hB = hB0 + ak[it];
                double v = 0.0;
                if (ia[it] >= 0 && hB < P.nHb) {
                    const int jb = __ldg(P.idxB + (i64)hB * P.n + ar[it]);
                    if (jb >= 0) v = signed_at(P.lt, (i64)(ia[it] >> 1) * P.nB + (jb >> 1), (ia[it] ^ jb) & 1);
                }
                As[ak[it]][(threadIdx.x + it * kNT) % kTM] = v;
            }
#pragma unroll
            for (int it = 0; it < IB; ++it) {
                const int hB = hB0 + bk[it];
                double v = 0.0;
                if (ib[it] >= 0 && hB < P.nHb) {
                    const int jb = __ldg(P.idxB + (i64)hB * P.n + br[it]);
                    if (jb >= 0) v = signed_at(P.rt, (i64)(ib[it] >> 1) * P.nB + (jb >> 1), (ib[it] ^ jb) & 1);
                }
                Bs[bk[it]][(threadIdx.x + it * kNT) % kTN] = v;
            }
            __syncthreads();
            acc.step(As, Bs);
            __syncthreads();
        }
    }
    acc.flush(P.C, P.M, m0, c0, P.M, P.M);
}

struct PairArgs {
    int npair, nB, nH2, nO, osplit;
    int spin;            // 0: pairs on the alpha index (rows of l~), 1: on the beta index (columns)
    const int *idx2;     // [nH2][npair]
    const double *lt, *rt;
    double *C;           // [npair][npair]
    const int *flag;     // as TabArgs::flag
};

// grid (ceil(npair / 64), ceil(npair / 128), min(nH2 * nos, 65535)), nos = ceil(nO / osplit).
// K = (h2, o), o the other spin's string: item z = h2 * nos + (range of osplit
// strings o); CTA z takes items z, z + gridDim.z, ... and each item in 32-row
// slices of o.  All items of a CTA add into the same output tile, flushed once.
__global__ void __launch_bounds__(kNT, 1) pair2_kernel(const PairArgs P)
{
    if (P.flag && *P.flag == 0) return;
    extern __shared__ __align__(16) double smem_pair[];
    double(*As)[kLS] = reinterpret_cast<double(*)[kLS]>(smem_pair);
    double(*Bs)[kXS] = reinterpret_cast<double(*)[kXS]>(smem_pair + kTK * kLS);
    const int m0 = blockIdx.x * kTM, c0 = blockIdx.y * kTN;
    const int nos = (P.nO + P.osplit - 1) / P.osplit;
    const i64 nitems = (i64)P.nH2 * nos;
    constexpr int IA = kTK * kTM / kNT, IB = kTK * kTN / kNT;
    int ak[IA], ja[IA], bk[IB], jb[IB];   // per fill item: slice row and pair column (or -1)
#pragma unroll
    for (int it = 0; it < IA; ++it) {
        const int i = threadIdx.x + it * kNT, j = m0 + i % kTM;
        ak[it] = i / kTM;
        ja[it] = j < P.npair ? j : -1;
    }
#pragma unroll
    for (int it = 0; it < IB; ++it) {
        const int i = threadIdx.x + it * kNT, j = c0 + i % kTN;
        bk[it] = i / kTN;
        jb[it] = j < P.npair ? j : -1;
    }
    Acc acc;
    acc.zero();
    for (i64 item = blockIdx.z; item < nitems; item += gridDim.z) {
        const int h2 = (int)(item / nos), o0 = (int)(item % nos) * P.osplit, o1 = min(P.nO, o0 + P.osplit);
        int ia[IA], ib[IB];
#pragma unroll
        for (int it = 0; it < IA; ++it) ia[it] = ja[it] >= 0 ? __ldg(P.idx2 + (i64)h2 * P.npair + ja[it]) : -1;
#pragma unroll
        for (int it = 0; it < IB; ++it) ib[it] = jb[it] >= 0 ? __ldg(P.idx2 + (i64)h2 * P.npair + jb[it]) : -1;
        for (int s0 = o0; s0 < o1; s0 += kTK) {
#pragma unroll
            for (int it = 0; it < IA; ++it) {
                const int o = s0 + ak[it];
                double v = 0.0;
                if (ia[it] >= 0 && o < o1) {
                    const i64 e = P.spin == 0 ? (i64)(ia[it] >> 1) * P.nB + o : (i64)o * P.nB + (ia[it] >> 1);
                    v = signed_at(P.lt, e, ia[it] & 1);
                }
                As[ak[it]][(threadIdx.x + it * kNT) % kTM] = v;
            }
#pragma unroll
            for (int it = 0; it < IB; ++it) {
                const int o = s0 + bk[it];
                double v = 0.0;
                if (ib[it] >= 0 && o < o1) {
                    const i64 e = P.spin == 0 ? (i64)(ib[it] >> 1) * P.nB + o : (i64)o * P.nB + (ib[it] >> 1);
                    v = signed_at(P.rt, e, ib[it] & 1);
                }
                Bs[bk[it]][(threadIdx.x + it * kNT) % kTN] = v;
            }
            __syncthreads();
            acc.step(As, Bs);
            __syncthreads();
        }
    }
    acc.flush(P.C, P.npair, m0, c0, P.npair, P.npair);
}

// D1a[p][q] = sum_r C[p n + r][q n + r] / nel_b, D1b[r][s] = sum_p C[p n + r][p n + s] / nel_a
__global__ void d1_kernel(int n, int nel_a, int nel_b, const double *__restrict__ C, double *__restrict__ D1a,
                          double *__restrict__ D1b, const int *__restrict__ flag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * n || (flag && *flag == 0)) return;
    const int x = i / n, y = i % n;
    const i64 M = (i64)n * n;
    double sa = 0.0, sb = 0.0;
    for (int k = 0; k < n; ++k) {
        sa += C[(i64)(x * n + k) * M + (y * n + k)];
        sb += C[(i64)(k * n + x) * M + (k * n + y)];
    }
    D1a[i] = nel_b > 0 ? sa / nel_b : 0.0;
    D1b[i] = nel_a > 0 ? sb / nel_a : 0.0;
}

struct Tables {
    int n, npair;
    const double *D1a, *D1b, *C, *C2a, *C2b;
};

// <a+_p a+_q a_r a_s> from C2[pq][rs] = <a+_p a+_q a_s a_r> (p > q, r > s)
__device__ __forceinline__ double g2(const double *C2, int npair, int p, int q, int r, int s)
{
    if (p == q || r == s || !C2) return 0.0;
    double sg = -1.0;
    if (p < q) { const int t = p; p = q; q = t; sg = -sg; }
    if (r < s) { const int t = r; r = s; s = t; sg = -sg; }
    return sg * C2[(i64)(p * (p - 1) / 2 + q) * npair + (r * (r - 1) / 2 + s)];
}

__device__ __forceinline__ double table_at(const Tables &T, int kind, int i0, int i1, int i2, int i3)
{
    const int n = T.n;
    switch (kind) {
    case BSIM_POOL_D1A: return T.D1a[i0 * n + i1];
    case BSIM_POOL_D1B: return T.D1b[i0 * n + i1];
    case BSIM_POOL_TAB: return T.C[(i64)(i0 * n + i2) * ((i64)n * n) + (i1 * n + i3)];
    case BSIM_POOL_GAA: return g2(T.C2a, T.npair, i0, i1, i2, i3);
    case BSIM_POOL_GBB: return g2(T.C2b, T.npair, i0, i1, i2, i3);
    default: return 0.0;
    }
}

// grads[g] = coef (X[dagger(i)] - X[i]); 0 for zero groups; general groups get
// NaN, or keep their value when keep_general is set (the pair-list kernels wrote it)
__global__ void assemble_kernel(i64 ngs, const int *__restrict__ kind, const int4 *__restrict__ idx,
                                const double *__restrict__ coef, Tables T, double *__restrict__ grads,
                                const int *__restrict__ flag, int keep_general)
{
    const i64 g = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngs || (flag && *flag == 0)) return;
    const int k = kind[g];
    if (k <= 0) {
        if (k == 0) grads[g] = 0.0;
        else if (!keep_general) grads[g] = __longlong_as_double(0x7ff8000000000000ll);
        return;
    }
    const int4 i = idx[g];
    double fwd = table_at(T, k, i.x, i.y, i.z, i.w), dag;
    if (k == BSIM_POOL_D1A || k == BSIM_POOL_D1B) dag = table_at(T, k, i.y, i.x, 0, 0);
    else if (k == BSIM_POOL_TAB) dag = table_at(T, k, i.y, i.x, i.w, i.z);
    else dag = table_at(T, k, i.w, i.z, i.y, i.x);
    grads[g] = coef[g] * (dag - fwd);
}

// ---- host ---------------------------------------------------------------------------
struct PoolDensity {
    unsigned magic = kPoolDensityMagic;
    const void *basis = nullptr;
    bool u64s = false;
    int n = 0, nA = 0, nB = 0, nel_a = 0, nel_b = 0;
    int nHa = 0, nHb = 0, nH2a = 0, nH2b = 0, npair = 0;
    i64 ngs = 0;
    bool embed = false;                  // blocked basis: scatter into the union-string arrays
    std::vector<int> blk_na, blk_nb, blk_as, blk_bs;
    std::vector<i64> blk_off;
    int *gA = nullptr, *gB = nullptr;    // [astrs.size()], [bstrs.size()]: union index of each block-list string
    Arena arena;
    int *idxA = nullptr, *idxB = nullptr, *idx2A = nullptr, *idx2B = nullptr, *kind = nullptr;
    int4 *idx = nullptr;
    double *coef = nullptr, *lt = nullptr, *rt = nullptr, *C = nullptr, *C2a = nullptr, *C2b = nullptr,
           *D1a = nullptr, *D1b = nullptr;
    ~PoolDensity() { arena.release(); magic = 0; }
};

// Hole table of one spin: hole strings (nel - holes electrons, every removal of
// `holes` electrons from a string of strs) in increasing order, and per hole
// string h and created orbital (holes = 1: orbital p; holes = 2: pair x > y at
// x (x - 1) / 2 + y, created as a+_x a+_y |h>, a+_y first) the entry
// (index of the created string in strs << 1) | sign, or -1.
template <typename S>
int hole_table(int norb, int holes, const std::vector<S> &strs, std::vector<u64> &hs, std::vector<int> &tab)
{
    if (holes < 1 || holes > 2 || norb < 1 || norb > 64) return BSIM_ERR_ARG;
    std::unordered_map<u64, int> where;
    where.reserve(strs.size() * 2);
    for (size_t i = 0; i < strs.size(); ++i) where[(u64)strs[i]] = (int)i;
    std::vector<u64> h;
    for (S s0 : strs) {
        const u64 s = (u64)s0;
        for (u64 m = s; m; m &= m - 1) {
            const u64 e1 = m & (~m + 1);
            if (holes == 1) { h.push_back(s ^ e1); continue; }
            for (u64 m2 = m & (m - 1); m2; m2 &= m2 - 1) h.push_back(s ^ e1 ^ (m2 & (~m2 + 1)));
        }
    }
    std::sort(h.begin(), h.end());
    h.erase(std::unique(h.begin(), h.end()), h.end());
    hs = h;
    const int w = holes == 1 ? norb : norb * (norb - 1) / 2;
    tab.assign(h.size() * (size_t)w, -1);
    auto below = [](u64 s, int o) { return __builtin_popcountll(s & ((1ull << o) - 1ull)); };   // o <= 63
    for (size_t k = 0; k < h.size(); ++k) {
        const u64 hk = h[k];
        if (holes == 1) {
            for (int p = 0; p < norb; ++p) {
                if ((hk >> p) & 1) continue;
                auto it = where.find(hk | (1ull << p));
                if (it == where.end()) continue;
                tab[k * w + p] = (it->second << 1) | (below(hk, p) & 1);
            }
        } else {
            for (int x = 1; x < norb; ++x)
                for (int y = 0; y < x; ++y) {
                    if (((hk >> x) & 1) || ((hk >> y) & 1)) continue;
                    auto it = where.find(hk | (1ull << x) | (1ull << y));
                    if (it == where.end()) continue;
                    const int par = below(hk, y) + below(hk | (1ull << y), x);
                    tab[k * w + x * (x - 1) / 2 + y] = (it->second << 1) | (par & 1);
                }
        }
    }
    return BSIM_OK;
}

template <typename Ti>
int density_create(const DevBasis<Ti> *B, i64 ngs, const int32_t *kind, const int32_t *idx, const double *coef,
                   PoolDensity **out, size_t max_bytes = ~size_t(0))
{
    if (B->nel_a < 1 || B->nel_b < 1) {
        set_error("pool density gradient: needs at least one electron of each spin");
        return BSIM_ERR_UNSUPPORTED;
    }
    const int n = B->norb, nbk = B->num_blocks;
    // union string lists (increasing); for one block they are the block's lists
    std::vector<Ti> as, bs;
    for (int k = 0; k < nbk; ++k) {
        as.insert(as.end(), B->astrs.begin() + B->astart[k], B->astrs.begin() + B->astart[k] + B->na[k]);
        bs.insert(bs.end(), B->bstrs.begin() + B->bstart[k], B->bstrs.begin() + B->bstart[k] + B->nb[k]);
    }
    std::sort(as.begin(), as.end());
    as.erase(std::unique(as.begin(), as.end()), as.end());
    std::sort(bs.begin(), bs.end());
    bs.erase(std::unique(bs.begin(), bs.end()), bs.end());
    const int nA = (int)as.size(), nB = (int)bs.size();
    // every launch size of density_grad is checked here, so a call never fails
    // after part of its work is queued: table entries are (index << 1) | sign in
    // an int, and the frame kernels put 256 beta strings per CTA on grid y
    if (as.size() >= (1u << 30) || bs.size() >= (1u << 30)) {
        set_error("pool density gradient: %zu alpha / %zu beta strings, above the 2^30 limit", as.size(), bs.size());
        return BSIM_ERR_TOO_LARGE;
    }
    if ((nB + 255) / 256 > 65535) {
        set_error("pool density gradient: %d beta strings, above the frame kernel's 65535 * 256", nB);
        return BSIM_ERR_TOO_LARGE;
    }
    for (i64 g = 0; g < ngs; ++g) {   // the assembly reads tables at these orbitals
        if (kind[g] < BSIM_POOL_GENERAL || kind[g] > BSIM_POOL_GBB) {
            set_error("pool density gradient: group %lld has kind %d", (long long)g, (int)kind[g]);
            return BSIM_ERR_ARG;
        }
        if (kind[g] > 0)
            for (int j = 0; j < 4; ++j)
                if (idx[4 * g + j] < 0 || idx[4 * g + j] >= n) {
                    set_error("pool density gradient: group %lld names orbital %d of a %d-orbital basis",
                              (long long)g, (int)idx[4 * g + j], n);
                    return BSIM_ERR_ARG;
                }
    }
    std::vector<int> gA(B->astrs.size(), 0), gB(B->bstrs.size(), 0);
    for (int k = 0; k < nbk; ++k) {
        for (int i = 0; i < B->na[k]; ++i)
            gA[B->astart[k] + i] =
                (int)(std::lower_bound(as.begin(), as.end(), B->astrs[B->astart[k] + i]) - as.begin());
        for (int i = 0; i < B->nb[k]; ++i)
            gB[B->bstart[k] + i] =
                (int)(std::lower_bound(bs.begin(), bs.end(), B->bstrs[B->bstart[k] + i]) - bs.begin());
    }
    std::vector<u64> hA, hB, h2A, h2B;
    std::vector<int> tA, tB, t2A, t2B;
    int st;
    if ((st = hole_table(n, 1, as, hA, tA)) != BSIM_OK) return st;
    if ((st = hole_table(n, 1, bs, hB, tB)) != BSIM_OK) return st;
    if (B->nel_a >= 2 && (st = hole_table(n, 2, as, h2A, t2A)) != BSIM_OK) return st;
    if (B->nel_b >= 2 && (st = hole_table(n, 2, bs, h2B, t2B)) != BSIM_OK) return st;
    auto *P = new PoolDensity;
    P->basis = B;
    P->u64s = sizeof(Ti) == 8;
    P->n = n; P->nA = nA; P->nB = nB; P->nel_a = B->nel_a; P->nel_b = B->nel_b;
    P->nHa = (int)hA.size(); P->nHb = (int)hB.size(); P->nH2a = (int)h2A.size(); P->nH2b = (int)h2B.size();
    P->npair = n * (n - 1) / 2;
    P->ngs = ngs;
    P->embed = nbk > 1;
    for (int k = 0; k < nbk; ++k) {
        P->blk_na.push_back(B->na[k]); P->blk_nb.push_back(B->nb[k]);
        P->blk_as.push_back(B->astart[k]); P->blk_bs.push_back(B->bstart[k]);
        P->blk_off.push_back(B->off[k]);
    }
    const i64 dim = (i64)nA * nB, M = (i64)n * n, np2 = (i64)P->npair * P->npair;
    const size_t bytes = 256 * 18 + sizeof(int) * (tA.size() + tB.size() + t2A.size() + t2B.size() + ngs) +
                         sizeof(int) * (gA.size() + gB.size()) +
                         sizeof(int4) * ngs + sizeof(double) * (ngs + 2 * dim + M * M + 2 * np2 + 2 * M);
    if (bytes > max_bytes) {
        delete P;
        set_error("pool density gradient: %zu bytes of tables above the limit of %zu", bytes, max_bytes);
        return BSIM_ERR_TOO_LARGE;
    }
    if ((st = P->arena.reserve(bytes)) != BSIM_OK) { delete P; return st; }
    P->idxA = P->arena.take<int>(tA.size());
    P->idxB = P->arena.take<int>(tB.size());
    P->idx2A = P->arena.take<int>(t2A.size());
    P->idx2B = P->arena.take<int>(t2B.size());
    P->kind = P->arena.take<int>(ngs);
    P->idx = P->arena.take<int4>(ngs);
    P->coef = P->arena.take<double>(ngs);
    P->lt = P->arena.take<double>(dim);
    P->rt = P->arena.take<double>(dim);
    P->C = P->arena.take<double>(M * M);
    P->C2a = P->arena.take<double>(np2);
    P->C2b = P->arena.take<double>(np2);
    P->D1a = P->arena.take<double>(M);
    P->D1b = P->arena.take<double>(M);
    P->gA = P->arena.take<int>(gA.size());
    P->gB = P->arena.take<int>(gB.size());
    auto up = [&](void *d, const void *h, size_t nb) { return nb ? cudaMemcpy(d, h, nb, cudaMemcpyHostToDevice) : cudaSuccess; };
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = up(P->idxA, tA.data(), sizeof(int) * tA.size());
    if (e == cudaSuccess) e = up(P->idxB, tB.data(), sizeof(int) * tB.size());
    if (e == cudaSuccess) e = up(P->idx2A, t2A.data(), sizeof(int) * t2A.size());
    if (e == cudaSuccess) e = up(P->idx2B, t2B.data(), sizeof(int) * t2B.size());
    if (e == cudaSuccess) e = up(P->kind, kind, sizeof(int) * ngs);
    if (e == cudaSuccess) e = up(P->idx, idx, sizeof(int4) * ngs);
    if (e == cudaSuccess) e = up(P->coef, coef, sizeof(double) * ngs);
    if (e == cudaSuccess) e = up(P->gA, gA.data(), sizeof(int) * gA.size());
    if (e == cudaSuccess) e = up(P->gB, gB.data(), sizeof(int) * gB.size());
    if (e != cudaSuccess) { delete P; return cuda_status(e, "pool density upload"); }
    *out = P;
    return BSIM_OK;
}

template <typename Ti>
int density_grad(PoolDensity *P, const double *l, const double *r, double *grads, cudaStream_t s,
                 const int *flag = nullptr, bool keep_general = false)
{
    const auto *B = static_cast<const DevBasis<Ti> *>(P->basis);
    const int n = P->n, nA = P->nA, nB = P->nB;
    const i64 M = (i64)n * n, np2 = (i64)P->npair * P->npair;
    if (!P->embed) {
        dim3 g(nA, (nB + 255) / 256);
        frame_pair_kernel<Ti><<<g, 256, 0, s>>>(nB, B->view.astrs + B->astart[0], B->view.bstrs + B->bstart[0], l, r,
                                                P->lt, P->rt, flag);
    } else {
        BSIM_CUDA(cudaMemsetAsync(P->lt, 0, sizeof(double) * (i64)nA * nB, s));
        BSIM_CUDA(cudaMemsetAsync(P->rt, 0, sizeof(double) * (i64)nA * nB, s));
        for (size_t k = 0; k < P->blk_na.size(); ++k) {
            const int nak = P->blk_na[k], nbk = P->blk_nb[k];
            if (nak == 0 || nbk == 0) continue;
            dim3 g(nak, (nbk + 255) / 256);
            embed_frame_kernel<Ti><<<g, 256, 0, s>>>(nbk, nB, B->view.astrs + P->blk_as[k], B->view.bstrs + P->blk_bs[k],
                                                     P->gA + P->blk_as[k], P->gB + P->blk_bs[k], l + P->blk_off[k],
                                                     r + P->blk_off[k], P->lt, P->rt, flag);
        }
    }
    BSIM_CUDA(cudaMemsetAsync(P->C, 0, sizeof(double) * M * M, s));
    BSIM_CUDA(cudaMemsetAsync(P->C2a, 0, sizeof(double) * np2, s));
    BSIM_CUDA(cudaMemsetAsync(P->C2b, 0, sizeof(double) * np2, s));
    if (P->nHa > 0 && P->nHb > 0) {
        TabArgs A{n, nB, P->nHa, P->nHb, (int)M, 0, P->idxA, P->idxB, P->lt, P->rt, P->C, flag};
        const int tiles = (int)(((M + kTM - 1) / kTM) * ((M + kTN - 1) / kTN));
        const int splits = std::max(1, std::min(P->nHa, (148 * 8 + tiles - 1) / tiles));
        A.hsplit = (P->nHa + splits - 1) / splits;
        dim3 g((unsigned)((M + kTM - 1) / kTM), (unsigned)((M + kTN - 1) / kTN),
               (unsigned)((P->nHa + A.hsplit - 1) / A.hsplit));   // at most 148 * 8 K splits
        BSIM_CUDA(cudaFuncSetAttribute(tab_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
        tab_kernel<<<g, kNT, kSmem, s>>>(A);
    }
    for (int spin = 0; spin < 2; ++spin) {
        const int nH2 = spin == 0 ? P->nH2a : P->nH2b, nO = spin == 0 ? nB : nA;
        if (nH2 == 0 || P->npair == 0) continue;
        PairArgs A{P->npair, nB, nH2, nO, 0, spin, spin == 0 ? P->idx2A : P->idx2B, P->lt, P->rt,
                   spin == 0 ? P->C2a : P->C2b, flag};
        const int tiles = ((P->npair + kTM - 1) / kTM) * ((P->npair + kTN - 1) / kTN);
        const int want = std::max(1, (148 * 8 + tiles * nH2 - 1) / (tiles * nH2));   // o-splits per hole string
        A.osplit = std::max(kTK, ((nO + want - 1) / want + kTK - 1) / kTK * kTK);
        const int nos = (nO + A.osplit - 1) / A.osplit;
        dim3 g((unsigned)((P->npair + kTM - 1) / kTM), (unsigned)((P->npair + kTN - 1) / kTN),
               (unsigned)std::min<i64>((i64)nH2 * nos, kMaxGridZ));
        BSIM_CUDA(cudaFuncSetAttribute(pair2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem));
        pair2_kernel<<<g, kNT, kSmem, s>>>(A);
    }
    d1_kernel<<<(unsigned)((M + 255) / 256), 256, 0, s>>>(n, P->nel_a, P->nel_b, P->C, P->D1a, P->D1b, flag);
    Tables T{n, P->npair, P->D1a, P->D1b, P->C, P->nH2a ? P->C2a : nullptr, P->nH2b ? P->C2b : nullptr};
    if (P->ngs > 0)
        assemble_kernel<<<(unsigned)((P->ngs + 255) / 256), 256, 0, s>>>(P->ngs, P->kind, P->idx, P->coef, T, grads,
                                                                          flag, keep_general ? 1 : 0);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

// ---- theta = 0 route of batchgrad --------------------------------------------------
__global__ void theta_zero_kernel(const double *__restrict__ thetas, i64 n, int *__restrict__ flag)
{
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        if (thetas[i] != 0.0) *flag = 0;   // every writer writes 0
}

}  // namespace

struct DensityRoute {
    const void *basis = nullptr;
    i64 basis_dim = 0;
    bool ok = false;                 // false: the route does not apply to this (basis, network)
    i64 ngs = 0;
    PoolDensity *P = nullptr;
    Arena arena;                     // skip mask and flag
    unsigned char *skip = nullptr;   // [ngs]: 1 for groups of a planned form (kind >= 0)
    int *flag = nullptr;             // nonzero: every theta of the current call is zero
    ~DensityRoute() { delete P; arena.release(); }
};

static std::mutex g_route_mu;

// Route for (B, N): groups classified by bsim_poolplan_classify from the
// network's host copy; applies when some group has a planned form and the
// dense tables take at most half of the free device memory (a blocked basis
// only when its union string arrays hold at most 4x its determinants).
// BSIM_POOL_DENSITY=0 turns the route off.
template <typename Ti>
int density_route(const DevBasis<Ti> *B, const DevNet<Ti> *N, DensityRoute **out)
{
    *out = nullptr;
    static const bool off = [] {
        const char *e = getenv("BSIM_POOL_DENSITY");
        return e && e[0] == '0';
    }();
    if (off || N->cplx || B->nel_a < 1 || B->nel_b < 1 || B->dim == 0 || N->ngs == 0 || B->norb > 64) return BSIM_OK;
    std::lock_guard<std::mutex> lk(g_route_mu);
    auto *R = static_cast<DensityRoute *>(N->density_state);
    if (R && R->basis == B && R->basis_dim == B->dim) {
        *out = R->ok ? R : nullptr;
        return BSIM_OK;
    }
    if (R) { delete R; const_cast<DevNet<Ti> *>(N)->density_state = nullptr; }
    R = new DensityRoute;
    R->basis = B;
    R->basis_dim = B->dim;
    R->ngs = N->ngs;
    auto &net = const_cast<DevNet<Ti> &>(*N);
    net.density_state = R;
    net.density_free = [](void *q) { delete static_cast<DensityRoute *>(q); };
    // the network in the flat form of bsim_poolplan_classify
    const i64 ngs = N->ngs;
    std::vector<uint64_t> axs(ngs), bxs(ngs), za, zb;
    std::vector<int64_t> ranks(ngs), nza(ngs), nzb(ngs);
    std::vector<double> wa, wb;
    for (i64 g = 0; g < ngs; ++g) {
        const GroupDev &G = N->groups[g];
        axs[g] = G.ax; bxs[g] = G.bx; ranks[g] = G.rank; nza[g] = G.nza; nzb[g] = G.nzb;
        for (int i = 0; i < G.nza; ++i) za.push_back((uint64_t)N->z[G.za_off + i]);
        for (int i = 0; i < G.nzb; ++i) zb.push_back((uint64_t)N->z[G.zb_off + i]);
        wa.insert(wa.end(), N->w.begin() + G.wa_off, N->w.begin() + G.wa_off + (i64)G.nza * G.rank);
        wb.insert(wb.end(), N->w.begin() + G.wb_off, N->w.begin() + G.wb_off + (i64)G.nzb * G.rank);
    }
    za.push_back(0); zb.push_back(0); wa.push_back(0.0); wb.push_back(0.0);   // never empty arrays
    std::vector<int32_t> kind(ngs), idx(4 * ngs);
    std::vector<double> coef(ngs);
    int st = bsim_poolplan_classify(B->norb, ngs, axs.data(), bxs.data(), ranks.data(), nza.data(), nzb.data(),
                                    za.data(), zb.data(), wa.data(), wb.data(), kind.data(), idx.data(), coef.data());
    if (st != BSIM_OK) return BSIM_OK;   // not applicable
    std::vector<unsigned char> skip(ngs);
    i64 planned = 0;
    for (i64 g = 0; g < ngs; ++g) planned += (skip[g] = kind[g] >= 0 ? 1 : 0);
    if (planned == 0) return BSIM_OK;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return cuda_status(cudaGetLastError(), "cudaMemGetInfo");
    if (B->num_blocks > 1) {   // union string arrays of a blocked basis
        std::vector<u64> as, bs;
        for (int k = 0; k < B->num_blocks; ++k) {
            for (int i = 0; i < B->na[k]; ++i) as.push_back((u64)B->astrs[B->astart[k] + i]);
            for (int i = 0; i < B->nb[k]; ++i) bs.push_back((u64)B->bstrs[B->bstart[k] + i]);
        }
        std::sort(as.begin(), as.end());
        std::sort(bs.begin(), bs.end());
        const double u = (double)(std::unique(as.begin(), as.end()) - as.begin()) *
                         (double)(std::unique(bs.begin(), bs.end()) - bs.begin());
        if (u > 4.0 * (double)B->dim) return BSIM_OK;
    }
    PoolDensity *P = nullptr;
    st = density_create(B, ngs, kind.data(), idx.data(), coef.data(), &P, free_b / 2);
    if (st == BSIM_ERR_TOO_LARGE || st == BSIM_ERR_UNSUPPORTED) { set_error(""); return BSIM_OK; }
    if (st != BSIM_OK) return st;
    R->P = P;
    if ((st = R->arena.reserve((size_t)ngs + 512)) != BSIM_OK) return st;
    R->flag = R->arena.take<int>(1);
    R->skip = R->arena.take<unsigned char>(ngs);
    BSIM_CUDA(cudaMemcpy(R->skip, skip.data(), (size_t)ngs, cudaMemcpyHostToDevice));
    R->ok = true;
    *out = R;
    return BSIM_OK;
}

int density_route_begin(DensityRoute *D, const double *thetas, cudaStream_t s)
{
    BSIM_CUDA(cudaMemsetAsync(D->flag, 0xff, sizeof(int), s));
    const unsigned grid = (unsigned)std::min<i64>(148 * 4, (D->ngs + 255) / 256);
    theta_zero_kernel<<<std::max(grid, 1u), 256, 0, s>>>(thetas, D->ngs, D->flag);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename Ti>
int density_route_finish(DensityRoute *D, const double *l, const double *r, double *grads, cudaStream_t s)
{
    return density_grad<Ti>(D->P, l, r, grads, s, D->flag, true);
}

const unsigned char *density_route_skip(const DensityRoute *D) { return D->skip; }
const int *density_route_flag(const DensityRoute *D) { return D->flag; }

template int density_route<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, DensityRoute **);
template int density_route<unsigned long long>(const DevBasis<unsigned long long> *,
                                               const DevNet<unsigned long long> *, DensityRoute **);
template int density_route_finish<unsigned>(DensityRoute *, const double *, const double *, double *, cudaStream_t);
template int density_route_finish<unsigned long long>(DensityRoute *, const double *, const double *, double *,
                                                      cudaStream_t);

}  // namespace bsim

extern "C" {

int bsim_pooldensity_hole_table(int64_t norb, int64_t holes, int64_t nstr, const uint64_t *strs, int64_t *nh,
                                int32_t *table)
{
    if (!strs || !nh) return bsim::BSIM_ERR_NULL;
    if (nstr < 1 || norb < 1 || norb > 64 || holes < 1 || holes > 2) return bsim::BSIM_ERR_ARG;
    std::vector<unsigned long long> s(strs, strs + nstr);
    std::vector<unsigned long long> hs;
    std::vector<int> tab;
    const int st = bsim::hole_table((int)norb, (int)holes, s, hs, tab);
    if (st != bsim::BSIM_OK) return st;
    *nh = (int64_t)hs.size();
    if (table) std::copy(tab.begin(), tab.end(), table);
    return bsim::BSIM_OK;
}

int bsim_pooldensity_create(void *basis, int64_t ngs, const int32_t *kind, const int32_t *idx, const double *coef,
                            void **out)
{
    if (!basis || !out || (ngs > 0 && (!kind || !idx || !coef))) return bsim::BSIM_ERR_NULL;
    if (ngs < 0) return bsim::BSIM_ERR_ARG;
    bsim::PoolDensity *P = nullptr;
    int st;
    if (bsim::is_u64_basis(basis)) {
        auto *B = static_cast<bsim::DevBasis<unsigned long long> *>(basis);
        if (!bsim::valid(B)) return bsim::BSIM_ERR_ARG;
        st = bsim::density_create(B, ngs, kind, idx, coef, &P);
    } else {
        auto *B = static_cast<bsim::DevBasis<unsigned> *>(basis);
        if (!bsim::valid(B)) return bsim::BSIM_ERR_ARG;
        st = bsim::density_create(B, ngs, kind, idx, coef, &P);
    }
    if (st == bsim::BSIM_OK) *out = P;
    return st;
}

int bsim_pooldensity_grad(void *plan, const double *l, const double *r, double *grads, bsim_stream_t stream)
{
    auto *P = static_cast<bsim::PoolDensity *>(plan);
    if (!P || !l || !r || (P->ngs > 0 && !grads)) return bsim::BSIM_ERR_NULL;
    if (P->magic != bsim::kPoolDensityMagic) return bsim::BSIM_ERR_ARG;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    return P->u64s ? bsim::density_grad<unsigned long long>(P, l, r, grads, s)
                   : bsim::density_grad<unsigned>(P, l, r, grads, s);
}

int bsim_pooldensity_destroy(void *plan)
{
    auto *P = static_cast<bsim::PoolDensity *>(plan);
    if (!P) return bsim::BSIM_ERR_NULL;
    if (P->magic != bsim::kPoolDensityMagic) return bsim::BSIM_ERR_ARG;
    delete P;
    return bsim::BSIM_OK;
}

}  // extern "C"
