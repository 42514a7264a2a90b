// Structured sigma (single-block bases): see fastplan.h for the frame.
//
// Per sigma application, with c~ = eps * c:
//   1. frame_transpose : c~ (row-major) and c~^T                       [HBM streaming]
//   2. pure_rows(alpha): s~ = D * c~ + sum_pure-alpha PA(a') PB(b) c~[a', b]
//   3. pure_rows(beta) : t  = same on c~^T with the pure-beta groups
//   4. per column tile of the intermediate Z:
//        mixed_gemm   : for every source row a', X[F][b] = sB_F c~[a', b^F] is
//                       gathered once and Y = Lam_conn(a') X (FP64/FP32 register-
//                       blocked GEMM, 8 excitations x 2 columns per thread),
//                       Z[a'][j][b] = sA_E(a') Y[j][b]
//        mixed_gather : s~[a, b] += sum_E Z[a^E][j(E)][b]               [coalesced]
//   5. final: sigma = eps * (s~ + t^T)
// Step 2/3 read source rows coalesced; the grid runs column-chunk-major so the
// chunk of every source row stays in L2 while all destination rows use it.
#include "fastplan.h"
#include "ops.h"
#include "tiles.cuh"

#include <cstdlib>
#include <mutex>

namespace bsim {

constexpr int kRowChunk = 1024;        // columns per CTA in the row kernels
constexpr int kMaxTab = 512;           // table-mode pure groups connected to one row

// ---- colex rank of a string (index in Gosper order of all strings with its popcount)
__device__ __forceinline__ int colex_rank(u64 s, const int *__restrict__ binom)
{
    int r = 0, i = 1;
    while (s) {
        const int p = __ffsll((long long)s) - 1;
        r += binom[p * 33 + i];
        ++i;
        s &= s - 1;
    }
    return r;
}

// ---- 1. frame + transpose ---------------------------------------------------------
template <typename Ti, typename Tin, typename T>
__global__ void frame_transpose_kernel(int nA, int nB, const Ti *__restrict__ astr_unused,
                                       const Ti *__restrict__ bstr, const u64 *__restrict__ Ka,
                                       const Tin *__restrict__ c, T *__restrict__ ct, T *__restrict__ ctT)
{
    __shared__ T tile[32][33];
    const int b0 = blockIdx.x * 32, a0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int i = ty; i < 32; i += blockDim.y) {
        const int a = a0 + i, b = b0 + tx;
        T v = T(0);
        if (a < nA && b < nB) {
            const i64 idx = (i64)a * nB + b;
            v = (T)c[idx];
            if (par((u64)bstr[b] & Ka[a])) v = -v;
            ct[idx] = v;
        }
        tile[i][tx] = v;
    }
    __syncthreads();
    for (int i = ty; i < 32; i += blockDim.y) {
        const int b = b0 + i, a = a0 + tx;
        if (a < nA && b < nB) ctT[(i64)b * nA + a] = tile[tx][i];
    }
}

// ---- 2/3. pure groups of one spin: row AXPY --------------------------------------
template <typename Ti, typename T>
__global__ void __launch_bounds__(256)
pure_rows_kernel(const SideDev S, int nrows, const Ti *__restrict__ rowstr, const int *__restrict__ rowmap,
                 int norb, const T *__restrict__ in, double *__restrict__ out, const double *__restrict__ PAd,
                 const double *__restrict__ PBd, int rank_d)
{
    // dynamic shared memory: [cap_c] src, [cap_c] coef, [cap_t] src, gid, [cap_t][4] pa
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int cap_c = S.ng, cap_t = min(S.ng, kMaxTab);
    double *ccoef = reinterpret_cast<double *>(smem_raw);
    double *tpa = ccoef + cap_c;                                  // [cap_t * kSideMaxRank]
    int *csrc = reinterpret_cast<int *>(tpa + (size_t)cap_t * kSideMaxRank);
    int *tsrc = csrc + cap_c;
    int *tgid = tsrc + cap_t;
    __shared__ int wcount[2][8], wbase[2][8];
    __shared__ int ntot[2];
    const int row = blockIdx.x;
    const int ncols = S.ncols;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const u64 s0 = (u64)rowstr[row];
    if (threadIdx.x < 2) ntot[threadIdx.x] = 0;
    __syncthreads();
    // phase 1: connected groups of this row, compacted in group order
    for (int base = 0; base < S.ng; base += blockDim.x) {
        const int g = base + threadIdx.x;
        int src = -1, mode = 0;
        double pa[kSideMaxRank] = {0.0, 0.0, 0.0, 0.0};
        double coef = 0.0;
        if (g < S.ng) {
            const u64 x = S.x[g];
            const u64 s = s0 ^ x;
            if (((s >> norb) == 0) && 2 * __popcll(s0 & x) == __popcll(x)) src = rowmap[s];
            if (src >= 0) {
                const int R = S.rank[g], nz = S.nz[g];
                const u64 *z = S.zmask + S.z_off[g];
                const double *w = S.w + S.w_off[g];
                for (int q = 0; q < nz; ++q) {
                    const bool odd = __popcll(s & z[q]) & 1;
                    for (int r = 0; r < R; ++r) {
                        const double v = w[(i64)r * nz + q];
                        pa[r] += odd ? -v : v;
                    }
                }
                mode = S.colmode[g];
                if (mode == 0)
                    for (int r = 0; r < R; ++r) coef += pa[r] * S.cconst[g * kSideMaxRank + r];
            }
        }
        const unsigned mc = __ballot_sync(0xffffffffu, src >= 0 && mode == 0);
        const unsigned mt = __ballot_sync(0xffffffffu, src >= 0 && mode == 1);
        if (lane == 0) { wcount[0][wid] = __popc(mc); wcount[1][wid] = __popc(mt); }
        __syncthreads();
        if (threadIdx.x < 2) {
            int acc = ntot[threadIdx.x];
            for (int w2 = 0; w2 < 8; ++w2) { wbase[threadIdx.x][w2] = acc; acc += wcount[threadIdx.x][w2]; }
            ntot[threadIdx.x] = acc;
        }
        __syncthreads();
        const unsigned below = (1u << lane) - 1u;
        if (src >= 0 && mode == 0) {
            const int pos = wbase[0][wid] + __popc(mc & below);
            if (pos < cap_c) { csrc[pos] = src; ccoef[pos] = coef; }
        } else if (src >= 0) {
            const int pos = wbase[1][wid] + __popc(mt & below);
            if (pos < cap_t) {
                tsrc[pos] = src; tgid[pos] = g;
                for (int r = 0; r < kSideMaxRank; ++r) tpa[pos * kSideMaxRank + r] = pa[r];
            }
        }
        __syncthreads();
    }
    const int nc = min(ntot[0], cap_c), nt = min(ntot[1], cap_t);
    // phase 2: one column chunk
    const int c0 = blockIdx.y * kRowChunk;
    constexpr int K = kRowChunk / 256;
    double acc[K];
    int col[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        col[k] = c0 + threadIdx.x + k * 256;
        acc[k] = 0.0;
        if (PAd && col[k] < ncols) {
            double d = 0.0;
            for (int r = 0; r < rank_d; ++r) d += PAd[(i64)row * rank_d + r] * PBd[(i64)col[k] * rank_d + r];
            acc[k] = d * (double)in[(i64)row * ncols + col[k]];
        }
    }
    constexpr int kBatch = 64;
    for (int e0 = 0; e0 < nc; e0 += kBatch) {
        const int e1 = min(nc, e0 + kBatch);
        T part[K];
#pragma unroll
        for (int k = 0; k < K; ++k) part[k] = T(0);
        for (int e = e0; e < e1; ++e) {
            const T cf = (T)ccoef[e];
            const T *srow = in + (i64)csrc[e] * ncols;
#pragma unroll
            for (int k = 0; k < K; ++k)
                if (col[k] < ncols) part[k] += cf * __ldg(srow + col[k]);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += (double)part[k];
    }
    for (int e = 0; e < nt; ++e) {
        const int g = tgid[e];
        const int R = S.rank[g];
        const T *srow = in + (i64)tsrc[e] * ncols;
        const i64 toff = S.ctab_off[g];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (col[k] >= ncols) continue;
            double f = 0.0;
            for (int r = 0; r < R; ++r) f += tpa[e * kSideMaxRank + r] * S.ctab[toff + (i64)r * ncols + col[k]];
            acc[k] += f * (double)__ldg(srow + col[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (col[k] < ncols) out[(i64)row * ncols + col[k]] = acc[k];
}

// ---- 4a. mixed GEMM -----------------------------------------------------------------
struct MixedArgs {
    int nA, nB, nE, nF, M, norb;
    const u64 *Emask, *Fmask, *mA, *mB;
    const void *Lam;        // T [nE x nF]
    const int *binom;
};

template <typename Ti, typename T>
__global__ void __launch_bounds__(256, 1)
mixed_gemm_kernel(const MixedArgs P, const Ti *__restrict__ astr, const Ti *__restrict__ bstr,
                  const T *__restrict__ ct, T *__restrict__ Z, int z0, int W)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nB = P.nB, K = P.nF, M = P.M;
    T *srow = reinterpret_cast<T *>(smem_raw);                               // [nB]
    T *lam = srow + ((nB + 7) & ~7);                                          // [K][64]
    T *xs = lam + (size_t)K * 64;                                             // [32][64]
    int *binom = reinterpret_cast<int *>(xs + 32 * 64);                       // [33*33]
    int *conn = binom + 33 * 33;                                              // [64]
    int *sgn = conn + 64;                                                     // [64]
    __shared__ int wcnt[8], cnt;
    const int a = blockIdx.x;
    const u64 sa = (u64)astr[a];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < 33 * 33; i += blockDim.x) binom[i] = P.binom[i];
    // connected alpha excitations of this source row, in E order
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (int base = 0; base < P.nE; base += blockDim.x) {
        const int e = base + threadIdx.x;
        const bool ok = e < P.nE && __popcll(sa & P.Emask[e]) == 1;
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (lane == 0) wcnt[wid] = __popc(m);
        __syncthreads();
        int off = cnt;
        for (int w2 = 0; w2 < wid; ++w2) off += wcnt[w2];
        if (ok) {
            const int j = off + __popc(m & ((1u << lane) - 1u));
            if (j < 64) { conn[j] = e; sgn[j] = (__popcll(sa & P.mA[e]) & 1) ? -1 : 1; }
        }
        __syncthreads();
        if (threadIdx.x == 0) for (int w2 = 0; w2 < 8; ++w2) cnt += wcnt[w2];
        __syncthreads();
    }
    const int m = min(cnt, 64);
    // stage the source row and Lam restricted to the connected excitations (signs folded)
    const T *crow = ct + (i64)a * nB;
    for (int b = threadIdx.x; b < nB; b += blockDim.x) srow[b] = crow[b];
    const T *Lam = static_cast<const T *>(P.Lam);
    for (int i = threadIdx.x; i < K * 64; i += blockDim.x) {
        const int f = i >> 6, j = i & 63;
        lam[i] = j < m ? (T)sgn[j] * Lam[(i64)conn[j] * K + f] : T(0);
    }
    __syncthreads();
    const int zend = min(nB, z0 + W);
    for (int cb = z0; cb < zend; cb += 64) {
        T acc[8][2];
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = T(0);
        for (int f0 = 0; f0 < K; f0 += 32) {
            const int nf = min(32, K - f0);
            __syncthreads();
            for (int i = threadIdx.x; i < 32 * 64; i += blockDim.x) {
                const int f = i >> 6, cl = i & 63, b = cb + cl;
                T x = T(0);
                if (f < nf && b < zend) {
                    const u64 bs = (u64)bstr[b], fm = P.Fmask[f0 + f];
                    if (__popcll(bs & fm) == 1) {
                        const u64 s = bs ^ fm;
                        x = srow[colex_rank(s, binom)];
                        if (__popcll(s & P.mB[f0 + f]) & 1) x = -x;
                    }
                }
                xs[i] = x;
            }
            __syncthreads();
            if (wid * 8 < m) {
                for (int f = 0; f < nf; ++f) {
                    const T *lr = lam + (size_t)(f0 + f) * 64 + wid * 8;
                    const T x0 = xs[f * 64 + 2 * lane], x1 = xs[f * 64 + 2 * lane + 1];
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const T l = lr[i];
                        acc[i][0] += l * x0;
                        acc[i][1] += l * x1;
                    }
                }
            }
        }
        if (wid * 8 < m) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int j = wid * 8 + i;
                if (j >= m) break;
                T *zr = Z + ((i64)a * M + j) * W;
                const int b = cb + 2 * lane;
                if (b < zend) zr[b - z0] = acc[i][0];
                if (b + 1 < zend) zr[b + 1 - z0] = acc[i][1];
            }
        }
    }
}

// ---- 4b. gather of the mixed contributions ------------------------------------------------
template <typename Ti, typename T>
__global__ void __launch_bounds__(256)
mixed_gather_kernel(const MixedArgs P, const Ti *__restrict__ astr, const int *__restrict__ amap,
                    const T *__restrict__ Z, double *__restrict__ sig, int z0, int W)
{
    __shared__ int esrc[64], ej[64];
    __shared__ int wcnt[8], cnt;
    const int a = blockIdx.x;
    const u64 s0 = (u64)astr[a];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (int base = 0; base < P.nE; base += blockDim.x) {
        const int e = base + threadIdx.x;
        bool ok = false;
        int src = -1, j = 0;
        if (e < P.nE && __popcll(s0 & P.Emask[e]) == 1) {
            const u64 s = s0 ^ P.Emask[e];
            src = amap[s];
            for (int e2 = 0; e2 < e; ++e2) j += __popcll(s & P.Emask[e2]) == 1;
            ok = src >= 0 && j < 64;
        }
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (lane == 0) wcnt[wid] = __popc(m);
        __syncthreads();
        int off = cnt;
        for (int w2 = 0; w2 < wid; ++w2) off += wcnt[w2];
        if (ok) {
            const int p = off + __popc(m & ((1u << lane) - 1u));
            if (p < 64) { esrc[p] = src; ej[p] = j; }
        }
        __syncthreads();
        if (threadIdx.x == 0) for (int w2 = 0; w2 < 8; ++w2) cnt += wcnt[w2];
        __syncthreads();
    }
    const int n = min(cnt, 64);
    const int zend = min(P.nB, z0 + W);
    for (int b = z0 + blockIdx.y * kRowChunk + threadIdx.x; b < min(zend, z0 + (blockIdx.y + 1) * kRowChunk);
         b += blockDim.x) {
        T part = T(0);
        for (int e = 0; e < n; ++e) part += __ldg(Z + ((i64)esrc[e] * P.M + ej[e]) * W + (b - z0));
        sig[(i64)a * P.nB + b] += (double)part;
    }
}

// ---- 5. final: sigma = eps * (s~ + t^T) ---------------------------------------------
template <typename Ti>
__global__ void final_kernel(int nA, int nB, const Ti *__restrict__ bstr, const u64 *__restrict__ Ka,
                             const double *__restrict__ tT, double *__restrict__ sig)
{
    __shared__ double tile[32][33];
    const int b0 = blockIdx.x * 32, a0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int i = ty; i < 32; i += blockDim.y) {   // t^T tile: rows b, cols a
        const int b = b0 + i, a = a0 + tx;
        tile[i][tx] = (a < nA && b < nB) ? tT[(i64)b * nA + a] : 0.0;
    }
    __syncthreads();
    for (int i = ty; i < 32; i += blockDim.y) {
        const int a = a0 + i, b = b0 + tx;
        if (a < nA && b < nB) {
            const i64 idx = (i64)a * nB + b;
            double v = sig[idx] + tile[tx][i];
            if (par((u64)bstr[b] & Ka[a])) v = -v;
            sig[idx] = v;
        }
    }
}

// ---- host ------------------------------------------------------------------------------------
static size_t pure_smem(int ng)
{
    const size_t ct = (size_t)std::min(ng, kMaxTab);
    return std::max<size_t>(16, (size_t)ng * (8 + 4) + ct * (kSideMaxRank * 8 + 8));
}

template <typename Ti>
struct FastScratch {
    void *ct = nullptr, *ctT = nullptr, *Z = nullptr, *tT = nullptr;
    size_t ct_n = 0, ctT_n = 0, z_n = 0, tT_n = 0;
    ~FastScratch() {
        for (void *p : {ct, ctT, Z, tT})
            if (p) cudaFree(p);
    }
};

template <typename Ti>
struct FastState {
    FastPlan<Ti> plan;
    FastScratch<Ti> scratch;
};

static std::mutex g_fast_mu;

template <typename Ti>
static int get_fast(const DevBasis<Ti> *B, const DevNet<Ti> *N, FastState<Ti> **out)
{
    std::lock_guard<std::mutex> lk(g_fast_mu);
    auto *st = static_cast<FastState<Ti> *>(N->fast_state);
    if (st && st->plan.basis == B && st->plan.basis_dim == B->dim) { *out = st; return BSIM_OK; }
    if (st) { delete st; const_cast<DevNet<Ti> *>(N)->fast_state = nullptr; }
    st = new FastState<Ti>();
    int rc = build_fast_plan(B, N, &st->plan);
    if (rc != BSIM_OK) { delete st; return rc; }
    const_cast<DevNet<Ti> *>(N)->fast_state = st;
    const_cast<DevNet<Ti> *>(N)->fast_free = [](void *p) { delete static_cast<FastState<Ti> *>(p); };
    *out = st;
    return BSIM_OK;
}

static size_t scratch_budget()
{
    const char *e = getenv("BSIM_SIGMA_SCRATCH_GB");
    double gb = e ? atof(e) : 24.0;
    if (gb < 0.05) gb = 0.05;
    return (size_t)(gb * 1e9);
}

static int ensure(void **p, size_t *have, size_t bytes)
{
    if (*have >= bytes && *p) return BSIM_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *have = 0;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) { *p = nullptr; return cuda_status(e, "sigma scratch"); }
    *have = bytes;
    return BSIM_OK;
}

template <typename Ti>
bool fast_sigma_available(const DevBasis<Ti> *B, const DevNet<Ti> *N)
{
    FastState<Ti> *st = nullptr;
    if (get_fast(B, N, &st) != BSIM_OK) return false;
    return st->plan.ok;
}

template <typename Ti, typename T>
static int run_fast(const DevBasis<Ti> *B, const DevNet<Ti> *N, FastState<Ti> *st, const double *src,
                    const float *src32, double *dst, cudaStream_t s)
{
    FastPlan<Ti> &P = st->plan;
    FastScratch<Ti> &S = st->scratch;
    const int nA = P.nA, nB = P.nB;
    const size_t dim = (size_t)nA * nB;
    int rc;
    if ((rc = ensure(&S.ct, &S.ct_n, dim * sizeof(T))) != BSIM_OK) return rc;
    if ((rc = ensure(&S.ctT, &S.ctT_n, dim * sizeof(T))) != BSIM_OK) return rc;
    if ((rc = ensure(&S.tT, &S.tT_n, dim * sizeof(double))) != BSIM_OK) return rc;
    T *ct = static_cast<T *>(S.ct), *ctT = static_cast<T *>(S.ctT);
    double *tT = static_cast<double *>(S.tT);
    // 1. frame + transpose
    dim3 tgrid((nB + 31) / 32, (nA + 31) / 32), tblk(32, 8);
    if (src32) frame_transpose_kernel<Ti, float, T><<<tgrid, tblk, 0, s>>>(nA, nB, P.d_astr, P.d_bstr, P.d_Ka, src32, ct, ctT);
    else frame_transpose_kernel<Ti, double, T><<<tgrid, tblk, 0, s>>>(nA, nB, P.d_astr, P.d_bstr, P.d_Ka, src, ct, ctT);
    // 2. pure alpha + diagonal -> dst (the frame's s~)
    {
        dim3 g(nA, (nB + kRowChunk - 1) / kRowChunk);
        const size_t sm = pure_smem(P.sideA.ng);
        BSIM_CUDA(cudaFuncSetAttribute(pure_rows_kernel<Ti, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        pure_rows_kernel<Ti, T><<<g, 256, sm, s>>>(P.sideA, nA, P.d_astr, B->view.amap, P.norb, ct, dst,
                                                  P.rank_d ? P.d_PAd : nullptr, P.d_PBd, P.rank_d);
    }
    // 3. pure beta on the transposed vector -> tT
    {
        dim3 g(nB, (nA + kRowChunk - 1) / kRowChunk);
        const size_t sm = pure_smem(P.sideB.ng);
        BSIM_CUDA(cudaFuncSetAttribute(pure_rows_kernel<Ti, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        pure_rows_kernel<Ti, T><<<g, 256, sm, s>>>(P.sideB, nB, P.d_bstr, B->view.bmap, P.norb, ctT, tT, nullptr,
                                                  nullptr, 0);
    }
    // 4. mixed
    if (P.nE > 0 && P.nF > 0 && P.M > 0) {
        const size_t per_col = (size_t)nA * P.M * sizeof(T);
        size_t Wz = std::max<size_t>(64, (scratch_budget() / per_col) / 64 * 64);
        Wz = std::min<size_t>(Wz, ((size_t)nB + 63) / 64 * 64);
        if ((rc = ensure(&S.Z, &S.z_n, per_col * Wz)) != BSIM_OK) return rc;
        MixedArgs ma{nA, nB, P.nE, P.nF, P.M, P.norb, P.d_Emask, P.d_Fmask, P.d_mA, P.d_mB,
                     sizeof(T) == 8 ? (const void *)P.d_Lam : (const void *)P.d_Lam32, P.d_binom};
        const size_t smem = mixed_smem_bytes(nB, P.nF, sizeof(T));
        if (smem > 227 * 1024) { set_error("mixed kernel needs %zu bytes of shared memory", smem); return BSIM_ERR_UNSUPPORTED; }
        BSIM_CUDA(cudaFuncSetAttribute(mixed_gemm_kernel<Ti, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        T *Z = static_cast<T *>(S.Z);
        for (int z0 = 0; z0 < nB; z0 += (int)Wz) {
            mixed_gemm_kernel<Ti, T><<<nA, 256, smem, s>>>(ma, P.d_astr, P.d_bstr, ct, Z, z0, (int)Wz);
            dim3 g(nA, (unsigned)((std::min<size_t>(Wz, nB - z0) + kRowChunk - 1) / kRowChunk));
            mixed_gather_kernel<Ti, T><<<g, 256, 0, s>>>(ma, P.d_astr, B->view.amap, Z, dst, z0, (int)Wz);
        }
    }
    // 5. final combine
    final_kernel<Ti><<<tgrid, tblk, 0, s>>>(nA, nB, P.d_bstr, P.d_Ka, tT, dst);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename Ti>
int sigma_fast(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *src, const float *src32, double *dst,
               bool mixed, cudaStream_t s, bool *used)
{
    *used = false;
    FastState<Ti> *st = nullptr;
    int rc = get_fast(B, N, &st);
    if (rc != BSIM_OK) return rc;
    if (!st->plan.ok || (mixed ? !st->plan.fits32 : !st->plan.fits64)) return BSIM_OK;
    rc = mixed ? run_fast<Ti, float>(B, N, st, src, src32, dst, s) : run_fast<Ti, double>(B, N, st, src, nullptr, dst, s);
    if (rc != BSIM_OK) return rc;
    if (!st->plan.residual.empty()) {
        rc = sigma_generic_accumulate(B, N, st->plan.d_resid, st->plan.d_resid_chunks, st->plan.n_resid_chunks, src,
                                      src32, dst, mixed, s);
        if (rc != BSIM_OK) return rc;
    }
    *used = true;
    return BSIM_OK;
}

template <typename Ti>
int fast_sigma_info(const DevBasis<Ti> *B, const DevNet<Ti> *N, std::string *why, int *nresid)
{
    FastState<Ti> *st = nullptr;
    int rc = get_fast(B, N, &st);
    if (rc != BSIM_OK) return rc;
    *why = st->plan.ok ? "structured" : st->plan.why;
    *nresid = (int)st->plan.residual.size();
    return st->plan.ok ? (st->plan.fits64 ? 1 : 2) : 0;
}

template int fast_sigma_info<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, std::string *, int *);
template bool fast_sigma_available<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *);
template int sigma_fast<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, const double *, const float *,
                                  double *, bool, cudaStream_t, bool *);

}  // namespace bsim
