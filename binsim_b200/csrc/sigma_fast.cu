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

// ---- 2/3. pure groups of one spin: row AXPY over the precomputed row lists -----------
template <typename T>
__global__ void __launch_bounds__(256)
pure_rows_kernel(const SideDev S, const SideCSR L, const T *__restrict__ in, double *__restrict__ out,
                 const double *__restrict__ PAd, const double *__restrict__ PBd, int rank_d)
{
    const int row = blockIdx.x;
    const int ncols = S.ncols;
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
    const i64 e_beg = L.cptr[row], e_end = L.cptr[row + 1];
    constexpr int kBatch = 64;   // FP32 partial sums span at most this many entries
    for (i64 e0 = e_beg; e0 < e_end; e0 += kBatch) {
        const i64 e1 = min(e_end, e0 + kBatch);
        T part[K];
#pragma unroll
        for (int k = 0; k < K; ++k) part[k] = T(0);
        i64 e = e0;
        for (; e + 4 <= e1; e += 4) {   // 4 entries x K columns of independent loads in flight
            const T *s0 = in + (i64)__ldg(L.csrc + e) * ncols, *s1 = in + (i64)__ldg(L.csrc + e + 1) * ncols;
            const T *s2 = in + (i64)__ldg(L.csrc + e + 2) * ncols, *s3 = in + (i64)__ldg(L.csrc + e + 3) * ncols;
            const T k0 = (T)__ldg(L.ccoef + e), k1 = (T)__ldg(L.ccoef + e + 1);
            const T k2 = (T)__ldg(L.ccoef + e + 2), k3 = (T)__ldg(L.ccoef + e + 3);
#pragma unroll
            for (int k = 0; k < K; ++k)
                if (col[k] < ncols) {
                    const T v0 = __ldg(s0 + col[k]), v1 = __ldg(s1 + col[k]);
                    const T v2 = __ldg(s2 + col[k]), v3 = __ldg(s3 + col[k]);
                    part[k] += k0 * v0 + k1 * v1 + k2 * v2 + k3 * v3;
                }
        }
        for (; e < e1; ++e) {
            const T cf = (T)__ldg(L.ccoef + e);
            const T *srow = in + (i64)__ldg(L.csrc + e) * ncols;
#pragma unroll
            for (int k = 0; k < K; ++k)
                if (col[k] < ncols) part[k] += cf * __ldg(srow + col[k]);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += (double)part[k];
    }
    for (i64 e = L.tptr[row]; e < L.tptr[row + 1]; ++e) {
        const int g = L.tgid[e];
        const int R = S.rank[g];
        const T *srow = in + (i64)L.tsrc[e] * ncols;
        const i64 toff = S.ctab_off[g];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (col[k] >= ncols) continue;
            double f = 0.0;
            for (int r = 0; r < R; ++r) f += L.tpa[e * kSideMaxRank + r] * S.ctab[toff + (i64)r * ncols + col[k]];
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
    const int *ranktab;     // colex byte tables
};

// colex rank from the byte tables (strings of up to 24 orbitals)
__device__ __forceinline__ int rank_bytes(unsigned s, const int *__restrict__ t)
{
    const unsigned b0 = s & 255u, b1 = (s >> 8) & 255u, b2 = (s >> 16) & 255u;
    const int o1 = __popc(b0), o2 = o1 + __popc(b1);
    return t[b0] + t[256 + b1 * 9 + o1] + t[256 + 256 * 9 + b2 * 17 + o2];
}

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

constexpr int kGemmThreads = 512;

// One CTA per source row a'.  Warp w owns excitations 4w..4w+3 of the row's
// connected list, lane l owns columns 4l..4l+3 of a kMixCols-column chunk.
template <typename Ti, typename T>
__global__ void __launch_bounds__(kGemmThreads, 1)
mixed_gemm_kernel(const MixedArgs P, const Ti *__restrict__ astr, const Ti *__restrict__ bstr,
                  const T *__restrict__ ct, T *__restrict__ Z, int z0, int W)
{
    using V2 = typename Vec2<T>::type;
    constexpr int NW = kGemmThreads / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nB = P.nB, K = P.nF, M = P.M;
    T *srow = reinterpret_cast<T *>(smem_raw);                               // [nB]
    T *lam = srow + ((nB + 7) & ~7);                                          // [K][64]
    T *xs = lam + (size_t)K * 64;                                             // [32][kMixCols]
    int *rtab = reinterpret_cast<int *>(xs + 32 * kMixCols);                  // [kRankTabInts]
    unsigned long long *cstr = reinterpret_cast<unsigned long long *>(rtab + kRankTabInts);   // [kMixCols]
    int *conn = reinterpret_cast<int *>(cstr + kMixCols);                     // [64]
    int *sgn = conn + 64;                                                     // [64]
    __shared__ int wcnt[NW], cnt;
    const int a = blockIdx.x;
    const u64 sa = (u64)astr[a];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kRankTabInts; i += blockDim.x) rtab[i] = P.ranktab[i];
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
        if (threadIdx.x == 0) for (int w2 = 0; w2 < NW; ++w2) cnt += wcnt[w2];
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
    const int zend = min(nB, z0 + W);
    const bool active = wid * 4 < m;
    for (int cb = z0; cb < zend; cb += kMixCols) {
        __syncthreads();
        for (int i = threadIdx.x; i < kMixCols; i += blockDim.x)
            cstr[i] = (cb + i < zend) ? (unsigned long long)bstr[cb + i] : 0ull;
        T acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = T(0);
        for (int f0 = 0; f0 < K; f0 += 32) {
            const int nf = min(32, K - f0);
            __syncthreads();
            // X slice: X[f][col] = sB_F(b^F) c~[a', rank(b^F)] for connected (F, b), else 0
            for (int i = threadIdx.x; i < 32 * kMixCols; i += blockDim.x) {
                const int f = i / kMixCols, cl = i % kMixCols;
                T x = T(0);
                if (f < nf && cb + cl < zend) {
                    const u64 bs = cstr[cl], fm = P.Fmask[f0 + f];
                    if (__popcll(bs & fm) == 1) {
                        const u64 sv = bs ^ fm;
                        x = srow[rank_bytes((unsigned)sv, rtab)];
                        if (__popcll(sv & P.mB[f0 + f]) & 1) x = -x;
                    }
                }
                xs[i] = x;
            }
            __syncthreads();
            if (active) {
#pragma unroll 4
                for (int f = 0; f < nf; ++f) {
                    const V2 *lr = reinterpret_cast<const V2 *>(lam + (size_t)(f0 + f) * 64 + wid * 4);
                    const V2 *xr = reinterpret_cast<const V2 *>(xs + f * kMixCols + 4 * lane);
                    const V2 xa = xr[0], xb = xr[1];
                    const V2 la = lr[0], lb = lr[1];
                    const T l[4] = {la.x, la.y, lb.x, lb.y};
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        acc[i][0] += l[i] * xa.x;
                        acc[i][1] += l[i] * xa.y;
                        acc[i][2] += l[i] * xb.x;
                        acc[i][3] += l[i] * xb.y;
                    }
                }
            }
        }
        if (active) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int j = wid * 4 + i;
                if (j >= m) break;
                T *zr = Z + ((i64)a * M + j) * W;
                const int b = cb + 4 * lane;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (b + q < zend) zr[b + q - z0] = acc[i][q];
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
        pure_rows_kernel<T><<<g, 256, 0, s>>>(P.sideA, P.csrA, ct, dst, P.rank_d ? P.d_PAd : nullptr, P.d_PBd,
                                              P.rank_d);
    }
    // 3. pure beta on the transposed vector -> tT
    {
        dim3 g(nB, (nA + kRowChunk - 1) / kRowChunk);
        pure_rows_kernel<T><<<g, 256, 0, s>>>(P.sideB, P.csrB, ctT, tT, nullptr, nullptr, 0);
    }
    // 4. mixed
    if (P.nE > 0 && P.nF > 0 && P.M > 0) {
        const size_t per_col = (size_t)nA * P.M * sizeof(T);
        size_t Wz = std::max<size_t>(kMixCols, (scratch_budget() / per_col) / kMixCols * kMixCols);
        Wz = std::min<size_t>(Wz, ((size_t)nB + kMixCols - 1) / kMixCols * kMixCols);
        if ((rc = ensure(&S.Z, &S.z_n, per_col * Wz)) != BSIM_OK) return rc;
        MixedArgs ma{nA, nB, P.nE, P.nF, P.M, P.norb, P.d_Emask, P.d_Fmask, P.d_mA, P.d_mB,
                     sizeof(T) == 8 ? (const void *)P.d_Lam : (const void *)P.d_Lam32, P.d_ranktab};
        const size_t smem = mixed_smem_bytes(nB, P.nF, sizeof(T));
        if (smem > 227 * 1024) { set_error("mixed kernel needs %zu bytes of shared memory", smem); return BSIM_ERR_UNSUPPORTED; }
        BSIM_CUDA(cudaFuncSetAttribute(mixed_gemm_kernel<Ti, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        T *Z = static_cast<T *>(S.Z);
        for (int z0 = 0; z0 < nB; z0 += (int)Wz) {
            mixed_gemm_kernel<Ti, T><<<nA, kGemmThreads, smem, s>>>(ma, P.d_astr, P.d_bstr, ct, Z, z0, (int)Wz);
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
