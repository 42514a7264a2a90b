// Structured sigma (single-block bases): see fastplan.h for the frame.
//
// Per sigma application, with c~ = eps * c:
//   1. frame_transpose : c~ (row-major, rows padded to ldA) and c~^T (rows
//                        padded to ldB)                                  [HBM streaming]
//   2. pure_rows(alpha): s~ = D * c~ + sum_pure-alpha PA(a') PB(b) c~[a', b]
//   3. pure_rows(beta) : t  = same on c~^T with the pure-beta groups
//   4. per column tile of the intermediate Z:
//        mixed_gemm   : for every source row a', X[F][b] = sB_F c~[a', b^F] is
//                       gathered once (through the precomputed index table
//                       gidx[F][b]) and Y = Lam_conn(a') X is a register-blocked
//                       GEMM; Z[a'][j][b] = sA_E(a') Y[j][b]
//        mixed_gather : s~[a, b] += sum_E Z[a^E][j(E)][b]               [coalesced]
//   5. final: sigma = eps * (s~ + t^T)
// Steps 2/3 read source rows with 16-byte vector loads; the grid runs
// column-chunk-major so the chunk of every source row stays in L2 while all
// destination rows use it.
#include "fastplan.h"
#include "ops.h"
#include "tiles.cuh"

#include <cstdlib>
#include <mutex>

namespace bsim {

constexpr int kRowChunk = 1024;        // columns per CTA in the row kernels (256 threads x 4)

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// four consecutive elements (16-byte aligned for float, 2 x 16 bytes for double)
__device__ __forceinline__ void load4(const float *p, float v[4])
{
    const float4 q = __ldg(reinterpret_cast<const float4 *>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void load4(const double *p, double v[4])
{
    const double2 q0 = __ldg(reinterpret_cast<const double2 *>(p));
    const double2 q1 = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
}

// ---- 1. frame + transpose ---------------------------------------------------------
// ct[a][b] (stride ldA) and ctT[b][a] (stride ldB); the padding columns are zero.
template <typename Ti, typename Tin, typename T>
__global__ void frame_transpose_kernel(int nA, int nB, int ldA, int ldB, const Ti *__restrict__ bstr,
                                       const u64 *__restrict__ Ka, const Tin *__restrict__ c, T *__restrict__ ct,
                                       T *__restrict__ ctT)
{
    __shared__ T tile[32][33];
    const int b0 = blockIdx.x * 32, a0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int i = ty; i < 32; i += blockDim.y) {
        const int a = a0 + i, b = b0 + tx;
        T v = T(0);
        if (a < nA && b < nB) {
            v = (T)c[(i64)a * nB + b];
            if (par((u64)bstr[b] & Ka[a])) v = -v;
        }
        if (a < nA && b < ldA) ct[(i64)a * ldA + b] = v;
        tile[i][tx] = v;
    }
    __syncthreads();
    for (int i = ty; i < 32; i += blockDim.y) {
        const int b = b0 + i, a = a0 + tx;
        if (b < nB && a < ldB) ctT[(i64)b * ldB + a] = tile[tx][i];
    }
}

// ---- 2/3. pure groups of one spin: row AXPY over the precomputed row lists -----------
// One CTA per (row, 1024-column chunk); each thread owns 4 consecutive columns.
// Constant-factor entries accumulate in T over batches of 64 entries, then in
// FP64; table entries and the diagonal are FP64 throughout.
template <typename T>
__global__ void __launch_bounds__(256)
pure_rows_kernel(int ncols, int ld_in, const SideCSR L, const T *__restrict__ in, double *__restrict__ out,
                 int ld_out, const double *__restrict__ PAd, const double *__restrict__ PBdT, int rank_d)
{
    const int row = blockIdx.x;
    const int c = blockIdx.y * kRowChunk + 4 * threadIdx.x;
    if (c >= ncols) return;
    const T *in_c = in + c;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (PAd) {
        T self[4];
        load4(in_c + (i64)row * ld_in, self);
        double d[4] = {0.0, 0.0, 0.0, 0.0};
        for (int r = 0; r < rank_d; ++r) {
            const double pa = __ldg(PAd + (i64)row * rank_d + r);
            double pb[4];
            load4(PBdT + (i64)r * ld_in + c, pb);
#pragma unroll
            for (int k = 0; k < 4; ++k) d[k] += pa * pb[k];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] = d[k] * (double)self[k];
    }
    const i64 e_beg = L.cptr[row], e_end = L.cptr[row + 1];
    const CEnt *__restrict__ ent = L.cent;
    constexpr int kBatch = 64;   // FP32 partial sums span at most this many entries
    for (i64 e0 = e_beg; e0 < e_end; e0 += kBatch) {
        const i64 e1 = min(e_end, e0 + kBatch);
        T part[4] = {T(0), T(0), T(0), T(0)};
        i64 e = e0;
        for (; e + 4 <= e1; e += 4) {   // 4 entries x 4 columns of independent loads in flight
            const CEnt E0 = ent[e], E1 = ent[e + 1], E2 = ent[e + 2], E3 = ent[e + 3];
            T v0[4], v1[4], v2[4], v3[4];
            load4(in_c + E0.off, v0);
            load4(in_c + E1.off, v1);
            load4(in_c + E2.off, v2);
            load4(in_c + E3.off, v3);
            const T k0 = (T)E0.coef, k1 = (T)E1.coef, k2 = (T)E2.coef, k3 = (T)E3.coef;
#pragma unroll
            for (int k = 0; k < 4; ++k) part[k] += k0 * v0[k] + k1 * v1[k] + k2 * v2[k] + k3 * v3[k];
        }
        for (; e < e1; ++e) {
            const CEnt E0 = ent[e];
            T v0[4];
            load4(in_c + E0.off, v0);
            const T k0 = (T)E0.coef;
#pragma unroll
            for (int k = 0; k < 4; ++k) part[k] += k0 * v0[k];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] += (double)part[k];
    }
    for (i64 e = L.tptr[row]; e < L.tptr[row + 1]; ++e) {
        const TEnt t = L.tent[e];
        const int R = (int)(t.toff_rank & 7);
        const double *tab = L.ctab + (t.toff_rank & ~7ll) + c;
        double f[4] = {0.0, 0.0, 0.0, 0.0};
        for (int r = 0; r < R; ++r) {
            double cr[4];
            load4(tab + (i64)r * ld_in, cr);
#pragma unroll
            for (int k = 0; k < 4; ++k) f[k] += t.pa[r] * cr[k];
        }
        T v[4];
        load4(in_c + t.off, v);
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] += f[k] * (double)v[k];
    }
    double *o = out + (i64)row * ld_out + c;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (c + k < ncols) o[k] = acc[k];
}

// ---- 4a. mixed GEMM -----------------------------------------------------------------
struct MixedArgs {
    int nA, nB, nE, nF, M, ldA, ldG;
    const u64 *Emask, *mA;
    const void *Lam;        // T [nE x nF]
    const int *gidx;        // [nF x ldG]: (rank(b^F) << 1 | sign) or -1
};

// Builds this row's connected alpha excitations (E order) into conn/sgn; returns the count.
template <int NT>
__device__ __forceinline__ int connected_excitations(const MixedArgs &P, u64 sa, int *conn, int *sgn, int *wcnt,
                                                     int *cnt)
{
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) *cnt = 0;
    __syncthreads();
    for (int base = 0; base < P.nE; base += NT) {
        const int e = base + threadIdx.x;
        const bool ok = e < P.nE && __popcll(sa & P.Emask[e]) == 1;
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (lane == 0) wcnt[wid] = __popc(m);
        __syncthreads();
        int off = *cnt;
        for (int w2 = 0; w2 < wid; ++w2) off += wcnt[w2];
        if (ok) {
            const int j = off + __popc(m & ((1u << lane) - 1u));
            if (j < 64) { conn[j] = e; sgn[j] = (__popcll(sa & P.mA[e]) & 1) ? -1 : 1; }
        }
        __syncthreads();
        if (threadIdx.x == 0) for (int w2 = 0; w2 < NW; ++w2) *cnt += wcnt[w2];
        __syncthreads();
    }
    return min(*cnt, 64);
}

// EPT consecutive Lam_conn values (32 bytes) from shared memory
template <int EPT>
__device__ __forceinline__ void load_lam(const double *p, double l[EPT])
{
    static_assert(EPT == 4, "FP64 GEMM uses 4 excitations per thread");
    const double2 q0 = reinterpret_cast<const double2 *>(p)[0], q1 = reinterpret_cast<const double2 *>(p)[1];
    l[0] = q0.x; l[1] = q0.y; l[2] = q1.x; l[3] = q1.y;
}
template <int EPT>
__device__ __forceinline__ void load_lam(const float *p, float l[EPT])
{
    static_assert(EPT == 8, "FP32 GEMM uses 8 excitations per thread");
    const float4 q0 = reinterpret_cast<const float4 *>(p)[0], q1 = reinterpret_cast<const float4 *>(p)[1];
    l[0] = q0.x; l[1] = q0.y; l[2] = q0.z; l[3] = q0.w;
    l[4] = q1.x; l[5] = q1.y; l[6] = q1.z; l[7] = q1.w;
}

// One CTA per source row a'.  Warp w owns excitations w*EPT .. w*EPT+EPT-1 of
// the row's connected list; lane l owns columns {2l, 2l+1, 64+2l, 64+2l+1} of a
// kMixCols-column chunk (conflict-free 2-element shared loads).  The X slice for
// (chunk, 32 F) is filled from the gather-index table, whose next slice is
// loaded into registers while the current one is multiplied.
template <typename Ti, typename T, int EPT>
__global__ void __launch_bounds__((64 / EPT) * 32, EPT == 8 ? 2 : 1)
mixed_gemm_kernel(const MixedArgs P, const Ti *__restrict__ astr, const T *__restrict__ ct, T *__restrict__ Z,
                  int z0, int W)
{
    constexpr int NT = (64 / EPT) * 32, NW = NT / 32;
    constexpr int ITEMS = 32 * kMixCols / NT;
    using V2 = typename Vec2<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = P.nF, M = P.M;
    T *srow = reinterpret_cast<T *>(smem_raw);                    // [ldA]
    T *lam = srow + P.ldA;                                         // [K][64]
    T *xs = lam + (size_t)K * 64;                                  // [32][kMixCols]
    int *conn = reinterpret_cast<int *>(xs + 32 * kMixCols);       // [64]
    int *sgn = conn + 64;                                          // [64]
    __shared__ int wcnt[NW], cnt;
    const int a = blockIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int m = connected_excitations<NT>(P, (u64)astr[a], conn, sgn, wcnt, &cnt);
    // stage the source row (16-byte copies) and Lam restricted to the connected excitations
    {
        const int4 *src = reinterpret_cast<const int4 *>(ct + (i64)a * P.ldA);
        int4 *dst = reinterpret_cast<int4 *>(srow);
        const int n16 = (int)((size_t)P.ldA * sizeof(T) / 16);
        for (int i = threadIdx.x; i < n16; i += NT) dst[i] = __ldg(src + i);
    }
    const T *Lam = static_cast<const T *>(P.Lam);
    for (int i = threadIdx.x; i < K * 64; i += NT) {
        const int f = i >> 6, j = i & 63;
        lam[i] = j < m ? (T)sgn[j] * Lam[(i64)conn[j] * K + f] : T(0);
    }
    const int zend = min(P.nB, z0 + W);
    const int ncb = (zend - z0 + kMixCols - 1) / kMixCols;
    const int nfc = (K + 31) / 32;
    const int nsteps = ncb * nfc;
    const bool active = wid * EPT < m;
    int gpre[ITEMS];
    auto load_g = [&](int step) {
        const int cb = z0 + (step / nfc) * kMixCols, f0 = (step % nfc) * 32;
#pragma unroll
        for (int it = 0; it < ITEMS; ++it) {
            const int i = threadIdx.x + it * NT;
            const int f = i / kMixCols, cl = i % kMixCols;
            gpre[it] = f0 + f < K ? __ldg(P.gidx + (i64)(f0 + f) * P.ldG + cb + cl) : -1;
        }
    };
    T acc[EPT][4];
#pragma unroll
    for (int i = 0; i < EPT; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = T(0);
    if (nsteps > 0) load_g(0);
    for (int step = 0; step < nsteps; ++step) {
        const int cbi = step / nfc, fci = step % nfc;
        const int f0 = fci * 32, nf = min(32, K - f0);
        __syncthreads();   // the previous slice is consumed (and srow/lam are staged)
#pragma unroll
        for (int it = 0; it < ITEMS; ++it) {
            const int g = gpre[it];
            T x = T(0);
            if (g >= 0) {
                x = srow[g >> 1];
                if (g & 1) x = -x;
            }
            xs[threadIdx.x + it * NT] = x;
        }
        __syncthreads();
        if (step + 1 < nsteps) load_g(step + 1);
        if (active) {
#pragma unroll 4
            for (int f = 0; f < nf; ++f) {
                T l[EPT];
                load_lam<EPT>(lam + (size_t)(f0 + f) * 64 + wid * EPT, l);
                const V2 xa = *reinterpret_cast<const V2 *>(xs + f * kMixCols + 2 * lane);
                const V2 xb = *reinterpret_cast<const V2 *>(xs + f * kMixCols + 64 + 2 * lane);
#pragma unroll
                for (int i = 0; i < EPT; ++i) {
                    acc[i][0] += l[i] * xa.x;
                    acc[i][1] += l[i] * xa.y;
                    acc[i][2] += l[i] * xb.x;
                    acc[i][3] += l[i] * xb.y;
                }
            }
        }
        if (fci == nfc - 1) {
            if (active) {
#pragma unroll
                for (int i = 0; i < EPT; ++i) {
                    const int j = wid * EPT + i;
                    if (j < m) {
                        T *zr = Z + ((i64)a * M + j) * W + cbi * kMixCols;
                        V2 v0, v1;
                        v0.x = acc[i][0]; v0.y = acc[i][1];
                        v1.x = acc[i][2]; v1.y = acc[i][3];
                        *reinterpret_cast<V2 *>(zr + 2 * lane) = v0;
                        *reinterpret_cast<V2 *>(zr + 64 + 2 * lane) = v1;
                    }
                }
            }
#pragma unroll
            for (int i = 0; i < EPT; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = T(0);
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
__global__ void final_kernel(int nA, int nB, int ldB, const Ti *__restrict__ bstr, const u64 *__restrict__ Ka,
                             const double *__restrict__ tT, double *__restrict__ sig)
{
    __shared__ double tile[32][33];
    const int b0 = blockIdx.x * 32, a0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int i = ty; i < 32; i += blockDim.y) {   // t^T tile: rows b, cols a
        const int b = b0 + i, a = a0 + tx;
        tile[i][tx] = (a < nA && b < nB) ? tT[(i64)b * ldB + a] : 0.0;
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

template <typename Ti, typename T, int EPT>
static int launch_mixed(const DevBasis<Ti> *B, FastPlan<Ti> &P, FastScratch<Ti> &S, const T *ct, double *dst,
                        cudaStream_t s)
{
    constexpr int NT = (64 / EPT) * 32;
    const int nA = P.nA, nB = P.nB;
    const size_t per_col = (size_t)nA * P.M * sizeof(T);
    size_t Wz = std::max<size_t>(kMixCols, (scratch_budget() / per_col) / kMixCols * kMixCols);
    Wz = std::min<size_t>(Wz, ((size_t)nB + kMixCols - 1) / kMixCols * kMixCols);
    int rc;
    if ((rc = ensure(&S.Z, &S.z_n, per_col * Wz)) != BSIM_OK) return rc;
    MixedArgs ma{nA, nB, P.nE, P.nF, P.M, P.ldA, P.ldG, P.d_Emask, P.d_mA,
                 sizeof(T) == 8 ? (const void *)P.d_Lam : (const void *)P.d_Lam32, P.d_gidx};
    const size_t smem = mixed_smem_bytes(nB, P.nF, sizeof(T));
    if (smem > 227 * 1024) { set_error("mixed kernel needs %zu bytes of shared memory", smem); return BSIM_ERR_UNSUPPORTED; }
    BSIM_CUDA(cudaFuncSetAttribute(mixed_gemm_kernel<Ti, T, EPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    T *Z = static_cast<T *>(S.Z);
    for (int z0 = 0; z0 < nB; z0 += (int)Wz) {
        mixed_gemm_kernel<Ti, T, EPT><<<nA, NT, smem, s>>>(ma, P.d_astr, ct, Z, z0, (int)Wz);
        dim3 g(nA, (unsigned)((std::min<size_t>(Wz, nB - z0) + kRowChunk - 1) / kRowChunk));
        mixed_gather_kernel<Ti, T><<<g, 256, 0, s>>>(ma, P.d_astr, B->view.amap, Z, dst, z0, (int)Wz);
    }
    return BSIM_OK;
}

template <typename Ti, typename T>
static int run_fast(const DevBasis<Ti> *B, const DevNet<Ti> *N, FastState<Ti> *st, const double *src,
                    const float *src32, double *dst, cudaStream_t s)
{
    FastPlan<Ti> &P = st->plan;
    FastScratch<Ti> &S = st->scratch;
    const int nA = P.nA, nB = P.nB;
    int rc;
    if ((rc = ensure(&S.ct, &S.ct_n, (size_t)nA * P.ldA * sizeof(T))) != BSIM_OK) return rc;
    if ((rc = ensure(&S.ctT, &S.ctT_n, (size_t)nB * P.ldB * sizeof(T))) != BSIM_OK) return rc;
    if ((rc = ensure(&S.tT, &S.tT_n, (size_t)nB * P.ldB * sizeof(double))) != BSIM_OK) return rc;
    T *ct = static_cast<T *>(S.ct), *ctT = static_cast<T *>(S.ctT);
    double *tT = static_cast<double *>(S.tT);
    // 1. frame + transpose (grid covers the padded strides)
    dim3 tgrid((nB + 31) / 32, (nA + 31) / 32), tblk(32, 8);
    if (src32)
        frame_transpose_kernel<Ti, float, T><<<tgrid, tblk, 0, s>>>(nA, nB, P.ldA, P.ldB, P.d_bstr, P.d_Ka, src32, ct, ctT);
    else
        frame_transpose_kernel<Ti, double, T><<<tgrid, tblk, 0, s>>>(nA, nB, P.ldA, P.ldB, P.d_bstr, P.d_Ka, src, ct, ctT);
    // 2. pure alpha + diagonal -> dst (the frame's s~)
    {
        dim3 g(nA, (nB + kRowChunk - 1) / kRowChunk);
        pure_rows_kernel<T><<<g, 256, 0, s>>>(nB, P.ldA, P.csrA, ct, dst, nB, P.rank_d ? P.d_PAd : nullptr,
                                              P.d_PBdT, P.rank_d);
    }
    // 3. pure beta on the transposed vector -> tT
    {
        dim3 g(nB, (nA + kRowChunk - 1) / kRowChunk);
        pure_rows_kernel<T><<<g, 256, 0, s>>>(nA, P.ldB, P.csrB, ctT, tT, P.ldB, nullptr, nullptr, 0);
    }
    // 4. mixed
    if (P.nE > 0 && P.nF > 0 && P.M > 0) {
        if constexpr (sizeof(T) == 8) rc = launch_mixed<Ti, T, 4>(B, P, S, ct, dst, s);
        else rc = launch_mixed<Ti, T, 8>(B, P, S, ct, dst, s);
        if (rc != BSIM_OK) return rc;
    }
    // 5. final combine
    final_kernel<Ti><<<tgrid, tblk, 0, s>>>(nA, nB, P.ldB, P.d_bstr, P.d_Ka, tT, dst);
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
