// Structured sigma (single-block bases): see fastplan.h for the frame.
//
// Per sigma application, with c~ = eps * c:
//   1. frame       : c~ (row-major, rows padded to ldA)               [HBM streaming]
//   2. pure_rows(alpha): s~ = D * c~ + sum_pure-alpha PA(a') PB(b) c~[a', b]
//   3. per column tile of the intermediate Z:
//        mixed_gemm   : for every source row a', X[F][b] = sB_F c~[a', b^F] is
//                       gathered once (through the precomputed index table
//                       gidx[F][b]) and Y = Lam_conn(a') X is a register-blocked
//                       GEMM; Z[a'][j][b] = sA_E(a') Y[j][b]
//        mixed_gather : s~[a, b] += sum_E Z[a^E][j(E)][b]               [coalesced]
//   4. transpose   : c~^T (rows padded to ldB) into the buffer c~ held
//   5. pure_rows(beta) : t  = same as 2 on c~^T with the pure-beta groups
//   6. final: sigma = eps * (s~ + t^T)
// The alpha side runs first so that c~ and c~^T share one buffer and t's buffer
// holds the alpha side's intermediate Z: the scratch of one sigma is one input
// copy in the bulk precision plus one FP64 vector (and a bounded Z).
// Steps 2/3 read source rows with 16-byte vector loads; the grid runs
// column-chunk-major so the chunk of every source row stays in L2 while all
// destination rows use it.
#include "fastplan.h"
#include "mixed.cuh"
#include "ops.h"
#include "tiles.cuh"

#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>

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
        if (ct && a < nA && b < ldA) ct[(i64)a * ldA + b] = v;
        tile[i][tx] = v;
    }
    if (!ctT) return;   // uniform across the CTA
    __syncthreads();
    for (int i = ty; i < 32; i += blockDim.y) {
        const int b = b0 + i, a = a0 + tx;
        if (b < nB && a < ldB) ctT[(i64)b * ldB + a] = tile[tx][i];
    }
}

// ---- 2/3. pure groups of one spin: row AXPY over the precomputed row lists -----------
// One CTA per (row, 1024-column chunk) of rows row_begin.. and columns
// [col_begin, ncols); each thread owns 4 consecutive columns.
// Constant-factor entries accumulate in T over batches of 64 entries, then in
// FP64; table entries and the diagonal are FP64 throughout.
template <typename T>
__global__ void __launch_bounds__(256)
pure_rows_kernel(int row_begin, int col_begin, int ncols, int ld_in, const SideCSR L, const T *__restrict__ in,
                 double *__restrict__ out, int ld_out, const double *__restrict__ PAd, const double *__restrict__ PBdT,
                 int rank_d)
{
    const int row = row_begin + blockIdx.x;
    const int c = col_begin + blockIdx.y * kRowChunk + 4 * threadIdx.x;
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
    // column-factor tables in the bulk precision (FP64 sums of the factor)
    const T *ctab = std::is_same<T, float>::value ? reinterpret_cast<const T *>(L.ctab32)
                                                  : reinterpret_cast<const T *>(L.ctab);
    for (i64 e = L.tptr[row]; e < L.tptr[row + 1]; ++e) {
        const TEnt t = L.tent[e];
        const int R = (int)(t.toff_rank & 7);
        const T *tab = ctab + (t.toff_rank & ~7ll) + c;
        double f[4] = {0.0, 0.0, 0.0, 0.0};
        T v[4];
        if constexpr (std::is_same<T, float>::value) {
            // FP32: the rank loop unrolled to its bound, every table row of the
            // entry and the source row loaded before the first use (measured per
            // sigma: 0.143 -> 0.126 ms at 12o, 26.5 -> 26.3 ms at 16o; the FP64
            // kernel, bound by L1 throughput, went 38.9 -> 43.9 ms at 16o with it)
            T cr[kSideMaxRank][4];
#pragma unroll
            for (int r = 0; r < kSideMaxRank; ++r)
                if (r < R) load4(tab + (i64)r * ld_in, cr[r]);
            load4(in_c + t.off, v);
#pragma unroll
            for (int r = 0; r < kSideMaxRank; ++r)
                if (r < R) {
#pragma unroll
                    for (int k = 0; k < 4; ++k) f[k] += t.pa[r] * (double)cr[r][k];
                }
        } else {
            for (int r = 0; r < R; ++r) {
                T cr[4];
                load4(tab + (i64)r * ld_in, cr);
#pragma unroll
                for (int k = 0; k < 4; ++k) f[k] += t.pa[r] * (double)cr[k];
            }
            load4(in_c + t.off, v);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] += f[k] * (double)v[k];
    }
    double *o = out + (i64)row * ld_out + c;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (c + k < ncols) o[k] = acc[k];
}

// ---- 4a. mixed GEMM -----------------------------------------------------------------
// (MixedArgs and connected_excitations: mixed.cuh)

// EPT consecutive Lam_conn values (32 bytes) from shared memory
template <int EPT>
__device__ __forceinline__ void load_lam(const double *p, double l[EPT])
{
    static_assert(EPT % 2 == 0, "pairs of excitations per 16-byte load");
#pragma unroll
    for (int i = 0; i < EPT / 2; ++i) {
        const double2 q = reinterpret_cast<const double2 *>(p)[i];
        l[2 * i] = q.x;
        l[2 * i + 1] = q.y;
    }
}
template <int EPT>
__device__ __forceinline__ void load_lam(const float *p, float l[EPT])
{
    static_assert(EPT == 8 || EPT == 10, "FP32 GEMM uses 8 (64-row tile) or 10 (80-row tile) excitations per thread");
    if constexpr (EPT == 8) {   // 32-byte aligned: two 16-byte loads
        const float4 q0 = reinterpret_cast<const float4 *>(p)[0], q1 = reinterpret_cast<const float4 *>(p)[1];
        l[0] = q0.x; l[1] = q0.y; l[2] = q0.z; l[3] = q0.w;
        l[4] = q1.x; l[5] = q1.y; l[6] = q1.z; l[7] = q1.w;
    } else {                    // 40-byte runs, 8-byte aligned
#pragma unroll
        for (int i = 0; i < EPT / 2; ++i) {
            const float2 q = reinterpret_cast<const float2 *>(p)[i];
            l[2 * i] = q.x;
            l[2 * i + 1] = q.y;
        }
    }
}

// Register tile of the two GEMMs: EPT output rows x the lane's 4 columns
// {2l, 2l+1, 64+2l, 64+2l+1}.  The FP32 tile keeps its accumulators as f32x2
// pairs and issues Blackwell's packed fma.rn.f32x2 (two IEEE single-precision
// FMAs per instruction, each rounded as a scalar fmaf), halving the FMA issue
// slots of the FP32-bulk GEMMs.
template <typename T, int EPT>
struct GemmTile {
    T v[EPT][4];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int i = 0; i < EPT; ++i) v[i][0] = v[i][1] = v[i][2] = v[i][3] = T(0);
    }
    __device__ __forceinline__ void step(const T *l, const T *xa, const T *xb)
    {
        const typename Vec2<T>::type a = *reinterpret_cast<const typename Vec2<T>::type *>(xa);
        const typename Vec2<T>::type b = *reinterpret_cast<const typename Vec2<T>::type *>(xb);
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            v[i][0] += l[i] * a.x;
            v[i][1] += l[i] * a.y;
            v[i][2] += l[i] * b.x;
            v[i][3] += l[i] * b.y;
        }
    }
    __device__ __forceinline__ void pair(int i, typename Vec2<T>::type &p0, typename Vec2<T>::type &p1) const
    {
        p0.x = v[i][0]; p0.y = v[i][1];
        p1.x = v[i][2]; p1.y = v[i][3];
    }
};

template <int EPT>
struct GemmTile<float, EPT> {
    unsigned long long p[EPT][2];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int i = 0; i < EPT; ++i) p[i][0] = p[i][1] = 0ull;   // +0.0f in both halves
    }
    __device__ __forceinline__ void step(const float *l, const float *xa, const float *xb)
    {
        const unsigned long long a = *reinterpret_cast<const unsigned long long *>(xa);
        const unsigned long long b = *reinterpret_cast<const unsigned long long *>(xb);
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            unsigned long long ll;
            asm("mov.b64 %0, {%1, %1};" : "=l"(ll) : "f"(l[i]));
            asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(p[i][0]) : "l"(ll), "l"(a));
            asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(p[i][1]) : "l"(ll), "l"(b));
        }
    }
    __device__ __forceinline__ void pair(int i, float2 &p0, float2 &p1) const
    {
        asm("mov.b64 {%0, %1}, %2;" : "=f"(p0.x), "=f"(p0.y) : "l"(p[i][0]));
        asm("mov.b64 {%0, %1}, %2;" : "=f"(p1.x), "=f"(p1.y) : "l"(p[i][1]));
    }
};

// Shared-memory strides of the GEMM operands: Lam/W_m rows of LS elements and
// X-slice rows of XS elements.  The FP64 tiles are read as mma fragments (lane
// (g, t) = (lane / 4, lane % 4) reads row t, column g (and g + 8) of a block); a
// row stride of 4 mod 16 doubles puts the 16 lanes of each half-warp on
// distinct banks.
template <typename T> struct GemmLayout { static constexpr int LS = 64, XS = kMixCols; };
template <> struct GemmLayout<double> { static constexpr int LS = 68, XS = kMixCols + 4; };

// FP64 on the tensor cores' DMMA path: 16x8 tile += 16x4 A (rows g, g + 8 of column t in lane (g, t)) x 4x8 B
// (row t, column g); the accumulator holds rows g and g + 8, columns 2t, 2t + 1.
__device__ __forceinline__ void dmma_16x8x4(double (&c)[4], double2 a, double b)
{
    asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, {%6}, "
                 "{%0, %1, %2, %3};"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a.x), "d"(a.y), "d"(b));
}

// The same with K = 8: A rows g, g + 8 of columns t (a01) and t + 4 (a23), B rows
// t (b.x) and t + 4 (b.y) of column g.
__device__ __forceinline__ void dmma_16x8x8(double (&c)[4], double2 a01, double2 a23, double2 b)
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
                 "{%0, %1, %2, %3};"
                 : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
                 : "d"(a01.x), "d"(a01.y), "d"(a23.x), "d"(a23.y), "d"(b.x), "d"(b.y));
}

template <typename T, int EPT>
struct GemmCore {
    // FP32 bulk: EPT rows x 4 columns per thread with packed f32x2 FMAs
    GemmTile<T, EPT> acc;
    __device__ __forceinline__ void zero() { acc.zero(); }
    __device__ __forceinline__ static bool active(int rows) { return (int)(threadIdx.x >> 5) * EPT < rows; }
    template <int LS = GemmLayout<T>::LS>
    __device__ __forceinline__ void step(const T *lam, const T *xs, int f0, int nf)
    {
        constexpr int XS = GemmLayout<T>::XS;
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll 4
        for (int f = 0; f < nf; ++f) {
            T l[EPT];
            load_lam<EPT>(lam + (size_t)(f0 + f) * LS + wid * EPT, l);
            acc.step(l, xs + f * XS + 2 * lane, xs + f * XS + 64 + 2 * lane);
        }
    }
    __device__ __forceinline__ void store(T *zbase, int W, int rows) const
    {
        using V2 = typename Vec2<T>::type;
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int j = wid * EPT + i;
            if (j < rows) {
                V2 v0, v1;
                acc.pair(i, v0, v1);
                *reinterpret_cast<V2 *>(zbase + (i64)j * W + 2 * lane) = v0;
                *reinterpret_cast<V2 *>(zbase + (i64)j * W + 64 + 2 * lane) = v1;
            }
        }
    }
};

template <int EPT>
struct GemmCore<double, EPT> {
    // warp w computes rows 16 (w / 4) .. + 15 and columns 32 (w % 4) .. + 31 of the
    // 64 x kMixCols output chunk as four 16x8 tiles of mma.sync m16n8k8
    static_assert(EPT == 4, "16 warps: 4 row groups x 4 column quarters");
    double c[4][4];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int k = 0; k < 4; ++k) c[k][0] = c[k][1] = c[k][2] = c[k][3] = 0.0;
    }
    __device__ __forceinline__ static bool active(int rows) { return (int)(threadIdx.x >> 7) * 16 < rows; }
    template <int LS = GemmLayout<double>::LS>
    __device__ __forceinline__ void step(const double *lam, const double *xs, int f0, int nf)
    {
        constexpr int XS = GemmLayout<double>::XS;
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const int g = lane >> 2, t = lane & 3, rg = wid >> 2, cq = wid & 3;
        const double *la = lam + (size_t)(f0 + t) * LS + rg * 16 + g;
        const double *xb = xs + t * XS + cq * 32 + g;
        for (int kk = 0; kk < nf; kk += 8) {   // slice rows past nf are zero in X and in Lam
            const double2 a01 = make_double2(la[(size_t)kk * LS], la[(size_t)kk * LS + 8]);
            const double2 a23 = make_double2(la[(size_t)(kk + 4) * LS], la[(size_t)(kk + 4) * LS + 8]);
            double2 b[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) b[k] = make_double2(xb[kk * XS + 8 * k], xb[(kk + 4) * XS + 8 * k]);
#pragma unroll
            for (int k = 0; k < 4; ++k) dmma_16x8x8(c[k], a01, a23, b[k]);
        }
    }
    __device__ __forceinline__ void store(double *zbase, int W, int rows) const
    {
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        const int g = lane >> 2, t = lane & 3, rg = wid >> 2, cq = wid & 3;
        const int j = rg * 16 + g;
        double *zr = zbase + (i64)j * W + cq * 32 + 2 * t;
        if (j < rows) {
#pragma unroll
            for (int k = 0; k < 4; ++k) *reinterpret_cast<double2 *>(zr + 8 * k) = make_double2(c[k][0], c[k][1]);
        }
        if (j + 8 < rows) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                *reinterpret_cast<double2 *>(zr + (i64)8 * W + 8 * k) = make_double2(c[k][2], c[k][3]);
        }
    }
};

// One CTA per source row a'.  Warp w owns excitations w*EPT .. w*EPT+EPT-1 of
// the row's connected list; lane l owns columns {2l, 2l+1, 64+2l, 64+2l+1} of a
// kMixCols-column chunk (conflict-free 2-element shared loads).  The X slice for
// (chunk, 32 F) is filled from the gather-index table, whose next slice is
// loaded into registers while the current one is multiplied.  With GROW the
// source row stays in global memory (L2) and the next slice's values, not only
// their indices, are prefetched.  A pass covers ROWS connected excitations: 64
// (FP64: 16 warps of 8x8 DMMA tiles; FP32: 8 warps x 8 rows), or 80 for FP32
// with 10 rows per warp (18 orbitals, 8 electrons: 80 connected singles in one
// pass instead of a 64-row and a 16-row pass).
template <typename Ti, typename T, int EPT, bool STREAM, bool GROW>
__global__ void __launch_bounds__(sizeof(T) == 8 ? 512 : 256, (sizeof(T) == 4 && EPT == 8) ? 2 : 1)
mixed_gemm_kernel(const MixedArgs P, const Ti *__restrict__ astr, const T *__restrict__ ct, T *__restrict__ Z,
                  int z0, int W, int jbase)
{
    constexpr int NT = sizeof(T) == 8 ? 512 : 256, NW = NT / 32;
    constexpr int ROWS = sizeof(T) == 8 ? 64 : NW * EPT;
    constexpr int ITEMS = 32 * kMixCols / NT;
    constexpr int LITEMS = STREAM ? 32 * ROWS / NT : 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = P.nF, M = P.M;
    T *srow = reinterpret_cast<T *>(smem_raw);                    // [ldA] unless GROW
    constexpr int LS = ROWS > 64 ? ROWS : GemmLayout<T>::LS, XS = GemmLayout<T>::XS;
    const int Kp = (K + 7) & ~7;   // whole K steps of 8 (FP64 m16n8k8), rows past K zero
    T *lam = srow + (GROW ? 0 : P.ldA);                            // [Kp or 32][LS], rows past K zero
    T *xs = lam + (size_t)(STREAM ? 32 : Kp) * LS;                 // [32][XS]
    int *conn = reinterpret_cast<int *>(xs + 32 * XS);             // [kMaxConn]
    int *sgn = conn + kMaxConn;                                    // [kMaxConn]
    __shared__ int wcnt[NW], cnt;
    const int a = blockIdx.x;
    const int m = connected_excitations<NT>(P, (u64)astr[a], conn, sgn, wcnt, &cnt);
    const int jm = min(ROWS, m - jbase);   // output rows of this pass
    if (jm <= 0) return;                   // uniform across the CTA
    const T *grow = ct + (i64)a * P.ldA;
    // stage the source row (16-byte copies) and, when it fits, Lam restricted to
    // this pass's connected excitations
    if (!GROW) {
        const int4 *src = reinterpret_cast<const int4 *>(grow);
        int4 *dst = reinterpret_cast<int4 *>(srow);
        const int n16 = (int)((size_t)P.ldA * sizeof(T) / 16);
        for (int i = threadIdx.x; i < n16; i += NT) dst[i] = __ldg(src + i);
    }
    const T *Lam = static_cast<const T *>(P.Lam);
    if (!STREAM)
        for (int i = threadIdx.x; i < Kp * LS; i += NT) {
            const int f = i / LS, j = i % LS;
            lam[i] = (j < jm && f < K) ? (T)sgn[jbase + j] * Lam[(i64)conn[jbase + j] * K + f] : T(0);
        }
    const int zend = min(P.cend, z0 + W);
    const int ncb = (zend - z0 + kMixCols - 1) / kMixCols;
    const int nfc = (K + 31) / 32;
    const int nsteps = ncb * nfc;
    const bool active = GemmCore<T, EPT>::active(jm);
    int gpre[GROW ? 1 : ITEMS];
    T gval[GROW ? ITEMS : 1];
    T lpre[LITEMS];
    auto load_g = [&](int step) {
        const int cb = z0 + (step / nfc) * kMixCols, f0 = (step % nfc) * 32;
#pragma unroll
        for (int it = 0; it < ITEMS; ++it) {
            const int i = threadIdx.x + it * NT;
            const int f = i / kMixCols, cl = i % kMixCols;
            const int g = f0 + f < K ? __ldg(P.gidx + (i64)(f0 + f) * P.ldG + cb + cl) : -1;
            if constexpr (GROW) {
                T x = T(0);
                if (g >= 0) {
                    x = __ldg(grow + (g >> 1));
                    if (g & 1) x = -x;
                }
                gval[it] = x;
            } else {
                gpre[it] = g;
            }
        }
        if (STREAM) {
#pragma unroll
            for (int it = 0; it < LITEMS; ++it) {
                const int i = threadIdx.x + it * NT;
                const int f = i / ROWS, j = i % ROWS;
                lpre[it] = (j < jm && f0 + f < K) ? (T)sgn[jbase + j] * __ldg(Lam + (i64)conn[jbase + j] * K + f0 + f)
                                                  : T(0);
            }
        }
    };
    GemmCore<T, EPT> acc;
    acc.zero();
    if (nsteps > 0) load_g(0);
    for (int step = 0; step < nsteps; ++step) {
        const int cbi = step / nfc, fci = step % nfc;
        const int f0 = fci * 32, nf = min(32, K - f0);
        __syncthreads();   // the previous slice is consumed (and srow/lam are staged)
#pragma unroll
        for (int it = 0; it < ITEMS; ++it) {
            T x;
            if constexpr (GROW) {
                x = gval[it];
            } else {
                const int g = gpre[it];
                x = T(0);
                if (g >= 0) {
                    x = srow[g >> 1];
                    if (g & 1) x = -x;
                }
            }
            const int i = threadIdx.x + it * NT;
            xs[(i / kMixCols) * XS + i % kMixCols] = x;
        }
        if (STREAM) {
#pragma unroll
            for (int it = 0; it < LITEMS; ++it) {
                const int i = threadIdx.x + it * NT;
                lam[(i / ROWS) * LS + i % ROWS] = lpre[it];
            }
        }
        __syncthreads();
        if (step + 1 < nsteps) load_g(step + 1);
        if (active) acc.template step<LS>(lam, xs, STREAM ? 0 : f0, nf);
        if (fci == nfc - 1) {
            if (active) acc.store(zchunk(Z, a, M, W, cbi) + jbase * kMixCols, kMixCols, jm);
            acc.zero();
        }
    }
}

// FP64 mixed GEMM with per-warp B fragments.  Warp w owns columns 8w..8w+7 of
// each 128-column chunk and all 64 output rows: four 16x8 tiles of
// mma.sync m16n8k8 (FP64 on the tensor cores' DMMA path), those past the pass's
// connected rows skipped; lane (g, t) gathers its own B fragment elements
// X[f0 + 4i + t][8w + g] from the source row (shared memory, or L2 with GROW),
// a 32-row F slice ahead.  No X slice is shared, so the warps never
// synchronise inside the loop.  Lam_conn (the A fragments, read by every warp)
// is staged once per CTA with rows g and g + 8 of each 16-row tile side by
// side, so a lane's two A elements of a K step are one 16-byte load.
constexpr int kDmmaLS = 34;   // double2 per F row: 32 + 2 (2 mod 8: conflict-free 16-byte fragment loads)
inline size_t mixed_dmma_smem(int ldA, int nF, bool grow)
{
    return (grow ? 0 : (size_t)ldA * 8) + (size_t)((nF + 31) & ~31) * kDmmaLS * 16 + 2 * kMaxConn * 4;
}

template <typename Ti, bool GROW>
__global__ void __launch_bounds__(512, 1)
mixed_dmma_kernel(const MixedArgs P, const Ti *__restrict__ astr, const double *__restrict__ ct,
                  double *__restrict__ Z, int z0, int W, int jbase)
{
    constexpr int NT = 512;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = P.nF, M = P.M;
    const int Kp = (K + 31) & ~31;
    double *srow = reinterpret_cast<double *>(smem_raw);            // [ldA] unless GROW
    double2 *lam = reinterpret_cast<double2 *>(srow + (GROW ? 0 : P.ldA));   // [Kp][kDmmaLS], rows past K zero
    int *conn = reinterpret_cast<int *>(lam + (size_t)Kp * kDmmaLS);        // [kMaxConn]
    int *sgn = conn + kMaxConn;                                              // [kMaxConn]
    __shared__ int wcnt[NT / 32], cnt;
    const int a = blockIdx.x;
    const int m = connected_excitations<NT>(P, (u64)astr[a], conn, sgn, wcnt, &cnt);
    const int jm = min(64, m - jbase);   // output rows of this pass
    if (jm <= 0) return;                 // uniform across the CTA
    const double *grow = ct + (i64)a * P.ldA;
    if (!GROW) {
        const int4 *src = reinterpret_cast<const int4 *>(grow);
        int4 *dst = reinterpret_cast<int4 *>(srow);
        const int n16 = P.ldA / 2;
        for (int i = threadIdx.x; i < n16; i += NT) dst[i] = __ldg(src + i);
    }
    // lam[f][8 rb + g] = (Lam_conn[16 rb + g][f], Lam_conn[16 rb + g + 8][f])
    const double *Lam = static_cast<const double *>(P.Lam);
    for (int i = threadIdx.x; i < Kp * kDmmaLS; i += NT) {
        const int f = i / kDmmaLS, q = i % kDmmaLS;
        const int j0 = (q >> 3) * 16 + (q & 7), j1 = j0 + 8;
        double2 v = make_double2(0.0, 0.0);
        if (q < 32 && f < K) {
            if (j0 < jm) v.x = (double)sgn[jbase + j0] * Lam[(i64)conn[jbase + j0] * K + f];
            if (j1 < jm) v.y = (double)sgn[jbase + j1] * Lam[(i64)conn[jbase + j1] * K + f];
        }
        lam[i] = v;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const int nrb = (jm + 15) >> 4;   // 16-row tiles holding connected rows
    const int zend = min(P.cend, z0 + W);
    const int ncb = (zend - z0 + kMixCols - 1) / kMixCols;
    const int nfc = (K + 31) / 32;
    const int nsteps = ncb * nfc;
    const int col = 8 * wid + g;     // this lane's B column within a chunk
    int gp[8];
    double gv[GROW ? 8 : 1];
    auto load = [&](int step) {
        const int cb = z0 + (step / nfc) * kMixCols, f0 = (step % nfc) * 32;
        const int *gb = P.gidx + (i64)(f0 + t) * P.ldG + cb + col;
#pragma unroll
        for (int i = 0; i < 8; ++i) gp[i] = f0 + 4 * i + t < K ? __ldg(gb + (i64)(4 * i) * P.ldG) : -1;
        if constexpr (GROW) {
#pragma unroll
            for (int i = 0; i < 8; ++i) gv[i] = gp[i] >= 0 ? __ldg(grow + (gp[i] >> 1)) : 0.0;
        }
    };
    double c[4][4];
#pragma unroll
    for (int rb = 0; rb < 4; ++rb) c[rb][0] = c[rb][1] = c[rb][2] = c[rb][3] = 0.0;
    if (nsteps > 0) load(0);
    for (int step = 0; step < nsteps; ++step) {
        const int cbi = step / nfc, fci = step % nfc;
        const int f0 = fci * 32, nk = (min(32, K - f0) + 3) >> 2;
        double x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int gg = gp[i];
            double v;
            if constexpr (GROW) v = gv[i];
            else v = gg >= 0 ? srow[gg >> 1] : 0.0;
            x[i] = (gg >= 0 && (gg & 1)) ? -v : v;
        }
        if (step + 1 < nsteps) load(step + 1);
        const double2 *la = lam + (size_t)(f0 + t) * kDmmaLS + g;
#pragma unroll
        for (int i = 0; i < 4; ++i) {   // K steps of 8: F rows f0 + 8i + t and f0 + 8i + 4 + t
            if (2 * i < nk) {
#pragma unroll
                for (int rb = 0; rb < 4; ++rb)
                    if (rb < nrb)
                        dmma_16x8x8(c[rb], la[(size_t)(8 * i) * kDmmaLS + rb * 8],
                                    la[(size_t)(8 * i + 4) * kDmmaLS + rb * 8], make_double2(x[2 * i], x[2 * i + 1]));
            }
        }
        if (fci == nfc - 1) {
            double *zr = zchunk(Z, a, M, W, cbi) + (jbase + g) * kMixCols + 8 * wid + 2 * t;
#pragma unroll
            for (int rb = 0; rb < 4; ++rb) {
                if (rb < nrb && rb * 16 + g < jm)
                    *reinterpret_cast<double2 *>(zr + rb * 16 * kMixCols) = make_double2(c[rb][0], c[rb][1]);
                if (rb < nrb && rb * 16 + g + 8 < jm)
                    *reinterpret_cast<double2 *>(zr + (rb * 16 + 8) * kMixCols) = make_double2(c[rb][2], c[rb][3]);
                c[rb][0] = c[rb][1] = c[rb][2] = c[rb][3] = 0.0;
            }
        }
    }
}

// ---- 4b. gather of the mixed contributions ------------------------------------------------
template <typename Ti, typename T>
__global__ void __launch_bounds__(256)
mixed_gather_kernel(const MixedArgs P, const BasisView<Ti> BV, const T *__restrict__ Z, double *__restrict__ sig,
                    int z0, int W)
{
    __shared__ int esrc[kMaxConn], ej[kMaxConn];
    __shared__ int wcnt[8], cnt;
    const int a = blockIdx.x;
    const u64 s0 = (u64)BV.astrs[a];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    for (int base = 0; base < P.nE; base += blockDim.x) {
        const int e = base + threadIdx.x;
        bool ok = false;
        int src = -1, j = 0;
        if (e < P.nE && __popcll(s0 & P.Emask[e]) == 1) {
            const u64 s = s0 ^ P.Emask[e];
            src = string_index(BV, BV.amap, BV.nel_a, (Ti)s);
            for (int e2 = 0; e2 < e; ++e2) j += __popcll(s & P.Emask[e2]) == 1;
            ok = src >= 0 && j < kMaxConn;
        }
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        if (lane == 0) wcnt[wid] = __popc(m);
        __syncthreads();
        int off = cnt;
        for (int w2 = 0; w2 < wid; ++w2) off += wcnt[w2];
        if (ok) {
            const int p = off + __popc(m & ((1u << lane) - 1u));
            if (p < kMaxConn) { esrc[p] = src; ej[p] = j; }
        }
        __syncthreads();
        if (threadIdx.x == 0) for (int w2 = 0; w2 < 8; ++w2) cnt += wcnt[w2];
        __syncthreads();
    }
    const int n = min(cnt, kMaxConn);
    const int zend = min(P.cend, z0 + W);
    for (int b = z0 + blockIdx.y * kRowChunk + threadIdx.x; b < min(zend, z0 + (blockIdx.y + 1) * kRowChunk);
         b += blockDim.x) {
        T part = T(0);
        const T *zc = Z + (i64)((b - z0) / kMixCols) * P.M * kMixCols + (b - z0) % kMixCols;
        for (int e = 0; e < n; ++e) part += __ldg(zc + (i64)esrc[e] * P.M * W + ej[e] * kMixCols);
        sig[(i64)a * P.nB + b] += (double)part;
    }
}

// ---- 2b/3b. same-spin doubles through intermediate strings ----------------------------

// 16-byte asynchronous copy global -> shared (cp.async, L2 only); src_bytes 0
// writes zeros without reading.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes)
{
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

constexpr int kRiStages = kRiStagesHost;   // X slices in flight in the intermediate-string GEMM

// One CTA per intermediate m: X[k][col] = c~[m + pair_k][col] for the nU pairs
// outside m, Z[m][j][col] = sum_k W[pair_j][pair_k] s(m, pair_k) X[k][col] (the
// sign of each source row is folded into W_m's column, so X rows are copied
// verbatim).  The X slices (32 rows x kMixCols columns) stream through a
// kRiStages-deep cp.async ring in shared memory.  Same tiling as the mixed
// GEMM: warp w owns output rows w*EPT.., lane l owns columns
// {2l, 2l+1, 64+2l, 64+2l+1} of a kMixCols chunk.  Rows 64 .. nU-1 (at most
// kRiMaxU - 64; 66 pairs at 18 orbitals and 8 electrons) are computed by every
// thread with scalar FMAs, one (row, column) output per thread and pass.
template <typename T, int EPT>
__global__ void __launch_bounds__((64 / EPT) * 32, sizeof(T) == 4 ? 2 : 1)
ri_gemm_kernel(const RIArgs P, const T *__restrict__ in, T *__restrict__ Z, int z0, int W)
{
    constexpr int NT = (64 / EPT) * 32;
    constexpr int TQ = ((kRiMaxU - 64) * kMixCols + NT - 1) / NT;   // tail outputs per thread
    constexpr int CH = 16 / (int)sizeof(T);                          // elements per 16-byte copy
    constexpr int CPR = kMixCols / CH;                               // copies per slice row
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = P.nU;
    constexpr int LS = GemmLayout<T>::LS + 8, XS = GemmLayout<T>::XS;
    const int Kp = (K + 7) & ~7;   // whole K steps of 8 (FP64 m16n8k8), rows past K zero
    T *wm = reinterpret_cast<T *>(smem_raw);                          // [Kp][LS], rows >= K zero
    T *xs = wm + (size_t)Kp * LS;                                      // [kRiStages][32][XS]
    long long *soff = reinterpret_cast<long long *>(xs + kRiStages * 32 * XS);   // [kRiMaxU]
    const int m = blockIdx.x;
    const int *srcm = P.src + (i64)m * K, *pidm = P.pid + (i64)m * K;
    for (int i = threadIdx.x; i < kRiMaxU; i += NT) {
        long long o = 0;
        if (i < K) {
            const int v = srcm[i];
            o = ((long long)(v >> 1) * P.ld_in) * 2 + (v & 1);   // row offset, sign in the low bit
        }
        soff[i] = o;
    }
    const T *Wt = static_cast<const T *>(P.W);
    for (int i = threadIdx.x; i < Kp * LS; i += NT) {
        const int k = i / LS, j = i % LS;
        T w = T(0);
        if (j < K && k < K) {
            w = Wt[(i64)pidm[j] * P.nP + pidm[k]];
            if (srcm[k] & 1) w = -w;
        }
        wm[i] = w;
    }
    __syncthreads();
    const int zend = min(P.cend, z0 + W);
    const int ncb = (zend - z0 + kMixCols - 1) / kMixCols;
    const int nfc = (K + 31) / 32;
    const int nsteps = ncb * nfc;
    const bool active = GemmCore<T, EPT>::active(K);
    const int ntail = K > 64 ? (K - 64) * kMixCols : 0;
    // copies of slice `step` into ring slot step % kRiStages (rows past K and
    // columns past the padded row length are zero-filled); one commit group per
    // call, empty past the last step, so the wait counts stay uniform
    auto issue = [&](int step) {
        if (step < nsteps) {
            const int cb = z0 + (step / nfc) * kMixCols, f0 = (step % nfc) * 32;
            T *dst = xs + (step % kRiStages) * 32 * XS;
            for (int i = threadIdx.x; i < 32 * CPR; i += NT) {
                const int k = i / CPR, c = (i % CPR) * CH;
                const int row = f0 + k, col = cb + c;
                const bool ok = row < K && col < P.ld_in;
                cp_async16(dst + k * XS + c, ok ? (const void *)(in + (soff[row] >> 1) + col) : (const void *)in,
                           ok ? 16 : 0);
            }
        }
        cp_async_commit();
    };
    GemmCore<T, EPT> acc;
    acc.zero();
    T tacc[TQ];
#pragma unroll
    for (int q = 0; q < TQ; ++q) tacc[q] = T(0);
#pragma unroll
    for (int st = 0; st < kRiStages - 1; ++st) issue(st);
    for (int step = 0; step < nsteps; ++step) {
        const int cbi = step / nfc, fci = step % nfc;
        const int f0 = fci * 32, nf = min(32, K - f0);
        cp_async_wait<kRiStages - 2>();   // this thread's copies of slice `step` landed
        __syncthreads();                  // everyone's did; the slot refilled below is consumed
        issue(step + kRiStages - 1);
        const T *xcur = xs + (step % kRiStages) * 32 * XS;
        if (active) acc.template step<LS>(wm, xcur, f0, nf);
#pragma unroll
        for (int q = 0; q < TQ; ++q) {
            const int o = threadIdx.x + q * NT;
            if (o < ntail) {
                const int row = 64 + o / kMixCols, col = o % kMixCols;
                T t = tacc[q];
                for (int f = 0; f < nf; ++f) t += wm[(f0 + f) * LS + row] * xcur[f * XS + col];
                tacc[q] = t;
            }
        }
        if (fci == nfc - 1) {
            if (active) acc.store(zchunk(Z, m, K, W, cbi), kMixCols, K);
            acc.zero();
#pragma unroll
            for (int q = 0; q < TQ; ++q) {
                const int o = threadIdx.x + q * NT;
                if (o < ntail) zchunk(Z, m, K, W, cbi)[(64 + o / kMixCols) * kMixCols + o % kMixCols] = tacc[q];
                tacc[q] = T(0);
            }
        }
    }
    cp_async_wait<0>();
}

// FP64 intermediate-string GEMM with per-warp B fragments (as mixed_dmma_kernel):
// warp w owns columns 8w..8w+7 of each 128-column chunk and all K output rows
// (ceil(K / 16) <= 5 m16n8k8 row tiles); lane (g, t) loads its B fragment elements
// X[f0 + 4i + t][8w + g] = c~[row][col] straight from global memory (L2), a
// 32-row K slice ahead, so the main loop has no block barrier; W_m (the A
// fragments, k-major rows of kRiLS elements, zero past K) is staged once.
constexpr int kRiLS = 84;   // 4 mod 16 doubles: conflict-free A fragment loads
inline size_t ri_dmma_smem(int nU) { return (size_t)((nU + 31) & ~31) * kRiLS * 8 + kRiMaxU * 8; }

__global__ void __launch_bounds__(512, 1)
ri_dmma_kernel(const RIArgs P, const double *__restrict__ in, double *__restrict__ Z, int z0, int W)
{
    constexpr int NT = 512, MAXRB = (kRiMaxU + 15) / 16;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int K = P.nU, Kp = (K + 31) & ~31;
    double *wm = reinterpret_cast<double *>(smem_raw);                       // [Kp][kRiLS]
    long long *soff = reinterpret_cast<long long *>(wm + (size_t)Kp * kRiLS);  // [kRiMaxU]
    const int m = blockIdx.x;
    const int *srcm = P.src + (i64)m * K, *pidm = P.pid + (i64)m * K;
    for (int i = threadIdx.x; i < K; i += NT) soff[i] = (long long)(__ldg(srcm + i) >> 1) * P.ld_in;
    const double *Wt = static_cast<const double *>(P.W);
    for (int i = threadIdx.x; i < Kp * kRiLS; i += NT) {
        const int k = i / kRiLS, j = i % kRiLS;
        double w = 0.0;
        if (j < K && k < K) {
            w = Wt[(i64)__ldg(pidm + j) * P.nP + __ldg(pidm + k)];
            if (__ldg(srcm + k) & 1) w = -w;
        }
        wm[i] = w;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const int nrb = (K + 15) >> 4;
    const int zend = min(P.cend, z0 + W);
    const int ncb = (zend - z0 + kMixCols - 1) / kMixCols;
    const int nfc = (K + 31) / 32;
    const int nsteps = ncb * nfc;
    const int col = 8 * wid + g;
    double xp[8];
    auto load = [&](int step) {
        const int c = z0 + (step / nfc) * kMixCols + col, f0 = (step % nfc) * 32;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int r = f0 + 4 * i + t;
            xp[i] = (r < K && c < P.ld_in) ? __ldg(in + soff[r] + c) : 0.0;
        }
    };
    double c_[MAXRB][4];
#pragma unroll
    for (int rb = 0; rb < MAXRB; ++rb) c_[rb][0] = c_[rb][1] = c_[rb][2] = c_[rb][3] = 0.0;
    if (nsteps > 0) load(0);
    for (int step = 0; step < nsteps; ++step) {
        const int cbi = step / nfc, fci = step % nfc;
        const int f0 = fci * 32, nk = (min(32, K - f0) + 3) >> 2;
        double x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = xp[i];
        if (step + 1 < nsteps) load(step + 1);
        const double *la = wm + (size_t)(f0 + t) * kRiLS + g;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            // K steps of 8 (rows f0 + 8i + t and f0 + 8i + 4 + t); an odd last
            // group of 4 rows takes one step of 4
            if (2 * i + 1 < nk) {
#pragma unroll
                for (int rb = 0; rb < MAXRB; ++rb)
                    if (rb < nrb)
                        dmma_16x8x8(c_[rb],
                                    make_double2(la[(size_t)(8 * i) * kRiLS + rb * 16],
                                                 la[(size_t)(8 * i) * kRiLS + rb * 16 + 8]),
                                    make_double2(la[(size_t)(8 * i + 4) * kRiLS + rb * 16],
                                                 la[(size_t)(8 * i + 4) * kRiLS + rb * 16 + 8]),
                                    make_double2(x[2 * i], x[2 * i + 1]));
            } else if (2 * i < nk) {
#pragma unroll
                for (int rb = 0; rb < MAXRB; ++rb)
                    if (rb < nrb)
                        dmma_16x8x4(c_[rb], make_double2(la[(size_t)(8 * i) * kRiLS + rb * 16],
                                                         la[(size_t)(8 * i) * kRiLS + rb * 16 + 8]), x[2 * i]);
            }
        }
        if (fci == nfc - 1) {
            double *zr = zchunk(Z, m, K, W, cbi) + g * kMixCols + 8 * wid + 2 * t;
#pragma unroll
            for (int rb = 0; rb < MAXRB; ++rb) {
                if (rb < nrb && rb * 16 + g < K)
                    *reinterpret_cast<double2 *>(zr + rb * 16 * kMixCols) = make_double2(c_[rb][0], c_[rb][1]);
                if (rb < nrb && rb * 16 + g + 8 < K)
                    *reinterpret_cast<double2 *>(zr + (rb * 16 + 8) * kMixCols) = make_double2(c_[rb][2], c_[rb][3]);
                c_[rb][0] = c_[rb][1] = c_[rb][2] = c_[rb][3] = 0.0;
            }
        }
    }
}

// out[row][b] += sum over the pairs pq in the row's string of s(m, pq) Z[m][slot(pq)][b]
template <typename T>
__global__ void __launch_bounds__(256)
ri_gather_kernel(const RIArgs P, const int2 *__restrict__ gath, const T *__restrict__ Z, double *__restrict__ out,
                 int ld_out, int z0, int W)
{
    __shared__ long long eoff[64];
    const int row = blockIdx.x;
    for (int e = threadIdx.x; e < P.npr; e += blockDim.x) {
        const int2 g = gath[(i64)row * P.npr + e];
        const int m = g.x / P.nU, slot = g.x % P.nU;
        eoff[e] = ((long long)m * P.nU * W + slot * kMixCols) * 2 + (g.y & 1);
    }
    __syncthreads();
    const int zend = min(P.cend, z0 + W);
    for (int b = z0 + blockIdx.y * kRowChunk + threadIdx.x; b < min(zend, z0 + (blockIdx.y + 1) * kRowChunk);
         b += blockDim.x) {
        T part = T(0);
        const T *zc = Z + (i64)((b - z0) / kMixCols) * P.nU * kMixCols + (b - z0) % kMixCols;
        for (int e = 0; e < P.npr; ++e) {
            const long long o = eoff[e];
            const T v = __ldg(zc + (o >> 1));
            part += (o & 1) ? -v : v;
        }
        out[(i64)row * ld_out + b] += (double)part;
    }
}

// ---- 5. final: sigma = eps * (s~ + t^T) ---------------------------------------------
template <typename Ti>
__global__ void final_kernel(int nA, int nB, int ldB, int col_begin, int col_end, const Ti *__restrict__ bstr,
                             const u64 *__restrict__ Ka, const double *__restrict__ tT, double *__restrict__ sig)
{
    __shared__ double tile[32][33];
    const int b0 = col_begin + blockIdx.x * 32, a0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int i = ty; i < 32; i += blockDim.y) {   // t^T tile: rows b, cols a
        const int b = b0 + i, a = a0 + tx;
        tile[i][tx] = (a < nA && b < col_end) ? tT[(i64)b * ldB + a] : 0.0;
    }
    __syncthreads();
    for (int i = ty; i < 32; i += blockDim.y) {
        const int a = a0 + i, b = b0 + tx;
        if (a < nA && b < col_end) {
            const i64 idx = (i64)a * nB + b;
            double v = sig[idx] + tile[tx][i];
            if (par((u64)bstr[b] & Ka[a])) v = -v;
            sig[idx] = v;
        }
    }
}

// ---- host ------------------------------------------------------------------------------------
// in: c~ (alpha side), then c~^T (beta side); tT: the alpha side's Z, then the
// beta-side result t; Z: the beta side's Z, and the alpha side's when the
// scratch limit allows a wider chunk than tT holds.
template <typename Ti>
struct FastScratch {
    void *in = nullptr, *tT = nullptr, *Z = nullptr;
    size_t in_n = 0, tT_n = 0, z_n = 0;
    ~FastScratch() {
        for (void *p : {in, tT, Z})
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

static size_t scratch_limit()
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
    cudaError_t e = dmalloc(p, bytes);
    if (e != cudaSuccess) { *p = nullptr; return cuda_status(e, "sigma scratch"); }
    *have = bytes;
    return BSIM_OK;
}

// BSIM_MIXED_ROWS80=0 keeps the 64-row FP32 mixed GEMM passes for 65..80
// connected singles (comparison and tests).
static bool mixed_rows80_off()
{
    const char *e = getenv("BSIM_MIXED_ROWS80");
    return e && e[0] == '0';
}

// Largest shared-memory footprint for which the mixed GEMM keeps the source row
// on chip (BSIM_MIXED_ROW_SMEM bytes lowers it, which moves the row to global
// memory at small sizes too).
static size_t mixed_row_limit()
{
    const char *e = getenv("BSIM_MIXED_ROW_SMEM");
    return e ? (size_t)atoll(e) : kSmemMax;
}

// Intermediate Z of one stage: chunk width (columns, a multiple of kMixCols) and
// buffer.  A buffer that is free during the stage (spare) is used when it holds
// at least the width the scratch limit would give; otherwise the Z scratch
// grows to the limit.
struct ZSlot {
    void *p;
    size_t w;
};
static int z_slot(void **zbuf, size_t *zhave, void *spare, size_t spare_n, size_t per_col, int ncols, ZSlot *out)
{
    const size_t need = ((size_t)ncols + kMixCols - 1) / kMixCols * kMixCols;
    const size_t wb = std::min(need, std::max<size_t>(kMixCols, (scratch_limit() / per_col) / kMixCols * kMixCols));
    const size_t ws = spare ? std::min(need, (spare_n / per_col) / kMixCols * kMixCols) : 0;
    if (ws >= wb) { *out = ZSlot{spare, ws}; return BSIM_OK; }
    const int rc = ensure(zbuf, zhave, per_col * wb);
    if (rc != BSIM_OK) return rc;
    *out = ZSlot{*zbuf, wb};
    return BSIM_OK;
}

template <typename Ti>
bool fast_sigma_available(const DevBasis<Ti> *B, const DevNet<Ti> *N)
{
    FastState<Ti> *st = nullptr;
    if (get_fast(B, N, &st) != BSIM_OK) return false;
    return st->plan.ok;
}

// Optional per-stage CUDA-event timing of one structured sigma (measurement
// entry point bsim_hvec_stage_times); stages: 0 frame+transpose, 1 pure alpha,
// 2 pure beta, 3 mixed GEMM, 4 mixed gather, 5 final combine, 6 residual groups,
// 7 intermediate-string GEMM, 8 intermediate-string gather.
struct StageTimer {
    struct Mark { cudaEvent_t e0, e1; int stage; };
    std::vector<Mark> marks;
    int begin(int stage, cudaStream_t s)
    {
        Mark m{nullptr, nullptr, stage};
        BSIM_CUDA(cudaEventCreate(&m.e0));
        BSIM_CUDA(cudaEventCreate(&m.e1));
        BSIM_CUDA(cudaEventRecord(m.e0, s));
        marks.push_back(m);
        return BSIM_OK;
    }
    int end(cudaStream_t s)
    {
        BSIM_CUDA(cudaEventRecord(marks.back().e1, s));
        return BSIM_OK;
    }
    int collect(double *ms, int *launches, int n)
    {
        for (int i = 0; i < n; ++i) { ms[i] = 0.0; launches[i] = 0; }
        for (auto &m : marks) {
            float t = 0.f;
            BSIM_CUDA(cudaEventSynchronize(m.e1));
            BSIM_CUDA(cudaEventElapsedTime(&t, m.e0, m.e1));
            if (m.stage < n) { ms[m.stage] += t; launches[m.stage] += 1; }
        }
        return BSIM_OK;
    }
    ~StageTimer()
    {
        for (auto &m : marks) { cudaEventDestroy(m.e0); cudaEventDestroy(m.e1); }
    }
};

#define STAGE(tm, id, s, ...)                                   \
    do {                                                        \
        if (tm) { int rc__ = (tm)->begin(id, s); if (rc__) return rc__; } \
        __VA_ARGS__;                                            \
        if (tm) { int rc__ = (tm)->end(s); if (rc__) return rc__; } \
    } while (0)

template <typename Ti, typename T, int EPT, bool STREAM, bool GROW>
static int launch_mixed_shape(const DevBasis<Ti> *B, FastPlan<Ti> &P, const MixedArgs &ma, const T *ct, T *Z,
                              double *dst, int c0, int c1, size_t Wz, size_t smem, cudaStream_t s, StageTimer *tm)
{
    constexpr int NT = sizeof(T) == 8 ? 512 : 256;
    constexpr int ROWS = sizeof(T) == 8 ? 64 : (NT / 32) * EPT;
    auto kern = mixed_gemm_kernel<Ti, T, EPT, STREAM, GROW>;
    BSIM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int passes = (P.M + ROWS - 1) / ROWS;   // ROWS connected excitations per GEMM pass
    for (int z0 = c0; z0 < c1; z0 += (int)Wz) {
        for (int pass = 0; pass < passes; ++pass)
            STAGE(tm, 3, s, (kern<<<P.nA, NT, smem, s>>>(ma, P.d_astr, ct, Z, z0, (int)Wz, ROWS * pass)));
        dim3 g(P.nA, (unsigned)((std::min<size_t>(Wz, c1 - z0) + kRowChunk - 1) / kRowChunk));
        STAGE(tm, 4, s, (mixed_gather_kernel<Ti, T><<<g, 256, 0, s>>>(ma, B->view, Z, dst, z0, (int)Wz)));
    }
    return BSIM_OK;
}

// BSIM_MIXED_DMMA=0 sends the FP64 mixed GEMM to the shared-X-slice kernel
// (read on every call: tests compare the two)
static bool mixed_dmma_on()
{
    const char *e = getenv("BSIM_MIXED_DMMA");
    return !(e && e[0] == '0');
}

// BSIM_MIXED_TC selects the FP32-bulk mixed GEMM kernel (read on every call:
// tests compare the paths): "0" the CUDA-core kernel, "global64" / "global80"
// the tensor-core kernel with the source row read from global memory and 64 /
// 80 excitations per pass wherever it applies, unset the automatic choice.
enum class MixedTc { off, automatic, global64, global80 };
static MixedTc mixed_tc_mode()
{
    const char *e = getenv("BSIM_MIXED_TC");
    if (!e || !e[0]) return MixedTc::automatic;
    if (e[0] == '0') return MixedTc::off;
    if (!strcmp(e, "global64")) return MixedTc::global64;
    if (!strcmp(e, "global80")) return MixedTc::global80;
    return MixedTc::automatic;
}

template <typename Ti, typename T, int EPT>
static int launch_mixed(const DevBasis<Ti> *B, FastPlan<Ti> &P, FastScratch<Ti> &S, const T *ct, double *dst,
                        int c0, int c1, cudaStream_t s, StageTimer *tm)
{
    const size_t per_col = (size_t)P.nA * P.M * sizeof(T);
    ZSlot z;
    int rc = z_slot(&S.Z, &S.z_n, S.tT, S.tT_n, per_col, c1 - c0, &z);
    if (rc != BSIM_OK) return rc;
    MixedArgs ma{P.nA, P.nB, P.nE, P.nF, P.M, P.ldA, P.ldG, c1, P.d_Emask, P.d_mA,
                 sizeof(T) == 8 ? (const void *)P.d_Lam : (const void *)P.d_Lam32, P.d_gidx};
    if constexpr (sizeof(T) == 4) {
        // FP32 bulk: the tensor-core (TF32 x 3) kernel, with the source row on chip
        // where it fits, else gathered from global memory (80 excitations per pass
        // when 65..80 are connected, as at 18 orbitals with 8 electrons)
        int tcN = 0;
        bool tcGrow = false;
        const MixedTc mode = mixed_tc_mode();
        const bool fit80 = P.M <= 80 && mixed_tc_smem(P.ldA, P.nF, 80, true) <= kSmemMax;
        const bool fit64g = mixed_tc_smem(P.ldA, P.nF, 64, true) <= kSmemMax;
        if (mode == MixedTc::global80 && fit80) tcN = 80, tcGrow = true;
        else if (mode == MixedTc::global64 && fit64g) tcN = 64, tcGrow = true;
        else if (mode != MixedTc::off) {
            if (mixed_tc_smem(P.ldA, P.nF, 64, false) <= std::min(kSmemMax, mixed_row_limit())) tcN = 64;
            else if (P.M > 64 && fit80) tcN = 80, tcGrow = true;
            else if (fit64g) tcN = 64, tcGrow = true;
        }
        if (tcN > 0) {
            const int passes = (P.M + tcN - 1) / tcN;
            T *Z = static_cast<T *>(z.p);
            const size_t Wz = z.w;
            for (int z0 = c0; z0 < c1; z0 += (int)Wz) {
                for (int pass = 0; pass < passes; ++pass)
                    STAGE(tm, 3, s, rc = mixed_gemm_tc<Ti>(ma, P.d_astr, ct, Z, z0, (int)Wz, tcN * pass, tcN,
                                                           tcGrow, s));
                if (rc != BSIM_OK) return rc;
                dim3 g(P.nA, (unsigned)((std::min<size_t>(Wz, c1 - z0) + kRowChunk - 1) / kRowChunk));
                STAGE(tm, 4, s, (mixed_gather_kernel<Ti, T><<<g, 256, 0, s>>>(ma, B->view, Z, dst, z0, (int)Wz)));
            }
            return BSIM_OK;
        }
    }
    if constexpr (sizeof(T) == 8) {
        // FP64: per-warp B fragments, the source row on chip where it fits
        if (mixed_dmma_on()) {
            const bool on_chip = mixed_dmma_smem(P.ldA, P.nF, false) <= std::min(kSmemMax, mixed_row_limit());
            const size_t smem = mixed_dmma_smem(P.ldA, P.nF, !on_chip);
            if (smem <= kSmemMax) {
                auto kern = on_chip ? mixed_dmma_kernel<Ti, false> : mixed_dmma_kernel<Ti, true>;
                BSIM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                const int passes = (P.M + 63) / 64;
                T *Z = static_cast<T *>(z.p);
                const size_t Wz = z.w;
                for (int z0 = c0; z0 < c1; z0 += (int)Wz) {
                    for (int pass = 0; pass < passes; ++pass)
                        STAGE(tm, 3, s, (kern<<<P.nA, 512, smem, s>>>(ma, P.d_astr, ct, Z, z0, (int)Wz, 64 * pass)));
                    dim3 g(P.nA, (unsigned)((std::min<size_t>(Wz, c1 - z0) + kRowChunk - 1) / kRowChunk));
                    STAGE(tm, 4, s, (mixed_gather_kernel<Ti, T><<<g, 256, 0, s>>>(ma, B->view, Z, dst, z0, (int)Wz)));
                }
                return BSIM_OK;
            }
        }
    }
    const int rows = (sizeof(T) == 4 && EPT == 10) ? 80 : 64;
    const MixedShape sh = mixed_shape(P.nB, P.nF, sizeof(T), mixed_row_limit(), rows);
    if (sh.smem > kSmemMax) { set_error("mixed kernel needs %zu bytes of shared memory", sh.smem); return BSIM_ERR_UNSUPPORTED; }
    T *Z = static_cast<T *>(z.p);
    if (sh.grow)
        return sh.stream ? launch_mixed_shape<Ti, T, EPT, true, true>(B, P, ma, ct, Z, dst, c0, c1, z.w, sh.smem, s, tm)
                         : launch_mixed_shape<Ti, T, EPT, false, true>(B, P, ma, ct, Z, dst, c0, c1, z.w, sh.smem, s, tm);
    return sh.stream ? launch_mixed_shape<Ti, T, EPT, true, false>(B, P, ma, ct, Z, dst, c0, c1, z.w, sh.smem, s, tm)
                     : launch_mixed_shape<Ti, T, EPT, false, false>(B, P, ma, ct, Z, dst, c0, c1, z.w, sh.smem, s, tm);
}

// BSIM_RI_DMMA=0 sends the FP64 intermediate-string GEMM to the shared-slice
// kernel instead of the per-warp-fragment one (read on every call: tests
// compare the two)
static bool ri_dmma_on()
{
    const char *e = getenv("BSIM_RI_DMMA");
    return !(e && e[0] == '0');
}

// BSIM_RI_TC=0 sends the FP32-bulk intermediate-string GEMM to the CUDA-core
// kernel (read on every call: tests compare the two paths)
static bool ri_tc_on()
{
    const char *e = getenv("BSIM_RI_TC");
    return !(e && e[0] == '0');
}

// Same-spin doubles of one side through the intermediate strings, columns [c0, c1)
// of the side's rows (all rows), accumulated into out.
template <typename T, int EPT>
static int launch_ri(const RISide &R, const T *in, int ld_in, double *out, int ld_out, int nrows, int c0, int c1,
                     void **zbuf, size_t *zhave, void *spare, size_t spare_n, cudaStream_t s, StageTimer *tm)
{
    constexpr int NT = (64 / EPT) * 32;
    if (c1 <= c0) return BSIM_OK;
    const size_t per_col = (size_t)R.nM * R.nU * sizeof(T);
    ZSlot z;
    int rc = z_slot(zbuf, zhave, spare, spare_n, per_col, c1 - c0, &z);
    if (rc != BSIM_OK) return rc;
    const size_t Wz = z.w;
    RIArgs ra{R.nM, R.nU, R.npr, R.nP, ld_in, c1, R.src, R.pid,
              sizeof(T) == 8 ? (const void *)R.W : (const void *)R.W32};
    const size_t smem = ri_smem_bytes(R.nU, sizeof(T));
    BSIM_CUDA(cudaFuncSetAttribute(ri_gemm_kernel<T, EPT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    T *Z = static_cast<T *>(z.p);
    if constexpr (sizeof(T) == 8) {
        // FP64: per-warp B fragments, all rows on the DMMA path (measured per
        // sigma: 45.5 against 49.7 ms at 16o, 712 against 772 ms at 18o for
        // the shared-slice kernel)
        if (ri_dmma_on() && R.nU <= kRiMaxU && ri_dmma_smem(R.nU) <= kSmemMax) {
            const size_t sm = ri_dmma_smem(R.nU);
            BSIM_CUDA(cudaFuncSetAttribute(ri_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
            for (int z0 = c0; z0 < c1; z0 += (int)Wz) {
                STAGE(tm, 7, s, (ri_dmma_kernel<<<R.nM, 512, sm, s>>>(ra, in, Z, z0, (int)Wz)));
                dim3 g(nrows, (unsigned)((std::min<size_t>(Wz, c1 - z0) + kRowChunk - 1) / kRowChunk));
                STAGE(tm, 8, s, (ri_gather_kernel<T><<<g, 256, 0, s>>>(ra, R.gath, Z, out, ld_out, z0, (int)Wz)));
            }
            return BSIM_OK;
        }
    }
    // FP32 bulk: the tensor-core (TF32 x 3) kernel
    bool tc = false;
    if constexpr (sizeof(T) == 4) tc = ri_tc_on() && ri_tc_supported(R.nU) && ri_tc_smem(R.nU) <= kSmemMax;
    for (int z0 = c0; z0 < c1; z0 += (int)Wz) {
        if constexpr (sizeof(T) == 4) {
            if (tc) {
                STAGE(tm, 7, s, rc = ri_gemm_tc(ra, in, Z, z0, (int)Wz, s));
                if (rc != BSIM_OK) return rc;
            }
        }
        if (!tc) STAGE(tm, 7, s, (ri_gemm_kernel<T, EPT><<<R.nM, NT, smem, s>>>(ra, in, Z, z0, (int)Wz)));
        dim3 g(nrows, (unsigned)((std::min<size_t>(Wz, c1 - z0) + kRowChunk - 1) / kRowChunk));
        STAGE(tm, 8, s, (ri_gather_kernel<T><<<g, 256, 0, s>>>(ra, R.gath, Z, out, ld_out, z0, (int)Wz)));
    }
    return BSIM_OK;
}

template <typename Ti, typename T>
static int run_fast(const DevBasis<Ti> *B, const DevNet<Ti> *N, FastState<Ti> *st, const double *src,
                    const float *src32, double *dst, int c0, int c1, cudaStream_t s, StageTimer *tm)
{
    FastPlan<Ti> &P = st->plan;
    FastScratch<Ti> &S = st->scratch;
    const int nA = P.nA, nB = P.nB;
    int rc;
    const size_t in_bytes = std::max((size_t)nA * P.ldA, (size_t)nB * P.ldB) * sizeof(T);
    if ((rc = ensure(&S.in, &S.in_n, in_bytes)) != BSIM_OK) return rc;
    if ((rc = ensure(&S.tT, &S.tT_n, (size_t)nB * P.ldB * sizeof(double))) != BSIM_OK) return rc;
    T *in = static_cast<T *>(S.in);
    double *tT = static_cast<double *>(S.tT);
    dim3 tgrid((nB + 31) / 32, (nA + 31) / 32), tblk(32, 8);
    auto frame = [&](T *ct, T *ctT) {
        if (src32)
            frame_transpose_kernel<Ti, float, T><<<tgrid, tblk, 0, s>>>(nA, nB, P.ldA, P.ldB, P.d_bstr, P.d_Ka, src32,
                                                                         ct, ctT);
        else
            frame_transpose_kernel<Ti, double, T><<<tgrid, tblk, 0, s>>>(nA, nB, P.ldA, P.ldB, P.d_bstr, P.d_Ka, src,
                                                                          ct, ctT);
    };
    // FP64: 16 warps of DMMA 8x8 tiles; FP32: 8 warps of 8 x 4 f32x2 register tiles
    constexpr int kEPT = sizeof(T) == 8 ? 4 : 8;
    // ---- alpha side: c~ in `in`, results into dst; tT's buffer is free for Z ----
    STAGE(tm, 0, s, frame(in, nullptr));
    {   // pure alpha + diagonal -> dst (the frame's s~)
        dim3 g(nA, (c1 - c0 + kRowChunk - 1) / kRowChunk);
        STAGE(tm, 1, s, (pure_rows_kernel<T><<<g, 256, 0, s>>>(0, c0, c1, P.ldA, P.csrA, in, dst, nB,
                                                               P.rank_d ? P.d_PAd : nullptr, P.d_PBdT, P.rank_d)));
    }
    if (P.riA.on) {   // same-spin alpha doubles through intermediate strings -> dst
        rc = launch_ri<T, kEPT>(P.riA, in, P.ldA, dst, nB, nA, c0, c1, &S.Z, &S.z_n, S.tT, S.tT_n, s, tm);
        if (rc != BSIM_OK) return rc;
    }
    if (P.nE > 0 && P.nF > 0 && P.M > 0) {
        // FP32 with 65..80 connected singles: one 80-row pass instead of 64 + 16 rows
        bool done = false;
        if constexpr (sizeof(T) == 4) {
            if (P.M > 64 && P.M <= 80 && !mixed_rows80_off()) {
                rc = launch_mixed<Ti, T, 10>(B, P, S, in, dst, c0, c1, s, tm);
                done = true;
            }
        }
        if (!done) rc = launch_mixed<Ti, T, kEPT>(B, P, S, in, dst, c0, c1, s, tm);
        if (rc != BSIM_OK) return rc;
    }
    // ---- beta side: c~^T in `in`, result t^T in tT (the beta doubles through
    //      intermediates when the whole sigma is computed, else through the rows) ----
    STAGE(tm, 0, s, frame(nullptr, in));
    const bool ri_b = P.riB.on && c0 == 0 && c1 == nB;
    {
        dim3 g(c1 - c0, (nA + kRowChunk - 1) / kRowChunk);
        STAGE(tm, 2, s, (pure_rows_kernel<T><<<g, 256, 0, s>>>(c0, 0, nA, P.ldB, ri_b ? P.csrBri : P.csrB, in, tT,
                                                               P.ldB, nullptr, nullptr, 0)));
    }
    if (ri_b) {
        rc = launch_ri<T, kEPT>(P.riB, in, P.ldB, tT, P.ldB, nB, 0, nA, &S.Z, &S.z_n, nullptr, 0, s, tm);
        if (rc != BSIM_OK) return rc;
    }
    // ---- final combine ----
    dim3 fgrid((c1 - c0 + 31) / 32, (nA + 31) / 32);
    STAGE(tm, 5, s, (final_kernel<Ti><<<fgrid, tblk, 0, s>>>(nA, nB, P.ldB, c0, c1, P.d_bstr, P.d_Ka, tT, dst)));
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename Ti>
static int sigma_fast_impl(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *src, const float *src32,
                           double *dst, bool mixed, cudaStream_t s, bool *used, StageTimer *tm)
{
    *used = false;
    FastState<Ti> *st = nullptr;
    int rc = get_fast(B, N, &st);
    if (rc != BSIM_OK) return rc;
    if (!st->plan.ok) return BSIM_OK;
    rc = mixed ? run_fast<Ti, float>(B, N, st, src, src32, dst, 0, st->plan.nB, s, tm)
               : run_fast<Ti, double>(B, N, st, src, nullptr, dst, 0, st->plan.nB, s, tm);
    if (rc != BSIM_OK) return rc;
    if (!st->plan.residual.empty()) {
        STAGE(tm, 6, s, rc = sigma_generic_accumulate(B, N, st->plan.d_resid, st->plan.d_resid_chunks,
                                                      st->plan.n_resid_chunks, src, src32, dst, mixed, s));
        if (rc != BSIM_OK) return rc;
    }
    *used = true;
    return BSIM_OK;
}

template <typename Ti>
int sigma_fast(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *src, const float *src32, double *dst,
               bool mixed, cudaStream_t s, bool *used)
{
    return sigma_fast_impl(B, N, src, src32, dst, mixed, s, used, (StageTimer *)nullptr);
}

template <typename Ti>
int sigma_fast_cols(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *src, double *dst, bool mixed,
                    i64 col_lo, i64 col_hi, cudaStream_t s)
{
    FastState<Ti> *st = nullptr;
    int rc = get_fast(B, N, &st);
    if (rc != BSIM_OK) return rc;
    const FastPlan<Ti> &P = st->plan;
    if (!P.ok || !P.residual.empty()) {
        set_error("column-band sigma needs the structured path with no residual groups (%s)",
                  P.ok ? "residual groups" : P.why.c_str());
        return BSIM_ERR_UNSUPPORTED;
    }
    if (col_lo < 0 || col_hi > P.nB || col_lo > col_hi || (col_lo % kMixCols) != 0) {
        set_error("column band [%lld, %lld) must lie in [0, %d) and start on a multiple of %d", (long long)col_lo,
                  (long long)col_hi, P.nB, kMixCols);
        return BSIM_ERR_ARG;
    }
    if (col_lo == col_hi) return BSIM_OK;
    return mixed ? run_fast<Ti, float>(B, N, st, src, nullptr, dst, (int)col_lo, (int)col_hi, s, nullptr)
                 : run_fast<Ti, double>(B, N, st, src, nullptr, dst, (int)col_lo, (int)col_hi, s, nullptr);
}

template <typename Ti>
int sigma_fast_stages(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *src, double *dst, bool mixed,
                      cudaStream_t s, double *ms, int *launches, int nstages)
{
    StageTimer tm;
    bool used = false;
    int rc = sigma_fast_impl(B, N, src, nullptr, dst, mixed, s, &used, &tm);
    if (rc != BSIM_OK) return rc;
    if (!used) { set_error("the structured sigma path is off for this basis and network"); return BSIM_ERR_UNSUPPORTED; }
    return tm.collect(ms, launches, nstages);
}

template <typename Ti>
int fast_sigma_info(const DevBasis<Ti> *B, const DevNet<Ti> *N, std::string *why, int *nresid)
{
    FastState<Ti> *st = nullptr;
    int rc = get_fast(B, N, &st);
    if (rc != BSIM_OK) return rc;
    *why = st->plan.ok ? std::string("structured") + (st->plan.riA.on ? " ri-alpha" : "") +
                             (st->plan.riB.on ? " ri-beta" : "")
                       : st->plan.why;
    *nresid = (int)st->plan.residual.size();
    return st->plan.ok ? (st->plan.row64 ? 1 : 2) : 0;
}

template int fast_sigma_info<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, std::string *, int *);
template bool fast_sigma_available<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *);
template int sigma_fast<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, const double *, const float *,
                                  double *, bool, cudaStream_t, bool *);
template int sigma_fast_cols<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, const double *, double *,
                                       bool, i64, i64, cudaStream_t);
template int sigma_fast_stages<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, const double *, double *,
                                         bool, cudaStream_t, double *, int *, int);

template int fast_sigma_info<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, std::string *, int *);
template bool fast_sigma_available<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *);
template int sigma_fast<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, const double *, const float *,
                                  double *, bool, cudaStream_t, bool *);
template int sigma_fast_cols<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, const double *, double *,
                                       bool, i64, i64, cudaStream_t);
template int sigma_fast_stages<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, const double *, double *,
                                         bool, cudaStream_t, double *, int *, int);

}  // namespace bsim
