// FP32-bulk mixed GEMM of the structured sigma on the 5th-generation tensor
// cores (tcgen05.mma kind::tf32, accumulators in tensor memory).
//
// Per source row a' the mixed part of sigma needs Y[j][b] = sum_F Lam_conn[j][F]
// X[F][b], X[F][b] = sB_F c~[a'][b ^ F] gathered from the row (see
// mixed_gemm_kernel in sigma_fast.cu).  Here the product is computed transposed,
// D[b][j] = sum_F X^T[b][F] Lam_conn^T[F][j], so that 128 columns b of a chunk are
// the MMA's M = 128 rows (one TMEM lane each) and the <= 64 connected excitations
// j are its N = 64 columns.  FP32 accuracy from TF32 inputs: every operand is
// split into x = hi + lo, hi = x with its 13 low mantissa bits cleared (exact in
// TF32) and lo = x - hi (exact in FP32), and D accumulates hi*hi + hi*lo + lo*hi
// in FP32 (Ootomo & Yokota 2022, "Recovering single precision accuracy from
// Tensor Cores while surpassing the FP32 theoretical peak"; the lo*lo term,
// ~2^-22 relative, is dropped).
//
// Shapes: N = 64 connected excitations per pass with the source row staged in
// shared memory (up to 16 orbitals with 8 electrons), or, when the row does not
// fit (18 orbitals: a 175 KB FP32 row), the row gathered from global memory (L2)
// with N = 64 or 80 (the 80 connected singles of 8 electrons in 18 orbitals in
// one pass).
//
// Warp roles (672 threads, one CTA per source row, one pass of N excitations):
//   warps 0-3   epilogue: tcgen05.ld of D (warp w reads TMEM lanes 32w..32w+31)
//               and the store of Z[a'][j][b];
//   warps 4-19  producers: the X^T slice of 40 F rows, gathered from the source
//               row in shared memory, split, written in the canonical K-major
//               layout (8-row x 16-byte core matrices) into a double buffer (the
//               gathers bound the kernel: 16 warps keep the tensor pipe fed);
//   warp 20     TMEM allocation (two N-column accumulators) and, lane 0, the
//               MMA issue: 3 MMAs of 128 x N x 8 per K step.
// Handoffs are mbarriers: afull/aempty per A buffer (producers -> MMA; the MMA
// completion, by tcgen05.commit, frees the buffer), dfull/dempty per
// accumulator (MMA -> epilogue and back).  Every wait is bounded: a wait that
// gives up (after 20 ms) raises the CTA's abort flag (every other wait then
// returns) and a device-wide one (later CTAs return at once), counts a timeout
// in g_tc_timeouts, and the CTA still waits (bounded) for its issued MMAs and
// frees its tensor memory before it exits.
#include "mixed.cuh"
#include "ops.h"

#include <cstdlib>

namespace bsim {

namespace {

constexpr int kTcThreads = 672;
constexpr int kTcProdWarps = 16;          // warps 4..19
constexpr int kTcMmaWarp = 20;
constexpr int kTcKS = 40;                 // F rows per A slice (a multiple of 8)
constexpr int kTcM = 128;                 // columns b per chunk: MMA M
template <int N> struct TcShape {
    static constexpr uint32_t tmem_cols = N <= 64 ? 128u : 256u;   // two N-column accumulators, a power of 2
};
constexpr unsigned long long kTcWaitNs = 20000000ull;   // a wait gives up after 20 ms
constexpr long kTcSpinCap = 1L << 26;                   // and after this many rounds in any case
constexpr uint32_t kCoreBytes = 128;      // one core matrix: 8 rows x 16 bytes (4 TF32)
// instruction descriptor of kind::tf32: D FP32 (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
template <int N>
constexpr uint32_t idesc_tf32() { return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
                                         ((uint32_t)(kTcM >> 4) << 24); }

__device__ int g_tc_timeouts;   // waits that gave up
__device__ int g_tc_abort;      // set with the first of them: later CTAs return at once

// Shared-memory layout (bytes from the dynamic base, 128-byte aligned pieces).
struct TcLayout {
    uint32_t srow, bh, bl, ah0, ah1, al0, al1, conn, sgn, bars, tmem, total;
    int kp8;        // K rounded up to the MMA's K step (8)
    uint32_t sbo_b; // byte stride between 8-row groups of B (all K chunks of a group)
};
__host__ __device__ inline uint32_t align128(uint32_t x) { return (x + 127u) & ~127u; }
__host__ __device__ inline TcLayout tc_layout(int ldA, int nF, int N, bool grow)
{
    TcLayout L{};
    L.kp8 = (nF + 7) & ~7;
    L.sbo_b = (uint32_t)(L.kp8 / 4) * kCoreBytes;
    const uint32_t bbytes = (uint32_t)(N / 8) * L.sbo_b;
    const uint32_t abytes = (uint32_t)(kTcM / 8) * (kTcKS / 4) * kCoreBytes;
    uint32_t o = 0;
    L.srow = o; o = align128(o + (grow ? 0u : (uint32_t)ldA * 4));
    L.bh = o; o = align128(o + bbytes);
    L.bl = o; o = align128(o + bbytes);
    L.ah0 = o; o = align128(o + abytes);
    L.ah1 = o; o = align128(o + abytes);
    L.al0 = o; o = align128(o + abytes);
    L.al1 = o; o = align128(o + abytes);
    L.conn = o; o = align128(o + kMaxConn * 4);
    L.sgn = o; o = align128(o + kMaxConn * 4);
    L.bars = o; o = align128(o + 9 * 8);
    L.tmem = o; o = align128(o + 4);
    L.total = o;
    return L;
}

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t a)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}"
                 : "=r"(ok)
                 : "r"(a), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for the phase of the given parity; false when the CTA aborts
// (its own wait gave up, another wait of the CTA did, or another CTA's did).
__device__ bool mbar_wait(uint32_t a, uint32_t parity, volatile int *abort_flag)
{
    const unsigned long long t0 = global_ns();
    for (long i = 0; i < kTcSpinCap; ++i) {
        if (mbar_try(a, parity)) return true;
        if (*abort_flag) return false;
        if ((i & 63) == 63) {
            if (*(volatile int *)&g_tc_abort) { *abort_flag = 1; return false; }
            if (global_ns() - t0 > kTcWaitNs) break;
        }
    }
    *abort_flag = 1;
    atomicExch(&g_tc_abort, 1);
    atomicAdd(&g_tc_timeouts, 1);
    return false;
}

// Bounded wait that ignores the abort flags: the wait for this CTA's own MMAs
// before its tensor memory is freed.
__device__ void mbar_wait_drain(uint32_t a, uint32_t parity)
{
    const unsigned long long t0 = global_ns();
    for (long i = 0; i < kTcSpinCap; ++i) {
        if (mbar_try(a, parity)) return;
        if ((i & 63) == 63 && global_ns() - t0 > kTcWaitNs) break;
    }
    atomicExch(&g_tc_abort, 1);
    atomicAdd(&g_tc_timeouts, 1);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared-memory matrix descriptor: no swizzle (canonical K-major core matrices),
// leading byte offset = next K chunk, stride byte offset = next 8-row group,
// descriptor version 1 (bits 46-47).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
                 "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
                 : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane, waited for.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                 "%12, %13, %14, %15}, [%16];\n\ttcgen05.wait::ld.sync.aligned;"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(taddr)
                 : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tf32_split(float x, float &hi, float &lo)
{
    hi = __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
    lo = x - hi;
}

// byte offset of element (row r, k) inside a K-major operand whose 8-row
// groups are sbo bytes apart (K chunks of 4 elements 128 bytes apart)
__device__ __forceinline__ uint32_t kmajor_off(int r, int k, uint32_t sbo)
{
    return (uint32_t)(r >> 3) * sbo + (uint32_t)(k >> 2) * kCoreBytes + (uint32_t)(r & 7) * 16u + (uint32_t)(k & 3) * 4u;
}

template <typename Ti, int N, bool GROW>
__global__ void __launch_bounds__(kTcThreads, 1)
mixed_gemm_tc_kernel(const MixedArgs P, const Ti *__restrict__ astr, const float *__restrict__ ct,
                     float *__restrict__ Z, int z0, int W, int jbase)
{
    static_assert(N % 16 == 0 && N >= 16 && N <= 128, "MMA N for M = 128: a multiple of 16");
    constexpr uint32_t kTmemCols = TcShape<N>::tmem_cols;
    constexpr uint32_t kIdesc = idesc_tf32<N>();
    extern __shared__ __align__(1024) unsigned char smem[];
    const TcLayout L = tc_layout(P.ldA, P.nF, N, GROW);
    const int K = P.nF;
    float *srow = reinterpret_cast<float *>(smem + L.srow);
    int *conn = reinterpret_cast<int *>(smem + L.conn);
    int *sgn = reinterpret_cast<int *>(smem + L.sgn);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + L.tmem);
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
    const uint32_t bar0 = sbase + L.bars;   // afull[2], aempty[2], dfull[2], dempty[2], done
    auto afull = [&](int i) { return bar0 + 8u * (uint32_t)i; };
    auto aempty = [&](int i) { return bar0 + 8u * (uint32_t)(2 + i); };
    auto dfull = [&](int i) { return bar0 + 8u * (uint32_t)(4 + i); };
    auto dempty = [&](int i) { return bar0 + 8u * (uint32_t)(6 + i); };
    const uint32_t done = bar0 + 64u;
    __shared__ int wcnt[kTcThreads / 32], cnt;
    __shared__ volatile int abort_flag;
    __shared__ int skip_all;
    const int a = blockIdx.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) skip_all = *(volatile int *)&g_tc_abort;
    __syncthreads();
    if (skip_all) return;   // an earlier CTA gave up a wait: the result is void (counted)
    const int m = connected_excitations<kTcThreads>(P, (u64)astr[a], conn, sgn, wcnt, &cnt);
    const int jm = min(N, m - jbase);
    if (jm <= 0) return;   // uniform across the CTA

    // ---- stage the source row and B = Lam_conn^T (hi and lo) ----
    {
        if (!GROW) {
            const int4 *src = reinterpret_cast<const int4 *>(ct + (i64)a * P.ldA);
            int4 *dst = reinterpret_cast<int4 *>(srow);
            const int n16 = P.ldA / 4;
            for (int i = threadIdx.x; i < n16; i += kTcThreads) dst[i] = __ldg(src + i);
        }
        const float *Lam = static_cast<const float *>(P.Lam);
        const int nk4 = L.kp8 / 4;
        // core matrix cm = (row group rg, K chunk kc); element e = (row r, k within chunk)
        for (int i = threadIdx.x; i < N * L.kp8; i += kTcThreads) {
            const int cm = i >> 5, e = i & 31;
            const int j = (cm / nk4) * 8 + (e & 7), f = (cm % nk4) * 4 + (e >> 3);
            const float x = (j < jm && f < K) ? (float)sgn[jbase + j] * Lam[(i64)conn[jbase + j] * K + f] : 0.f;
            float hi, lo;
            tf32_split(x, hi, lo);
            const uint32_t off = kmajor_off(j, f, L.sbo_b);
            *reinterpret_cast<float *>(smem + L.bh + off) = hi;
            *reinterpret_cast<float *>(smem + L.bl + off) = lo;
        }
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            mbar_init(afull(i), 32 * kTcProdWarps);
            mbar_init(aempty(i), 1);
            mbar_init(dfull(i), 1);
            mbar_init(dempty(i), 128);
        }
        mbar_init(done, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == kTcMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + L.tmem),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();   // B (generic-proxy stores) is read by the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const int zend = min(P.cend, z0 + W);
    const int ncb = (zend - z0 + kTcM - 1) / kTcM;
    const int nsl = (L.kp8 + kTcKS - 1) / kTcKS;
    const int nq = ncb * nsl;
    const uint32_t ah[2] = {sbase + L.ah0, sbase + L.ah1}, al[2] = {sbase + L.al0, sbase + L.al1};
    constexpr uint32_t kSboA = (kTcKS / 4) * kCoreBytes;   // 8-row groups of an A slice

    if (warp >= 4 && warp < 4 + kTcProdWarps) {
        // ---- producers ----
        // Producer warp pw owns core matrices cm = pw + 16 it (it < 10) of every
        // slice: 8 rows b (lanes & 7) x 4 slice rows f (lanes >> 3).  Their offsets
        // into the gather table (without the slice's f0 * ldG + cb), their slice
        // rows and their shared-memory offsets do not change between slices.
        const int pw = warp - 4;
        constexpr int nkc = kTcKS / 4, ncm = (kTcM / 8) * nkc;   // 160 core matrices per slice
        constexpr int PI = ncm / kTcProdWarps;
        static_assert(PI * kTcProdWarps == ncm, "every producer warp owns the same number of core matrices");
        int goff[PI], foff[PI], gp[PI];
        float gv[GROW ? PI : 1];   // GROW: the next slice's values, gathered from the row in L2
        const float *grow = ct + (i64)a * P.ldA;
        uint32_t soff[PI];
#pragma unroll
        for (int it = 0; it < PI; ++it) {
            const int cm = pw + it * kTcProdWarps;
            const int rg = cm / nkc, kc = cm % nkc;
            foff[it] = kc * 4 + (lane >> 3);
            goff[it] = foff[it] * P.ldG + rg * 8 + (lane & 7);
            soff[it] = (uint32_t)rg * kSboA + (uint32_t)kc * kCoreBytes + (uint32_t)(lane & 7) * 16u +
                       (uint32_t)(lane >> 3) * 4u;
        }
        auto prefetch = [&](int q) {
            const int f0 = (q % nsl) * kTcKS;
            const int *gbase = P.gidx + (i64)f0 * P.ldG + z0 + (q / nsl) * kTcM;
#pragma unroll
            for (int it = 0; it < PI; ++it) gp[it] = f0 + foff[it] < K ? __ldg(gbase + goff[it]) : -1;
            if constexpr (GROW) {
#pragma unroll
                for (int it = 0; it < PI; ++it) gv[it] = gp[it] >= 0 ? __ldg(grow + (gp[it] >> 1)) : 0.f;
            }
        };
        if (nq > 0) prefetch(0);
        for (int q = 0; q < nq; ++q) {
            const int buf = q & 1;
            if (q >= 2 && !mbar_wait(aempty(buf), (uint32_t)(((q >> 1) - 1) & 1), &abort_flag)) break;
            unsigned char *ahp = smem + (buf ? L.ah1 : L.ah0), *alp = smem + (buf ? L.al1 : L.al0);
#pragma unroll
            for (int it = 0; it < PI; ++it) {
                const int g = gp[it];
                float x;
                if constexpr (GROW) x = gv[it];
                else x = g >= 0 ? srow[g >> 1] : 0.f;
                if (g & 1) x = -x;
                float hi, lo;
                tf32_split(x, hi, lo);
                *reinterpret_cast<float *>(ahp + soff[it]) = hi;
                *reinterpret_cast<float *>(alp + soff[it]) = lo;
            }
            fence_async_smem();
            mbar_arrive(afull(buf));
            if (q + 1 < nq) prefetch(q + 1);
        }
    } else if (warp == kTcMmaWarp) {
        // ---- MMA issue ----
        if (lane == 0) {
            bool ok = true;
            for (int c = 0; c < ncb && ok; ++c) {
                const int dbuf = c & 1;
                if (c >= 2 && !mbar_wait(dempty(dbuf), (uint32_t)(((c >> 1) - 1) & 1), &abort_flag)) break;
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)dbuf * N;
                for (int s = 0; s < nsl; ++s) {
                    const int q = c * nsl + s, buf = q & 1;
                    if (!mbar_wait(afull(buf), (uint32_t)((q >> 1) & 1), &abort_flag)) { ok = false; break; }
                    tc_fence_after();
                    const int f0 = s * kTcKS, nks = (min(kTcKS, L.kp8 - f0) + 7) / 8;
                    for (int ks = 0; ks < nks; ++ks) {
                        const uint32_t aoff = (uint32_t)ks * 2u * kCoreBytes;
                        const uint32_t boff = (uint32_t)(f0 / 4 + 2 * ks) * kCoreBytes;
                        const uint64_t dah = umma_desc(ah[buf] + aoff, kCoreBytes, kSboA);
                        const uint64_t dal = umma_desc(al[buf] + aoff, kCoreBytes, kSboA);
                        const uint64_t dbh = umma_desc(sbase + L.bh + boff, kCoreBytes, L.sbo_b);
                        const uint64_t dbl = umma_desc(sbase + L.bl + boff, kCoreBytes, L.sbo_b);
                        umma_tf32(d, dah, dbh, kIdesc, (s | ks) != 0 ? 1u : 0u);
                        umma_tf32(d, dah, dbl, kIdesc, 1u);
                        umma_tf32(d, dal, dbh, kIdesc, 1u);
                    }
                    umma_commit(aempty(buf));   // the slice buffer is free once these MMAs completed
                }
                if (ok) umma_commit(dfull(dbuf));
            }
            umma_commit(done);   // every issued MMA has completed before TMEM is freed
            mbar_wait_drain(done, 0u);
        }
        __syncwarp();
    } else if (warp < 4) {
        // ---- epilogue: D (TMEM lanes 32 warp .. +31 = columns b) -> Z[a'][j][b] ----
        for (int c = 0; c < ncb; ++c) {
            const int dbuf = c & 1;
            if (!mbar_wait(dfull(dbuf), (uint32_t)((c >> 1) & 1), &abort_flag)) break;
            tc_fence_after();
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)dbuf * N;
            float *zb = Z + ((i64)a * P.M + jbase) * W + c * kTcM + warp * 32 + lane;
            // 16 columns (excitations j) at a time: TMEM -> registers -> Z
            for (int i = 0; i < N / 16 && 16 * i < jm; ++i) {
                float v[16];
                tmem_ld16(taddr + 16u * (uint32_t)i, v);
#pragma unroll
                for (int k = 0; k < 16; ++k)
                    if (16 * i + k < jm) zb[(i64)(16 * i + k) * W] = v[k];
            }
            tc_fence_before();
            if (c + 2 < ncb) mbar_arrive(dempty(dbuf));
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == kTcMmaWarp)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                     : "memory");
}

}  // namespace

size_t mixed_tc_smem(int ldA, int nF, int N, bool grow) { return tc_layout(ldA, nF, N, grow).total; }

template <typename Ti>
int mixed_gemm_tc(const MixedArgs &ma, const Ti *astr, const float *ct, float *Z, int z0, int W, int jbase, int N,
                  bool grow, cudaStream_t s)
{
    const size_t smem = mixed_tc_smem(ma.ldA, ma.nF, N, grow);
    auto launch = [&](auto kern) -> int {
        BSIM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<ma.nA, kTcThreads, smem, s>>>(ma, astr, ct, Z, z0, W, jbase);
        BSIM_CUDA(cudaGetLastError());
        return BSIM_OK;
    };
    if (N == 64) return grow ? launch(mixed_gemm_tc_kernel<Ti, 64, true>) : launch(mixed_gemm_tc_kernel<Ti, 64, false>);
    if (N == 80 && grow) return launch(mixed_gemm_tc_kernel<Ti, 80, true>);
    set_error("tensor-core mixed GEMM: no kernel for %d excitations per pass", N);
    return BSIM_ERR_UNSUPPORTED;
}

int mixed_tc_timeouts(int *count, bool reset)
{
    int h = 0;
    BSIM_CUDA(cudaMemcpyFromSymbol(&h, g_tc_timeouts, sizeof(int)));
    if (reset) {
        const int z = 0;
        BSIM_CUDA(cudaMemcpyToSymbol(g_tc_timeouts, &z, sizeof(int)));
        BSIM_CUDA(cudaMemcpyToSymbol(g_tc_abort, &z, sizeof(int)));
    }
    *count = h;
    return BSIM_OK;
}

template int mixed_gemm_tc<unsigned>(const MixedArgs &, const unsigned *, const float *, float *, int, int, int, int,
                                     bool, cudaStream_t);
template int mixed_gemm_tc<unsigned long long>(const MixedArgs &, const unsigned long long *, const float *, float *,
                                               int, int, int, int, bool, cudaStream_t);

}  // namespace bsim
