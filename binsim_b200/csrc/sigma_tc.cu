// FP32-bulk GEMMs of the structured sigma on the 5th-generation tensor cores
// (tcgen05.mma kind::tf32, accumulators in tensor memory): the mixed-excitation
// product and the same-spin doubles through intermediate strings.
//
// Both are, per CTA, Y[j][b] = sum_k B[j][k] X[k][b] over the columns b of a Z
// window, with a CTA-specific B and X rows taken from c~:
//   mixed (one CTA per source row a'): B = Lam_conn (the row's connected alpha
//     excitations j), X[F][b] = sB_F c~[a'][b ^ F] gathered from the row (see
//     mixed_gemm_kernel in sigma_fast.cu);
//   intermediate (one CTA per intermediate string m): B = W_m (pair-pair
//     integrals of the pairs outside m, the sign of each source row folded in),
//     X[k][b] = c~[m + pair_k][b], whole rows of c~ (ri_gemm_kernel).
// The product is computed transposed, D[b][j] = sum_k X^T[b][k] B^T[k][j], so that
// 128 columns b of a chunk are the MMA's M = 128 rows (one TMEM lane each) and
// the j are its N columns.  FP32 accuracy from TF32 inputs: every operand is
// split into x = hi + lo, hi = x with its 13 low mantissa bits cleared (exact in
// TF32) and lo = x - hi (exact in FP32), and D accumulates hi*hi + hi*lo + lo*hi
// in FP32 (Ootomo & Yokota 2022, "Recovering single precision accuracy from
// Tensor Cores while surpassing the FP32 theoretical peak"; the lo*lo term,
// ~2^-22 relative, is dropped).
//
// Mixed shapes: N = 64 connected excitations per pass with the source row staged
// in shared memory (up to 16 orbitals with 8 electrons), or, when the row does
// not fit (18 orbitals: a 175 KB FP32 row), the row gathered from global memory
// (L2) with N = 64 or 80 (the 80 connected singles of 8 electrons in 18 orbitals
// in one pass).  Intermediate shapes: N = the pairs outside an intermediate
// rounded up to 16 (45 -> 48 at 16 orbitals, 66 -> 80 at 18).
//
// Warp roles (672 threads, one CTA per row or intermediate):
//   warps 0-3   epilogue: tcgen05.ld of D (warp w reads TMEM lanes 32w..32w+31)
//               and the store of the chunk's contiguous [j][128] block of Z;
//   warps 4-19  producers: the X^T slice of KS k rows (gathered from the source
//               row; or copied from the c~ rows with cp.async into a ring of
//               slices, RS - 1 ahead, then transposed), split, written in the
//               canonical K-major layout (8-row x 16-byte core matrices) into a
//               double buffer (the loads bound the kernel: 16 warps keep the
//               tensor pipe fed);
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
constexpr int kTcM = 128;                 // columns b per chunk: MMA M
constexpr int kMixKS = 48;                // F rows per A slice of the mixed product, row on chip
constexpr int kMixKSGrow = 40;            // the same, row read from global memory
constexpr int kMixStages = 2;             // its A stages
constexpr int kRiStages = 2, kRiRing = 4; // the intermediate product's A stages and copy-ring slots
constexpr unsigned long long kTcWaitNs = 20000000ull;   // a wait gives up after 20 ms
constexpr long kTcSpinCap = 1L << 26;                   // and after this many rounds in any case
constexpr unsigned kTcSuspendNs = 20000;                // longest sleep in one test of a phase
constexpr uint32_t kCoreBytes = 128;      // one core matrix: 8 rows x 16 bytes (4 TF32)

// two N-column accumulators, allocated as a power of 2 of at least 32 columns
template <int N>
constexpr uint32_t tmem_cols() { return N <= 16 ? 32u : N <= 32 ? 64u : N <= 64 ? 128u : 256u; }
// instruction descriptor of kind::tf32: D FP32 (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
template <int N>
constexpr uint32_t idesc_tf32() { return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
                                         ((uint32_t)(kTcM >> 4) << 24); }

__device__ int g_tc_timeouts;   // waits that gave up
__device__ int g_tc_abort;      // set with the first of them: later CTAs return at once

// Shared-memory layout (bytes from the dynamic base, 128-byte aligned pieces).
struct TcLayout {
    uint32_t srow, bh, bl, ah, al, abytes, tab, bars, tmem, total;
    int kp8;        // K rounded up to the MMA's K step (8)
    uint32_t sbo_b; // byte stride between 8-row groups of B (all K chunks of a group)
};
__host__ __device__ inline uint32_t align128(uint32_t x) { return (x + 127u) & ~127u; }
// srow_bytes: the source row staged on chip (0 when it is not); S: A stages of
// KS rows (hi and lo parts); tab_bytes: the CTA's index tables
__host__ __device__ inline TcLayout tc_layout(uint32_t srow_bytes, int K, int N, int KS, int S, uint32_t tab_bytes)
{
    TcLayout L{};
    L.kp8 = (K + 7) & ~7;
    L.sbo_b = (uint32_t)(L.kp8 / 4) * kCoreBytes;
    const uint32_t bbytes = (uint32_t)(N / 8) * L.sbo_b;
    const uint32_t abytes = (uint32_t)(kTcM / 8) * (uint32_t)(KS / 4) * kCoreBytes;
    uint32_t o = 0;
    L.srow = o; o = align128(o + srow_bytes);
    L.bh = o; o = align128(o + bbytes);
    L.bl = o; o = align128(o + bbytes);
    L.abytes = abytes;
    L.ah = o; o = align128(o + (uint32_t)S * abytes);
    L.al = o; o = align128(o + (uint32_t)S * abytes);
    L.tab = o; o = align128(o + tab_bytes);
    L.bars = o; o = align128(o + (uint32_t)(2 * S + 5) * 8);
    L.tmem = o; o = align128(o + 4);
    L.total = o;
    return L;
}
// mixed product: the connected lists (conn, sgn) in the table area
__host__ __device__ inline TcLayout mixed_layout(int ldA, int nF, int N, bool grow)
{
    return tc_layout(grow ? 0u : (uint32_t)ldA * 4u, nF, N, grow ? kMixKSGrow : kMixKS, kMixStages,
                     2u * kMaxConn * 4u);
}
// intermediate product: K = pairs outside the intermediate, slices of KS rows
// (a multiple of 16), kRiStages A stages and a copy ring of kRiRing slices
// (kRiRing - 1 in flight), placed in the table area after the row offsets
__host__ __device__ inline int ri_n(int K) { return (K + 15) & ~15; }
__host__ __device__ inline int ri_ks(int K) { return K > 32 && K <= 48 ? 48 : 32; }
__host__ __device__ inline uint32_t ri_raw_off() { return align128((uint32_t)kRiMaxU * 8u); }
__host__ __device__ inline TcLayout ri_layout(int K)
{
    const int KS = ri_ks(K);
    return tc_layout(0u, K, ri_n(K), KS, kRiStages,
                     ri_raw_off() + (uint32_t)(kRiRing * KS * kTcM * 4));
}

__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t a)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
// One test of the phase; the thread may sleep in it (up to kTcSuspendNs) until
// the phase completes, so a waiting warp takes no issue slots from the others.
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
                 "selp.b32 %0, 1, 0, P1;\n\t}"
                 : "=r"(ok)
                 : "r"(a), "r"(parity), "n"(kTcSuspendNs)
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
// The flags and the clock are read after each test that came back without the
// phase, i.e. at most once per suspend period.
__device__ bool mbar_wait(uint32_t a, uint32_t parity, volatile int *abort_flag)
{
    if (mbar_try(a, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (long i = 1; i < kTcSpinCap; ++i) {
        if (mbar_try(a, parity)) return true;
        if (*abort_flag) return false;
        if (*(volatile int *)&g_tc_abort) { *abort_flag = 1; return false; }
        if (global_ns() - t0 > kTcWaitNs) break;
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
        if (global_ns() - t0 > kTcWaitNs) break;
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

// B = [N x kp8] K-major, hi and lo parts: bval(j, k) for j < jm and k < K, zero
// elsewhere.
template <int N, typename BVal>
__device__ __forceinline__ void stage_b(const TcLayout &L, unsigned char *smem, int jm, int K, BVal bval)
{
    const int nk4 = L.kp8 / 4;
    // core matrix cm = (row group, K chunk); element e = (row r, k within chunk)
    for (int i = threadIdx.x; i < N * L.kp8; i += kTcThreads) {
        const int cm = i >> 5, e = i & 31;
        const int j = (cm / nk4) * 8 + (e & 7), k = (cm % nk4) * 4 + (e >> 3);
        const float x = (j < jm && k < K) ? bval(j, k) : 0.f;
        float hi, lo;
        tf32_split(x, hi, lo);
        const uint32_t off = kmajor_off(j, k, L.sbo_b);
        *reinterpret_cast<float *>(smem + L.bh + off) = hi;
        *reinterpret_cast<float *>(smem + L.bl + off) = lo;
    }
}

// Barrier initialisation and TMEM allocation; every thread leaves with the
// accumulators' TMEM address (B and any staged row are visible to the MMAs).
template <int N, int S>
__device__ __forceinline__ uint32_t tc_begin(const TcLayout &L, uint32_t sbase, unsigned char *smem,
                                             volatile int *abort_flag)
{
    const uint32_t bar0 = sbase + L.bars;   // afull[S], aempty[S], dfull[2], dempty[2], done
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; ++i) {
            mbar_init(bar0 + 8u * (uint32_t)i, 32 * kTcProdWarps);
            mbar_init(bar0 + 8u * (uint32_t)(S + i), 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(bar0 + 8u * (uint32_t)(2 * S + i), 1);
            mbar_init(bar0 + 8u * (uint32_t)(2 * S + 2 + i), 128);
        }
        mbar_init(bar0 + 8u * (uint32_t)(2 * S + 4), 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if ((threadIdx.x >> 5) == kTcMmaWarp) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + L.tmem),
                     "r"(tmem_cols<N>())
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();   // B (generic-proxy stores) is read by the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    return *reinterpret_cast<volatile uint32_t *>(smem + L.tmem);
}

template <int N>
__device__ __forceinline__ void tc_end(uint32_t tmem)
{
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if ((threadIdx.x >> 5) == kTcMmaWarp)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols<N>())
                     : "memory");
}

// The pipelined product over ncb column chunks of 128 (from z0) and the KS-row
// slices of each: producers fill A slices through src, lane 0 of the MMA warp
// issues the MMAs into the two accumulators, the epilogue warps store D's first
// jm columns to zrow[(c * zrows + j) * 128 + b] (zrow: row j = 0 of chunk 0 of
// this CTA's Z block, zrows: rows per chunk block).
//
// Slice q covers rows (q % nsl) * KS.. and chunk columns (q / nsl) * 128.. from
// z0 and lives in A stage q % S (hi and lo parts, K-major).  Src (one per producer thread) fills the slices: setup(pw, lane) once,
// begin(nq) once, then per slice produce(q, free) (its elements of slice q, rows
// past K zero, split into the stage; free(t) waits until stage t % S may be
// overwritten for slice t and is false when the CTA aborts; produce is false
// then too), and finish() before the producer leaves.
template <int N, int KS, int S, typename Src>
__device__ __forceinline__ void tc_pipeline(const TcLayout &L, unsigned char *smem, uint32_t sbase, uint32_t tmem,
                                            int ncb, int jm, float *zrow, int zrows, Src &src,
                                            volatile int *abort_flag)
{
    static_assert(N % 16 == 0 && N >= 16 && N <= 128, "MMA N for M = 128: a multiple of 16");
    static_assert(KS % 8 == 0, "slices of whole MMA K steps");
    constexpr uint32_t kIdesc = idesc_tf32<N>();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t bar0 = sbase + L.bars;
    auto afull = [&](int i) { return bar0 + 8u * (uint32_t)i; };
    auto aempty = [&](int i) { return bar0 + 8u * (uint32_t)(S + i); };
    auto dfull = [&](int i) { return bar0 + 8u * (uint32_t)(2 * S + i); };
    auto dempty = [&](int i) { return bar0 + 8u * (uint32_t)(2 * S + 2 + i); };
    const uint32_t done = bar0 + 8u * (uint32_t)(2 * S + 4);
    const int nsl = (L.kp8 + KS - 1) / KS;
    const int nq = ncb * nsl;
    // A descriptors: core matrices 8 rows b x 4 k, K chunks 128 bytes apart,
    // 8-row groups KS / 4 chunks apart; one K step of 8 is two chunks
    constexpr uint32_t kLboA = kCoreBytes, kSboA = (KS / 4) * kCoreBytes, kStepA = 2u * kCoreBytes;

    if (warp >= 4 && warp < 4 + kTcProdWarps) {
        // ---- producers ----
        auto free_stage = [&](int t) -> bool {
            return t < S || mbar_wait(aempty(t % S), (uint32_t)(((t / S) - 1) & 1), abort_flag);
        };
        src.setup(warp - 4, lane);
        src.begin(nq);
        for (int q = 0; q < nq; ++q) {
            if (!src.produce(q, free_stage)) break;
            fence_async_smem();
            mbar_arrive(afull(q % S));
        }
        src.finish();
    } else if (warp == kTcMmaWarp) {
        // ---- MMA issue ----
        if (lane == 0) {
            bool ok = true;
            for (int c = 0; c < ncb && ok; ++c) {
                const int dbuf = c & 1;
                if (c >= 2 && !mbar_wait(dempty(dbuf), (uint32_t)(((c >> 1) - 1) & 1), abort_flag)) break;
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)dbuf * N;
                for (int s = 0; s < nsl; ++s) {
                    const int q = c * nsl + s, st = q % S;
                    if (!mbar_wait(afull(st), (uint32_t)((q / S) & 1), abort_flag)) { ok = false; break; }
                    tc_fence_after();
                    const int f0 = s * KS, nks = (min(KS, L.kp8 - f0) + 7) / 8;
                    const uint32_t ah = sbase + L.ah + (uint32_t)st * L.abytes, al = sbase + L.al + (uint32_t)st * L.abytes;
                    for (int ks = 0; ks < nks; ++ks) {
                        const uint32_t aoff = (uint32_t)ks * kStepA;
                        const uint32_t boff = (uint32_t)(f0 / 4 + 2 * ks) * kCoreBytes;
                        const uint64_t dah = umma_desc(ah + aoff, kLboA, kSboA);
                        const uint64_t dal = umma_desc(al + aoff, kLboA, kSboA);
                        const uint64_t dbh = umma_desc(sbase + L.bh + boff, kCoreBytes, L.sbo_b);
                        const uint64_t dbl = umma_desc(sbase + L.bl + boff, kCoreBytes, L.sbo_b);
                        umma_tf32(d, dah, dbh, kIdesc, (s | ks) != 0 ? 1u : 0u);
                        umma_tf32(d, dah, dbl, kIdesc, 1u);
                        umma_tf32(d, dal, dbh, kIdesc, 1u);
                    }
                    umma_commit(aempty(st));   // the stage is free once these MMAs completed
                }
                if (ok) umma_commit(dfull(dbuf));
            }
            umma_commit(done);   // every issued MMA has completed before TMEM is freed
            mbar_wait_drain(done, 0u);
        }
        __syncwarp();
    } else if (warp < 4) {
        // ---- epilogue: D (TMEM lanes 32 warp .. +31 = columns b) -> Z[row][j][b] ----
        for (int c = 0; c < ncb; ++c) {
            const int dbuf = c & 1;
            if (!mbar_wait(dfull(dbuf), (uint32_t)((c >> 1) & 1), abort_flag)) break;
            tc_fence_after();
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)dbuf * N;
            float *zb = zrow + (i64)c * zrows * kTcM + warp * 32 + lane;
            // 16 columns (excitations j) at a time: TMEM -> registers -> Z
            for (int i = 0; i < N / 16 && 16 * i < jm; ++i) {
                float v[16];
                tmem_ld16(taddr + 16u * (uint32_t)i, v);
#pragma unroll
                for (int k = 0; k < 16; ++k)
                    if (16 * i + k < jm) zb[(16 * i + k) * kTcM] = v[k];
            }
            tc_fence_before();
            if (c + 2 < ncb) mbar_arrive(dempty(dbuf));
        }
    }
}

// byte offset of element (column b, slice row k) in an A slice of KS rows
template <int KS>
__device__ __forceinline__ uint32_t a_off(int b, int k)
{
    return (uint32_t)(b >> 3) * (uint32_t)((KS / 4) * kCoreBytes) + (uint32_t)(k >> 2) * kCoreBytes +
           (uint32_t)(b & 7) * 16u + (uint32_t)(k & 3) * 4u;
}
__device__ __forceinline__ void put_split(unsigned char *hi, unsigned char *lo, uint32_t off, float x)
{
    float h, l;
    tf32_split(x, h, l);
    *reinterpret_cast<float *>(hi + off) = h;
    *reinterpret_cast<float *>(lo + off) = l;
}

// AND of a predicate over the 512 producer threads (named barrier 1); also a
// barrier among them.
__device__ __forceinline__ bool producers_all(bool p)
{
    uint32_t r;
    asm volatile("{\n\t.reg .pred pi, po;\n\tsetp.ne.u32 pi, %1, 0;\n\t"
                 "bar.red.and.pred po, 1, %2, pi;\n\tselp.u32 %0, 1, 0, po;\n\t}"
                 : "=r"(r)
                 : "r"(p ? 1u : 0u), "n"(32 * kTcProdWarps)
                 : "memory");
    return r != 0;
}

// X^T[b][F] = sB_F c~[a'][b ^ F] through the gather table (rank(b ^ F) << 1 |
// sign, or -1), from the row staged in shared memory or (GROW) read from
// global memory a slice ahead into registers.  Producer warp pw owns core
// matrices cm = pw + 16 it of every slice: 8 columns b (lanes & 7) x 4 slice
// rows (lanes >> 3), conflict-free stores.
template <int KS, bool GROW>
struct GatherSrc {
    static constexpr int nkc = KS / 4, PI = (kTcM / 8) * nkc / kTcProdWarps;
    static_assert(PI * kTcProdWarps == (kTcM / 8) * nkc, "every producer warp owns the same number of core matrices");
    const int *gidx;
    const float *row;
    int ldG, K, z0, nsl, nq;
    int goff[PI], foff[PI], gp[PI];
    uint32_t soff[PI];
    float gv[GROW ? PI : 1];
    __device__ __forceinline__ void setup(int pw, int lane)
    {
#pragma unroll
        for (int it = 0; it < PI; ++it) {
            const int cm = pw + it * kTcProdWarps;
            const int b = (cm / nkc) * 8 + (lane & 7), k = (cm % nkc) * 4 + (lane >> 3);
            foff[it] = k;
            goff[it] = k * ldG + b;
            soff[it] = a_off<KS>(b, k);
        }
    }
    __device__ __forceinline__ void prefetch(int q)
    {
        const int f0 = (q % nsl) * KS;
        const int *gbase = gidx + (i64)f0 * ldG + z0 + (q / nsl) * kTcM;
#pragma unroll
        for (int it = 0; it < PI; ++it) gp[it] = f0 + foff[it] < K ? __ldg(gbase + goff[it]) : -1;
        if constexpr (GROW) {
#pragma unroll
            for (int it = 0; it < PI; ++it) gv[it] = gp[it] >= 0 ? __ldg(row + (gp[it] >> 1)) : 0.f;
        }
    }
    unsigned char *ah, *al;   // A stages (hi, lo)
    uint32_t abytes;
    __device__ __forceinline__ void begin(int n) { nq = n; if (nq > 0) prefetch(0); }
    template <typename Free>
    __device__ __forceinline__ bool produce(int q, Free &free)
    {
        if (!free(q)) return false;
        unsigned char *hi = ah + (size_t)(q % kMixStages) * abytes, *lo = al + (size_t)(q % kMixStages) * abytes;
#pragma unroll
        for (int it = 0; it < PI; ++it) {
            const int g = gp[it];
            float x;
            if constexpr (GROW) x = gv[it];
            else x = g >= 0 ? row[g >> 1] : 0.f;
            put_split(hi, lo, soff[it], (g & 1) ? -x : x);
        }
        if (q + 1 < nq) prefetch(q + 1);
        return true;
    }
    __device__ __forceinline__ void finish() {}
};

// X^T[b][F] = sB_F c~[a'][b ^ F] from the row staged in shared memory, one
// slice of gather indices prefetched into registers.  A thread's element
// group is (column b, four F rows 4 kc .. 4 kc + 3): a warp reads the gather
// indices of 32 consecutive columns of an F row (coalesced), gathers their
// values from the row (consecutive columns of one F land on few banks), and
// writes each column's four values, split, as one 16-byte K-major core row of
// the hi and of the lo stage.
template <int KS>
struct GatherColSrc {
    static constexpr int QI = KS / 16;   // (column, 4 rows) groups per thread and slice
    static_assert(QI * 16 == KS, "KS a multiple of 16");
    const int *gidx;
    const float *row;         // the source row, shared memory
    unsigned char *ah, *al;   // A stages (hi, lo)
    uint32_t abytes;
    int ldG, K, z0, nsl, nq, p;
    int gp[QI][4];
    __device__ __forceinline__ void setup(int pw, int lane) { p = pw * 32 + lane; }
    __device__ __forceinline__ void prefetch(int q)
    {
        const int f0 = (q % nsl) * KS, cb = z0 + (q / nsl) * kTcM;
#pragma unroll
        for (int i = 0; i < QI; ++i) {
            const int id = p + 32 * kTcProdWarps * i, kc = id >> 7, b = id & 127;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int f = f0 + 4 * kc + e;
                gp[i][e] = f < K ? __ldg(gidx + (i64)f * ldG + cb + b) : -1;
            }
        }
    }
    __device__ __forceinline__ void begin(int n) { nq = n; if (nq > 0) prefetch(0); }
    __device__ __forceinline__ float value(int g) const
    {
        if (g < 0) return 0.f;
        const float x = row[g >> 1];
        return (g & 1) ? -x : x;
    }
    template <typename Free>
    __device__ __forceinline__ bool produce(int q, Free &free)
    {
        if (!free(q)) return false;
        unsigned char *hi = ah + (size_t)(q % kMixStages) * abytes, *lo = al + (size_t)(q % kMixStages) * abytes;
#pragma unroll
        for (int i = 0; i < QI; ++i) {
            const int id = p + 32 * kTcProdWarps * i, kc = id >> 7, b = id & 127;
            float4 h, l;
            tf32_split(value(gp[i][0]), h.x, l.x);
            tf32_split(value(gp[i][1]), h.y, l.y);
            tf32_split(value(gp[i][2]), h.z, l.z);
            tf32_split(value(gp[i][3]), h.w, l.w);
            const uint32_t off = a_off<KS>(b, 4 * kc);
            *reinterpret_cast<float4 *>(hi + off) = h;
            *reinterpret_cast<float4 *>(lo + off) = l;
        }
        if (q + 1 < nq) prefetch(q + 1);
        return true;
    }
    __device__ __forceinline__ void finish() {}
};

// X^T[b][k] = c~[row_k][b]: whole rows of c~ at the element offsets roff[k]
// (shared memory), columns past ld and rows past K read as zero.  The rows of a
// slice are copied with cp.async as they lie (a warp copies one 512-byte row
// segment) into a ring of RS slices, RS - 1 slices ahead; once a slice has
// landed (every producer's copies: a named barrier, which also makes the
// producers agree on going on), warp w reads columns 32 (w % 4) .. + 31 of four
// consecutive rows 4 kc .. 4 kc + 3 (conflict-free 4-byte loads) and writes each
// column's four values, split, as one 16-byte K-major core-matrix row of the hi
// and of the lo stage.
template <int KS, int RS>
struct RowRingSrc {
    static constexpr int QI = KS / 16;   // quads copied and core rows written per thread and slice
    static_assert(QI * 16 == KS, "KS a multiple of 16");
    const float *in;
    const long long *roff;
    unsigned char *ah, *al;   // A stages (hi, lo)
    uint32_t abytes;
    float *raw;               // [RS][KS][128]
    uint32_t raw_s;           // its shared address
    int K, ld, z0, nsl, nq, p;
    __device__ __forceinline__ void setup(int pw, int lane) { p = pw * 32 + lane; }
    __device__ __forceinline__ void issue(int t)
    {
        if (t < nq) {
            const int f0 = (t % nsl) * KS, cb = z0 + (t / nsl) * kTcM;
#pragma unroll
            for (int i = 0; i < QI; ++i) {
                const int id = p + 32 * kTcProdWarps * i, k = id >> 5, c4 = (id & 31) * 4;
                const int r = f0 + k, col = cb + c4;
                const bool ok = r < K && col < ld;
                const void *g = ok ? (const void *)(in + roff[r] + col) : (const void *)in;
                const uint32_t d = raw_s + (uint32_t)(((t % RS) * KS + k) * kTcM + c4) * 4u;
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(g), "r"(ok ? 16 : 0)
                             : "memory");
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");   // one group per slice, empty past the last
    }
    __device__ __forceinline__ void begin(int n)
    {
        nq = n;
#pragma unroll
        for (int t = 0; t < RS - 1; ++t) issue(t);
    }
    template <typename Free>
    __device__ __forceinline__ bool produce(int q, Free &free)
    {
        const bool mine = free(q);
        asm volatile("cp.async.wait_group %0;\n" ::"n"(RS - 2) : "memory");   // this thread's copies of slice q
        if (!producers_all(mine)) return false;                                // everyone's, and all go on
        const float *src = raw + (size_t)(q % RS) * KS * kTcM;
        unsigned char *hi = ah + (size_t)(q % kRiStages) * abytes, *lo = al + (size_t)(q % kRiStages) * abytes;
#pragma unroll
        for (int i = 0; i < QI; ++i) {
            const int id = p + 32 * kTcProdWarps * i, kc = id >> 7, b = id & 127;
            const float *col = src + 4 * kc * kTcM + b;
            float4 h, l;
            tf32_split(col[0], h.x, l.x);
            tf32_split(col[kTcM], h.y, l.y);
            tf32_split(col[2 * kTcM], h.z, l.z);
            tf32_split(col[3 * kTcM], h.w, l.w);
            const uint32_t off = a_off<KS>(b, 4 * kc);
            *reinterpret_cast<float4 *>(hi + off) = h;
            *reinterpret_cast<float4 *>(lo + off) = l;
        }
        issue(q + RS - 1);   // into the slot of slice q - 1, which every producer has read
        return true;
    }
    __device__ __forceinline__ void finish() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
};

template <typename Ti, int N, bool GROW>
__global__ void __launch_bounds__(kTcThreads, 1)
mixed_gemm_tc_kernel(const MixedArgs P, const Ti *__restrict__ astr, const float *__restrict__ ct,
                     float *__restrict__ Z, int z0, int W, int jbase)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const TcLayout L = mixed_layout(P.ldA, P.nF, N, GROW);
    const int K = P.nF;
    float *srow = reinterpret_cast<float *>(smem + L.srow);
    int *conn = reinterpret_cast<int *>(smem + L.tab);
    int *sgn = conn + kMaxConn;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
    __shared__ int wcnt[kTcThreads / 32], cnt;
    __shared__ volatile int abort_flag;
    __shared__ int skip_all;
    const int a = blockIdx.x;
    if (threadIdx.x == 0) skip_all = *(volatile int *)&g_tc_abort;
    __syncthreads();
    if (skip_all) return;   // an earlier CTA gave up a wait: the result is void (counted)
    const int m = connected_excitations<kTcThreads>(P, (u64)astr[a], conn, sgn, wcnt, &cnt);
    const int jm = min(N, m - jbase);
    if (jm <= 0) return;   // uniform across the CTA

    // ---- stage the source row and B = Lam_conn^T (hi and lo) ----
    if (!GROW) {
        const int4 *src = reinterpret_cast<const int4 *>(ct + (i64)a * P.ldA);
        int4 *dst = reinterpret_cast<int4 *>(srow);
        const int n16 = P.ldA / 4;
        for (int i = threadIdx.x; i < n16; i += kTcThreads) dst[i] = __ldg(src + i);
    }
    const float *Lam = static_cast<const float *>(P.Lam);
    stage_b<N>(L, smem, jm, K, [&](int j, int f) {
        return (float)sgn[jbase + j] * Lam[(i64)conn[jbase + j] * K + f];
    });
    const uint32_t tmem = tc_begin<N, kMixStages>(L, sbase, smem, &abort_flag);

    const int zend = min(P.cend, z0 + W);
    const int ncb = (zend - z0 + kTcM - 1) / kTcM;
    float *zrow = zchunk(Z, a, P.M, W, 0) + jbase * kTcM;
    if constexpr (GROW) {
        GatherSrc<kMixKSGrow, true> src;
        src.gidx = P.gidx;
        src.row = ct + (i64)a * P.ldA;
        src.ldG = P.ldG;
        src.K = K;
        src.z0 = z0;
        src.nsl = (L.kp8 + kMixKSGrow - 1) / kMixKSGrow;
        src.ah = smem + L.ah;
        src.al = smem + L.al;
        src.abytes = L.abytes;
        tc_pipeline<N, kMixKSGrow, kMixStages>(L, smem, sbase, tmem, ncb, jm, zrow, P.M, src, &abort_flag);
    } else {
        GatherColSrc<kMixKS> src;
        src.gidx = P.gidx;
        src.row = srow;
        src.ldG = P.ldG;
        src.K = K;
        src.z0 = z0;
        src.nsl = (L.kp8 + kMixKS - 1) / kMixKS;
        src.ah = smem + L.ah;
        src.al = smem + L.al;
        src.abytes = L.abytes;
        tc_pipeline<N, kMixKS, kMixStages>(L, smem, sbase, tmem, ncb, jm, zrow, P.M, src, &abort_flag);
    }
    tc_end<N>(tmem);
}

// One CTA per intermediate m: Z[m][j][b] = sum_k W[pair_j][pair_k] s(m, pair_k)
// c~[m + pair_k][b] for the K pairs outside m.
template <int N, int KS>
__global__ void __launch_bounds__(kTcThreads, 1)
ri_gemm_tc_kernel(const RIArgs P, const float *__restrict__ in, float *__restrict__ Z, int z0, int W)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    const int K = P.nU;
    const TcLayout L = ri_layout(K);
    long long *roff = reinterpret_cast<long long *>(smem + L.tab);
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
    __shared__ volatile int abort_flag;
    __shared__ int skip_all;
    const int m = blockIdx.x;
    if (threadIdx.x == 0) skip_all = *(volatile int *)&g_tc_abort;
    __syncthreads();
    if (skip_all) return;   // an earlier CTA gave up a wait: the result is void (counted)
    const int *srcm = P.src + (i64)m * K, *pidm = P.pid + (i64)m * K;
    for (int i = threadIdx.x; i < K; i += kTcThreads) roff[i] = (long long)(__ldg(srcm + i) >> 1) * P.ld_in;
    const float *Wt = static_cast<const float *>(P.W);
    stage_b<N>(L, smem, K, K, [&](int j, int k) {
        const float w = Wt[(i64)__ldg(pidm + j) * P.nP + __ldg(pidm + k)];
        return (__ldg(srcm + k) & 1) ? -w : w;
    });
    const uint32_t tmem = tc_begin<N, kRiStages>(L, sbase, smem, &abort_flag);   // its barrier also publishes roff

    const int zend = min(P.cend, z0 + W);
    const int ncb = (zend - z0 + kTcM - 1) / kTcM;
    RowRingSrc<KS, kRiRing> src;
    src.in = in;
    src.roff = roff;
    src.ah = smem + L.ah;
    src.al = smem + L.al;
    src.abytes = L.abytes;
    src.raw = reinterpret_cast<float *>(smem + L.tab + ri_raw_off());
    src.raw_s = sbase + L.tab + ri_raw_off();
    src.K = K;
    src.ld = P.ld_in;
    src.z0 = z0;
    src.nsl = (L.kp8 + KS - 1) / KS;
    tc_pipeline<N, KS, kRiStages>(L, smem, sbase, tmem, ncb, K, zchunk(Z, m, K, W, 0), K, src, &abort_flag);
    tc_end<N>(tmem);
}

}  // namespace

// shared memory of a CTA: the dynamic layout plus the kernels' static part
// (1 KB with the dynamic base aligned to 1 KB)
constexpr size_t kTcStaticSmem = 1024;
size_t mixed_tc_smem(int ldA, int nF, int N, bool grow) { return mixed_layout(ldA, nF, N, grow).total + kTcStaticSmem; }

template <typename Ti>
int mixed_gemm_tc(const MixedArgs &ma, const Ti *astr, const float *ct, float *Z, int z0, int W, int jbase, int N,
                  bool grow, cudaStream_t s)
{
    const size_t smem = mixed_layout(ma.ldA, ma.nF, N, grow).total;
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

bool ri_tc_supported(int nU) { return nU >= 1 && nU <= kRiMaxU && ri_n(nU) <= 80; }
size_t ri_tc_smem(int nU) { return ri_layout(nU).total + kTcStaticSmem; }

int ri_gemm_tc(const RIArgs &ra, const float *in, float *Z, int z0, int W, cudaStream_t s)
{
    if (!ri_tc_supported(ra.nU)) {
        set_error("tensor-core intermediate GEMM: %d pairs outside an intermediate", ra.nU);
        return BSIM_ERR_UNSUPPORTED;
    }
    const size_t smem = ri_layout(ra.nU).total;
    auto launch = [&](auto kern) -> int {
        BSIM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<ra.nM, kTcThreads, smem, s>>>(ra, in, Z, z0, W);
        BSIM_CUDA(cudaGetLastError());
        return BSIM_OK;
    };
    switch (ri_n(ra.nU)) {
    case 16: return launch(ri_gemm_tc_kernel<16, 32>);
    case 32: return launch(ri_gemm_tc_kernel<32, 32>);
    case 48: return launch(ri_gemm_tc_kernel<48, 48>);
    case 64: return launch(ri_gemm_tc_kernel<64, 32>);
    default: return launch(ri_gemm_tc_kernel<80, 32>);
    }
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
