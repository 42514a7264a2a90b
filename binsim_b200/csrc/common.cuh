// Internal header of libcuotf: status codes, device data layout, small device helpers.
//
// Layout in HBM (one symmetry block shown; blocks are concatenated):
//   determinant (a, b) of block k lives at  off[k] + a * nb[k] + b   (alpha-major,
//   reference basis/basis.hpp:327), so a beta string index is the fastest-moving
//   one and a warp whose lanes take consecutive b reads/writes coalesced lines.
//   Strings: per block, alpha then beta lists in Gosper (ascending) order.
//   Groups: AoS table `GroupDev` in the network's ORIGINAL order; Z masks and
//   weights in two flat arrays (`z`, `w`) addressed by per-group offsets.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <vector>
#include <string>

namespace bsim {

using i64 = long long;
using u64 = unsigned long long;

// ---- status codes returned by every v2 entry point --------------------------
enum Status : int {
    BSIM_OK = 0,
    BSIM_ERR_NULL = -1,        // a required handle / pointer is null
    BSIM_ERR_ARG = -2,         // an argument is out of range
    BSIM_ERR_UNSUPPORTED = -3, // configuration not supported (e.g. norb too large)
    BSIM_ERR_ALLOC = -4,       // device allocation failed
    BSIM_ERR_TIMEOUT = -5,     // a bounded device wait gave up
    BSIM_ERR_CUDA = -6,        // a CUDA runtime call failed (see bsim_last_error)
    BSIM_ERR_TOO_LARGE = -7,   // request exceeds a fixed capacity
};

void set_error(const char *fmt, ...);
const char *last_error();
int cuda_status(cudaError_t e, const char *what);

// Every device allocation of the library goes through dmalloc / dmalloc_async,
// which count the calls; bsim_device_alloc_count() returns the count, so a
// caller can check that a stretch of calls allocated nothing.
void note_device_alloc();
long long device_alloc_count();
cudaError_t trim_library_pool();   // hand the pool's unused memory back to the device
template <typename T>
inline cudaError_t dmalloc(T **p, size_t bytes)
{
    note_device_alloc();
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), bytes);
    if (e == cudaErrorMemoryAllocation) {   // memory the library's pool keeps may be what is missing
        (void)cudaGetLastError();
        if (trim_library_pool() == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(p), bytes);
    }
    return e;
}
// Stream-ordered allocations come from the library's own pool on the current
// device, whose release threshold keeps freed memory for the next allocation:
// a solver that allocates its vectors on every call then pays the mapping of
// that memory once per process, not once per call.
cudaError_t library_pool(cudaMemPool_t *pool);
template <typename T>
inline cudaError_t dmalloc_async(T **p, size_t bytes, cudaStream_t s)
{
    note_device_alloc();
    cudaMemPool_t pool;
    const cudaError_t e = library_pool(&pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(reinterpret_cast<void **>(p), bytes, pool, s);
}

#define BSIM_CUDA(call)                                              \
    do {                                                             \
        cudaError_t e__ = (call);                                    \
        if (e__ != cudaSuccess) return ::bsim::cuda_status(e__, #call); \
    } while (0)

// ---- device views -----------------------------------------------------------
constexpr int kMaxRank = 64;      // ranks above this are rejected at network build
constexpr int kMaxIrreps = 16;

template <typename Ti>
struct BasisView {
    int num_blocks, num_irreps, norb;
    i64 dim;
    const int *blk_asym, *blk_bsym, *blk_na, *blk_nb, *blk_astart, *blk_bstart;
    const i64 *blk_off;
    const Ti *astrs, *bstrs;   // per-block string lists (alpha, beta)
    const int *amap, *bmap;    // string -> index in its irrep list, or -1: indexed by the
                               // string itself (dense) or by its colex rank (rank_maps)
    const int *block_map;      // [num_irreps^2] -> block or -1
    int nel_a, nel_b, rank_maps;
    const long long *binom;    // [65 x 65] binomials for the colex rank (rank_maps)
};

// Index of string s in its irrep's list (or -1 when s is not a string of the
// basis).  Dense tables up to 2^26 entries; above that, the colex rank of s
// among all strings with its electron count (Gosper order is colex order)
// indexes a table of C(norb, n) entries.
template <typename Ti>
__device__ __forceinline__ int string_index(const BasisView<Ti> &B, const int *map, int nel, Ti s)
{
    const unsigned long long x = (unsigned long long)s;
    if (B.norb < 64 && (x >> B.norb)) return -1;
    if (!B.rank_maps) return map[x];
    if (__popcll(x) != nel) return -1;
    long long r = 0;
    int i = 1;
    for (unsigned long long y = x; y; y &= y - 1, ++i) r += B.binom[(__ffsll((long long)y) - 1) * 65 + i];
    return map[r];
}

// One group of the OTF network (reference ham/otf.hpp:67-112).
struct GroupDev {
    u64 ax, bx;
    int rank, nza, nzb, type;   // type: 0 diag, 1 pure alpha, 2 pure beta, 3 mixed
    int asym, bsym, orig, pad;
    i64 za_off, zb_off, wa_off, wb_off;  // into z[] and w[] (w col-major [nz x rank])
};

template <typename Ti>
struct NetView {
    int ngs;
    const GroupDev *g;    // original order
    const Ti *z;          // all za then zb masks
    const double *w;      // all weights
    const float *w32;     // fp32 copy of w (mixed-precision sigma)
};

// ---- device helpers ---------------------------------------------------------
__device__ __forceinline__ int par(unsigned int x) { return __popc(x) & 1; }
__device__ __forceinline__ int par(unsigned long long x) { return __popcll(x) & 1; }

// P_r(s) = sum_k (-1)^{popc(s & z_k)} w[r*nz + k]  (reference core/math.hpp:37-78)
template <typename Ti, typename Tw>
__device__ __forceinline__ void phase_vec(Ti s, const Ti *__restrict__ z, int nz,
                                          const Tw *__restrict__ w, int rank, Tw *out)
{
    for (int r = 0; r < rank; ++r) out[r] = Tw(0);
    for (int k = 0; k < nz; ++k) {
        const bool odd = par(s & z[k]);
        for (int r = 0; r < rank; ++r) {
            const Tw v = w[(i64)r * nz + k];
            out[r] += odd ? -v : v;
        }
    }
}

template <typename Ti, typename Tw>
__device__ __forceinline__ Tw phase1(Ti s, const Ti *__restrict__ z, int nz, const Tw *__restrict__ w)
{
    Tw v = Tw(0);
    for (int k = 0; k < nz; ++k) v += par(s & z[k]) ? -w[k] : w[k];
    return v;
}

// Index of (string ^ mask) in its irrep list, or -1 if it is not a string of
// the basis.  Same-length strings map through the dense table.
template <typename Ti>
__device__ __forceinline__ int str_index(const int *__restrict__ map, Ti s) { return map[s]; }

// block-wide sum of a double, result valid in thread 0
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh /*[32]*/)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = (lane < NT / 32) ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

}  // namespace bsim
