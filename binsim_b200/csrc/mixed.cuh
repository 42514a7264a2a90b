// Shared pieces of the structured sigma's GEMM kernels, the mixed-excitation and
// the intermediate-string products (sigma_fast.cu: CUDA-core and DMMA paths;
// sigma_tc.cu: the tcgen05 paths).
#pragma once
#include "fastplan.h"

namespace bsim {

struct MixedArgs {
    int nA, nB, nE, nF, M, ldA, ldG;
    int cend;               // end of the column range being computed (nB for a whole sigma)
    const u64 *Emask, *mA;
    const void *Lam;        // T [nE x nF]
    const int *gidx;        // [nF x ldG]: (rank(b^F) << 1 | sign) or -1
};

// Layout of the GEMM outputs Z (a window of W columns, W a multiple of 128):
// for output row group r (a source row, or an intermediate string) of R rows,
// chunk c of 128 columns is one contiguous [R][128] block, so a chunk's output
// is written as one piece.  zchunk gives the block of (r, c).
template <typename T>
__host__ __device__ __forceinline__ T *zchunk(T *Z, int r, int R, int W, int c)
{
    return Z + (i64)r * R * W + (i64)c * R * kMixCols;
}

struct RIArgs {
    int nM, nU, npr, nP, ld_in, cend;
    const int *src, *pid;
    const void *W;          // T [nP x nP]
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
            if (j < kMaxConn) { conn[j] = e; sgn[j] = (__popcll(sa & P.mA[e]) & 1) ? -1 : 1; }
        }
        __syncthreads();
        if (threadIdx.x == 0) for (int w2 = 0; w2 < NW; ++w2) *cnt += wcnt[w2];
        __syncthreads();
    }
    return min(*cnt, kMaxConn);
}

// FP32-bulk mixed GEMM on the tensor cores (sigma_tc.cu): one launch of one
// pass of N excitations (from jbase) over the Z window [z0, z0 + W), N = 64 with
// the source row on chip or read from global memory (grow), or N = 80 with
// grow; the shared memory a shape needs; count of bounded waits that gave up
// (0 in normal operation).
size_t mixed_tc_smem(int ldA, int nF, int N, bool grow);
template <typename Ti>
int mixed_gemm_tc(const MixedArgs &ma, const Ti *astr, const float *ct, float *Z, int z0, int W, int jbase, int N,
                  bool grow, cudaStream_t s);
// FP32-bulk intermediate-string GEMM on the tensor cores: whether a side with
// nU pairs outside an intermediate has a kernel, the shared memory it needs, one
// launch over the Z window [z0, z0 + W).
bool ri_tc_supported(int nU);
size_t ri_tc_smem(int nU);
int ri_gemm_tc(const RIArgs &ra, const float *in, float *Z, int z0, int W, cudaStream_t s);
int mixed_tc_timeouts(int *count, bool reset);

}  // namespace bsim
