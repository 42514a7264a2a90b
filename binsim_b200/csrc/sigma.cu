// sigma = H c over the OTF network (reference op/hvec.hpp:481-496 and
// cuda/hvec.cuh:432-446), and diag(H) (reference op/hvec.hpp:498-554).
//
// One launch covers every group, so each destination element is written once
// (no memset, no atomics): a CTA keeps its 32 x 32 tile of sigma in registers
// (4 rows x 1 column per thread) across all chunks of groups.
//
// FP32-bulk variant: phases, weights and the gathered source are FP32 and a
// chunk's products are summed in FP32; the per-chunk partial is added into an
// FP64 accumulator, so rounding is bounded per chunk (<= 64 terms) while the
// long sum over all chunks stays FP64.
#include "ops.h"
#include "tiles.cuh"

#include <cstdlib>

namespace bsim {

template <typename Ti, bool MIXED>
__global__ void __launch_bounds__(kTileThreads)
sigma_tile_kernel(const BasisView<Ti> B, const NetView<Ti> N, const int *__restrict__ plan_g,
                  const int4 *__restrict__ chunks, int nchunks, const i64 *__restrict__ tile_start,
                  const double *__restrict__ src, const float *__restrict__ src32, double *__restrict__ dst,
                  i64 tile_lo, int accumulate)
{
    using Tw = typename std::conditional<MIXED, float, double>::type;
    __shared__ TileSmem<Tw> S;
    const TileCoord c = decode_tile(B, tile_start, tile_lo + blockIdx.x);
    const int lane = threadIdx.x & 31, wrow = (threadIdx.x >> 5) * kRowsPerWarp;
    double acc[kRowsPerWarp] = {0.0, 0.0, 0.0, 0.0};

    for (int ci = 0; ci < nchunks; ++ci) {
        const int4 ch = chunks[ci];
        const int G = ch.y, R = ch.z;
        __syncthreads();
        fill_chunk<Ti, Tw, false>(B, N, plan_g, ch.x, G, R, c, S, nullptr);
        __syncthreads();
        Tw part[kRowsPerWarp] = {Tw(0), Tw(0), Tw(0), Tw(0)};
        for (int gl = 0; gl < G; ++gl) {
            const int sc = S.col[gl][lane];
            if (sc < 0) continue;
#pragma unroll
            for (int i = 0; i < kRowsPerWarp; ++i) {
                const i64 row = S.row[gl][wrow + i];
                if (row < 0) continue;
                Tw v;
                if (R == 1) {
                    v = S.pa[gl][wrow + i] * S.pb[gl][lane];
                } else if (R == 2) {
                    v = S.pa[2 * gl][wrow + i] * S.pb[2 * gl][lane] +
                        S.pa[2 * gl + 1][wrow + i] * S.pb[2 * gl + 1][lane];
                } else {
                    v = Tw(0);
                    for (int r = 0; r < R; ++r) v += S.pa[gl * R + r][wrow + i] * S.pb[gl * R + r][lane];
                }
                if constexpr (MIXED) part[i] += v * __ldg(src32 + row + sc);
                else part[i] += v * __ldg(src + row + sc);
            }
        }
#pragma unroll
        for (int i = 0; i < kRowsPerWarp; ++i) acc[i] += (double)part[i];
    }
    const int b = c.tb * kTile + lane;
    if (b < c.nb) {
        const i64 base = B.blk_off[c.k];
#pragma unroll
        for (int i = 0; i < kRowsPerWarp; ++i) {
            const int a = c.ta * kTile + wrow + i;
            if (a < c.na) {
                const i64 di = base + (i64)a * c.nb + b;
                dst[di] = accumulate ? dst[di] + acc[i] : acc[i];
            }
        }
    }
}

// diag(H) += D, D(a,b) = sum_r PA_r(a) PB_r(b) for the first diagonal group.
template <typename Ti>
__global__ void __launch_bounds__(kTileThreads)
diag_tile_kernel(const BasisView<Ti> B, const NetView<Ti> N, int gid, const i64 *__restrict__ tile_start,
                 double *__restrict__ diag)
{
    __shared__ double pa[kMaxRank][kTile];
    __shared__ double pb[kMaxRank][kTile];
    const TileCoord c = decode_tile(B, tile_start, blockIdx.x);
    const GroupDev gd = N.g[gid];
    const int R = gd.rank;
    for (int t = threadIdx.x; t < 2 * kTile; t += blockDim.x) {
        const int j = t & 31;
        const bool isrow = t >= kTile;
        const int idx = (isrow ? c.ta : c.tb) * kTile + j;
        const int lim = isrow ? c.na : c.nb;
        if (idx >= lim) continue;
        const Ti s = isrow ? B.astrs[B.blk_astart[c.k] + idx] : B.bstrs[B.blk_bstart[c.k] + idx];
        const Ti *z = N.z + (isrow ? gd.za_off : gd.zb_off);
        const double *w = N.w + (isrow ? gd.wa_off : gd.wb_off);
        const int nz = isrow ? gd.nza : gd.nzb;
        for (int r = 0; r < R; ++r) {
            double v = 0.0;
            for (int q = 0; q < nz; ++q) v += par(s & z[q]) ? -w[(i64)r * nz + q] : w[(i64)r * nz + q];
            (isrow ? pa : pb)[r][j] = v;
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, wrow = (threadIdx.x >> 5) * kRowsPerWarp;
    const int b = c.tb * kTile + lane;
    if (b >= c.nb) return;
    for (int i = 0; i < kRowsPerWarp; ++i) {
        const int a = c.ta * kTile + wrow + i;
        if (a >= c.na) continue;
        double v = 0.0;
        for (int r = 0; r < R; ++r) v += pa[r][wrow + i] * pb[r][lane];
        diag[B.blk_off[c.k] + (i64)a * c.nb + b] += v;
    }
}

__global__ void to_f32_kernel(const double *__restrict__ x, float *__restrict__ y, i64 n)
{
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        y[i] = (float)x[i];
}

// ---- host launchers -------------------------------------------------------------
template <typename Ti>
int tile_prefix(const DevBasis<Ti> *B, Workspace &ws, const i64 **out_dev, i64 *ntiles)
{
    std::vector<i64> pref(B->num_blocks + 1, 0);
    for (int k = 0; k < B->num_blocks; ++k) {
        const i64 ta = (B->na[k] + kTile - 1) / kTile, tb = (B->nb[k] + kTile - 1) / kTile;
        pref[k + 1] = pref[k] + ta * tb;
    }
    *ntiles = pref[B->num_blocks];
    return ws.tile_table(pref, out_dev);
}

template <typename Ti>
i64 num_tiles(const DevBasis<Ti> *B)
{
    i64 t = 0;
    for (int k = 0; k < B->num_blocks; ++k)
        t += (i64)((B->na[k] + kTile - 1) / kTile) * ((B->nb[k] + kTile - 1) / kTile);
    return t;
}

template <typename Ti>
int sigma_tiles(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *src, const float *src32, double *dst,
                bool mixed, i64 tile_lo, i64 tile_hi, cudaStream_t s)
{
    if (B->dim == 0) return BSIM_OK;
    Workspace &ws = workspace_for(B);
    const i64 *tp = nullptr;
    i64 ntiles = 0;
    int st = tile_prefix(B, ws, &tp, &ntiles);
    if (st != BSIM_OK) return st;
    if (tile_lo < 0 || tile_hi > ntiles || tile_lo > tile_hi) {
        set_error("tile range [%lld, %lld) outside [0, %lld)", tile_lo, tile_hi, ntiles);
        return BSIM_ERR_ARG;
    }
    const i64 nt = tile_hi - tile_lo;
    if (nt == 0) return BSIM_OK;
    if (nt > 0x7fffffffLL) { set_error("too many tiles"); return BSIM_ERR_TOO_LARGE; }
    if (N->plan_chunks.empty()) {
        if (tile_lo == 0 && tile_hi == ntiles) BSIM_CUDA(cudaMemsetAsync(dst, 0, sizeof(double) * B->dim, s));
        else { set_error("empty network with a partial tile range"); return BSIM_ERR_ARG; }
        return BSIM_OK;
    }
    if (mixed && !src32) {
        float *tmp = nullptr;
        st = ws.f32_buffer(B->dim, &tmp);
        if (st != BSIM_OK) return st;
        to_f32_kernel<<<1184, 256, 0, s>>>(src, tmp, B->dim);
        src32 = tmp;
    }
    if (mixed)
        sigma_tile_kernel<Ti, true><<<(unsigned)nt, kTileThreads, 0, s>>>(
            B->view, N->view, N->d_plan_groups, N->d_plan_chunks, (int)N->plan_chunks.size(), tp, nullptr, src32, dst,
            tile_lo, 0);
    else
        sigma_tile_kernel<Ti, false><<<(unsigned)nt, kTileThreads, 0, s>>>(
            B->view, N->view, N->d_plan_groups, N->d_plan_chunks, (int)N->plan_chunks.size(), tp, src, nullptr, dst,
            tile_lo, 0);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename Ti>
int sigma_generic_accumulate(const DevBasis<Ti> *B, const DevNet<Ti> *N, const int *plan_g, const int4 *chunks,
                             int nchunks, const double *src, const float *src32, double *dst, bool mixed,
                             cudaStream_t s)
{
    if (nchunks == 0 || B->dim == 0) return BSIM_OK;
    Workspace &ws = workspace_for(B);
    const i64 *tp = nullptr;
    i64 ntiles = 0;
    int st = tile_prefix(B, ws, &tp, &ntiles);
    if (st != BSIM_OK) return st;
    if (mixed && !src32) {
        float *tmp = nullptr;
        st = ws.f32_buffer(B->dim, &tmp);
        if (st != BSIM_OK) return st;
        to_f32_kernel<<<1184, 256, 0, s>>>(src, tmp, B->dim);
        src32 = tmp;
    }
    if (mixed)
        sigma_tile_kernel<Ti, true><<<(unsigned)ntiles, kTileThreads, 0, s>>>(B->view, N->view, plan_g, chunks,
                                                                             nchunks, tp, nullptr, src32, dst, 0, 1);
    else
        sigma_tile_kernel<Ti, false><<<(unsigned)ntiles, kTileThreads, 0, s>>>(B->view, N->view, plan_g, chunks,
                                                                              nchunks, tp, src, nullptr, dst, 0, 1);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

// Structured path when the plan accepts the (basis, network) pair, else the
// generic tile kernel.  BSIM_SIGMA_GENERIC=1 forces the generic kernel.
template <typename Ti>
int sigma(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *src, const float *src32, double *dst,
          bool mixed, cudaStream_t s)
{
    static const bool force_generic = [] {
        const char *e = getenv("BSIM_SIGMA_GENERIC");
        return e && e[0] == '1';
    }();
    if (!force_generic && B->dim > 0) {
        bool used = false;
        int st = sigma_fast(B, N, src, src32, dst, mixed, s, &used);
        if (st != BSIM_OK) return st;
        if (used) return BSIM_OK;
    }
    return sigma_tiles(B, N, src, src32, dst, mixed, 0, num_tiles(B), s);
}

template <typename Ti>
int diag_elements(const DevBasis<Ti> *B, const DevNet<Ti> *N, double *diag, cudaStream_t s)
{
    if (N->diag_group < 0 || B->dim == 0) return BSIM_OK;
    Workspace &ws = workspace_for(B);
    const i64 *tp = nullptr;
    i64 ntiles = 0;
    int st = tile_prefix(B, ws, &tp, &ntiles);
    if (st != BSIM_OK) return st;
    diag_tile_kernel<Ti><<<(unsigned)ntiles, kTileThreads, 0, s>>>(B->view, N->view, N->diag_group, tp, diag);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template int tile_prefix<unsigned>(const DevBasis<unsigned> *, Workspace &, const i64 **, i64 *);
template int sigma<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, const double *, const float *,
                             double *, bool, cudaStream_t);
template int sigma_tiles<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, const double *,
                                   const float *, double *, bool, i64, i64, cudaStream_t);
template i64 num_tiles<unsigned>(const DevBasis<unsigned> *);
template int sigma_generic_accumulate<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, const int *,
                                                const int4 *, int, const double *, const float *, double *, bool,
                                                cudaStream_t);
template int diag_elements<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, double *, cudaStream_t);
template int tile_prefix<unsigned long long>(const DevBasis<unsigned long long> *, Workspace &, const i64 **, i64 *);
template int sigma<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, const double *, const float *,
                             double *, bool, cudaStream_t);
template int sigma_tiles<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, const double *,
                                   const float *, double *, bool, i64, i64, cudaStream_t);
template i64 num_tiles<unsigned long long>(const DevBasis<unsigned long long> *);
template int sigma_generic_accumulate<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, const int *,
                                                const int4 *, int, const double *, const float *, double *, bool,
                                                cudaStream_t);
template int diag_elements<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, double *, cudaStream_t);

}  // namespace bsim
