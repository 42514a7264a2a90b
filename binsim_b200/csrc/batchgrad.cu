// Pool gradient: grads[orig] = <l| G_g e^{theta_g G_g} |r> (reference orientation)
// for every group g of a pool network at its own angle thetas[orig]
// (reference op/batchgrad.hpp:529-540, cuda/batchgrad.cuh:362-378).
// ADAPT-VQE screening calls it with theta = 0, l = psi, r = H psi.
//
// Same 32 x 32 tiles as sigma with the unordered-pair rule.  Grid
// (splits, chunks): a CTA owns one chunk of <= 32 groups and walks a strided
// subset of the tiles, reducing each group's contribution warp-wise into a
// shared-memory accumulator; at the end one global atomicAdd per (CTA, group).
// Diagonal groups contribute zero for real vectors and are skipped.
#include "ops.h"
#include "tiles.cuh"

namespace bsim {

template <typename Ti>
__global__ void __launch_bounds__(kTileThreads)
batchgrad_tile_kernel(const BasisView<Ti> B, const NetView<Ti> N, const int *__restrict__ plan_g,
                      const int4 *__restrict__ chunks, const i64 *__restrict__ tile_start, i64 ntiles,
                      const double *__restrict__ thetas, const double *__restrict__ l, const double *__restrict__ r,
                      double *__restrict__ grads, const unsigned char *__restrict__ skip, const int *__restrict__ flag)
{
    __shared__ TileSmem<double> S;
    __shared__ double sacc[kTile];
    __shared__ double scd[kTile], sco[kTile];
    __shared__ int stype[kTile];
    const int4 ch = chunks[blockIdx.y];
    const int G = ch.y, R = ch.z;
    const bool route = skip && flag && *flag != 0;
    for (int t = threadIdx.x; t < G; t += blockDim.x) {
        const GroupDev gd = N.g[plan_g[ch.x + t]];
        const double th = thetas[gd.orig];
        sacc[t] = 0.0;
        scd[t] = -sin(th);
        sco[t] = cos(th);
        // type 0 is skipped: diagonal groups, and groups the theta = 0 density route gives
        stype[t] = (route && skip[gd.orig]) ? 0 : gd.type;
    }
    const int lane = threadIdx.x & 31, wrow = (threadIdx.x >> 5) * kRowsPerWarp;
    for (i64 t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const TileCoord c = decode_tile(B, tile_start, t);
        __syncthreads();
        fill_chunk<Ti, double, true>(B, N, plan_g, ch.x, G, R, c, S, nullptr);
        __syncthreads();
        const i64 dbase = B.blk_off[c.k] + (i64)(c.ta * kTile + wrow) * c.nb + c.tb * kTile + lane;
        for (int gl = 0; gl < G; ++gl) {
            if (stype[gl] == 0) continue;
            const int sc = S.col[gl][lane];
            double acc = 0.0;
            if (sc >= 0) {
                for (int i = 0; i < kRowsPerWarp; ++i) {
                    const i64 row = S.row[gl][wrow + i];
                    if (row < 0) continue;
                    double vt = 0.0;
                    for (int q = 0; q < R; ++q) vt += S.pa[gl * R + q][wrow + i] * S.pb[gl * R + q][lane];
                    const i64 si = row + sc, di = dbase + (i64)i * c.nb;
                    const double vd = scd[gl] * (vt * vt), vo = sco[gl] * vt;
                    const double rvi = r[si], rvj = r[di];
                    acc += l[si] * (rvi * vd + rvj * vo) + l[di] * (rvj * vd - rvi * vo);
                }
            }
            acc = warp_sum(acc);
            if (lane == 0 && acc != 0.0) atomicAdd(&sacc[gl], acc);
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < G; t += blockDim.x)
        if (stype[t] != 0) atomicAdd(&grads[N.g[plan_g[ch.x + t]].orig], sacc[t]);
}

template <typename Ti>
int batchgrad(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *thetas, const double *l, const double *r,
              double *grads, cudaStream_t s)
{
    if (N->ngs == 0) return BSIM_OK;
    // ADAPT screening (every theta zero): the groups of the planned forms go
    // through the transition densities; whether every theta is zero is decided
    // on the device, so the call stays asynchronous
    DensityRoute *D = nullptr;
    int st = B->dim > 0 ? density_route(B, N, &D) : BSIM_OK;
    if (st != BSIM_OK) return st;
    const unsigned char *skip = nullptr;
    const int *flag = nullptr;
    if (D) {
        if ((st = density_route_begin(D, thetas, s)) != BSIM_OK) return st;
        skip = density_route_skip(D);
        flag = density_route_flag(D);
    }
    auto finish = [&]() { return D ? density_route_finish<Ti>(D, l, r, grads, s) : BSIM_OK; };
    if (B->dim > 0) {   // single-block bases: one launch over the groups' pair lists
        bool used = false;
        int st0 = pair_list_batchgrad(B, N, thetas, l, r, grads, s, &used, skip, flag);
        if (st0 != BSIM_OK) return st0;
        if (used) return finish();
    }
    BSIM_CUDA(cudaMemsetAsync(grads, 0, sizeof(double) * N->ngs, s));
    if (B->dim == 0 || N->plan_chunks.empty()) return finish();
    Workspace &ws = workspace_for(B);
    const i64 *tp = nullptr;
    i64 ntiles = 0;
    st = tile_prefix(B, ws, &tp, &ntiles);
    if (st != BSIM_OK) return st;
    const int nch = (int)N->plan_chunks.size();
    if (nch > 65535) { set_error("too many group chunks (%d)", nch); return BSIM_ERR_TOO_LARGE; }
    i64 splits = std::max<i64>(1, std::min<i64>(ntiles, (148 * 16 + nch - 1) / nch));
    dim3 grid((unsigned)splits, (unsigned)nch);
    batchgrad_tile_kernel<Ti><<<grid, kTileThreads, 0, s>>>(B->view, N->view, N->d_plan_groups, N->d_plan_chunks, tp,
                                                           ntiles, thetas, l, r, grads, skip, flag);
    BSIM_CUDA(cudaGetLastError());
    return finish();
}

template int batchgrad<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, const double *, const double *,
                                 const double *, double *, cudaStream_t);
template int batchgrad<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, const double *, const double *,
                                 const double *, double *, cudaStream_t);

}  // namespace bsim
