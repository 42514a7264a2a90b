// Single-generator pair operators: expm, grad, backgrad
// (reference op/expm.hpp:374-438, op/grad.hpp:397-465, op/backgrad.hpp:406-474,
//  update rules core/math.hpp:132-215; GPU counterparts cuda/expm.cuh,
//  cuda/grad.cuh, cuda/backgrad.cuh), and the operators the reference has on
// the CPU only: tvec (op/tvec.hpp), backtran (op/backtran.hpp), batchexpm
// (op/batchexpm.hpp) and the per-group transition <l|T|r> of batchtran
// (op/batchtran.hpp), with the update rules of core/math.hpp:165-252.
//
// Launch shape: one CTA per destination alpha row of every block
// (grid = max_na x num_blocks).  A CTA whose row is connected to a source row
// (and passes the once-per-pair rule) walks the row's beta columns with lanes
// on consecutive columns: the destination row segment is read and written
// coalesced, the source side is the row a^ax at columns idx(b^bx).  Every
// unordered pair is owned by exactly one thread, so the in-place updates need
// no atomics.
//
// grad/backgrad reduce deterministically: each CTA writes its partial sum to a
// scratch slot, and the last CTA to finish (atomic ticket) adds all slots in
// index order and writes the result.
#include "ops.h"

namespace bsim {

constexpr int kPairThreads = 256;
constexpr int kExpm = kPairExpm, kGrad = kPairGrad, kBackgrad = kPairBackgrad;

// third vector (backtran's b) and the matrix shape of batchexpm
struct PairExtra {
    double *b;
    int ld, nv;
};
// operators that act on diagonal groups too (the others skip them: real vectors)
__host__ __device__ constexpr bool pair_diag_op(int op) { return op == kPairTvec || op == kPairBacktran || op == kPairTran; }
// operators with a scalar result (deterministic last-CTA reduction)
__host__ __device__ constexpr bool pair_reduces(int op) { return op == kPairGrad || op == kPairBackgrad || op == kPairTran; }

// Ticket counters for the last-CTA reduction live with the partials: the
// scratch buffer holds [nslots partials][1 counter as unsigned long long].
template <typename Ti, int OP>
__global__ void __launch_bounds__(kPairThreads)
pair_row_kernel(const BasisView<Ti> B, const NetView<Ti> N, int gid, PairAngles ang, double *__restrict__ l,
                double *__restrict__ r, double *__restrict__ partials, unsigned long long *__restrict__ ticket,
                double *__restrict__ out, int accumulate, PairExtra X)
{
    __shared__ double spa[kMaxRank];
    __shared__ double red[32];
    __shared__ bool last;
    const int kd = blockIdx.y, a = blockIdx.x;
    const GroupDev g = N.g[gid];
    const int nirr = B.num_irreps;
    bool active = (g.type != 0 || pair_diag_op(OP)) && a < B.blk_na[kd];
    int ks = -1, sa = -1;
    Ti s_a = 0;
    if (active) {
        const int as = B.blk_asym[kd] ^ g.asym, bs = B.blk_bsym[kd] ^ g.bsym;
        ks = (as < nirr && bs < nirr) ? B.block_map[as * nirr + bs] : -1;
        active = ks >= kd;   // ks == -1 fails too
    }
    if (active) {
        s_a = B.astrs[B.blk_astart[kd] + a] ^ (Ti)g.ax;
        sa = g.ax ? string_index(B, B.amap, B.nel_a, s_a) : a;
        active = sa >= 0 && !(ks == kd && g.type != 2 && sa < a);
    }
    double acc = 0.0;
    if (active) {
        const int R = g.rank;
        for (int q = threadIdx.x; q < R; q += blockDim.x)
            spa[q] = 0.0;
        __syncthreads();
        if (threadIdx.x < R) {
            const Ti *z = N.z + g.za_off;
            const double *w = N.w + g.wa_off + (i64)threadIdx.x * g.nza;
            double v = 0.0;
            for (int q = 0; q < g.nza; ++q) v += par(s_a & z[q]) ? -w[q] : w[q];
            spa[threadIdx.x] = v;
        }
        __syncthreads();
        const int nb = B.blk_nb[kd], nbs = B.blk_nb[ks];
        const bool same = (ks == kd);
        const i64 drow = B.blk_off[kd] + (i64)a * nb;
        const i64 srow = B.blk_off[ks] + (i64)sa * nbs;
        const Ti *bstrs = B.bstrs + B.blk_bstart[kd];
        const Ti *zb = N.z + g.zb_off;
        const double *wb = N.w + g.wb_off;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            const Ti s_b = bstrs[b] ^ (Ti)g.bx;
            const int sb = g.bx ? string_index(B, B.bmap, B.nel_b, s_b) : b;
            if (sb < 0 || (same && g.type == 2 && sb < b)) continue;
            double vt = 0.0;
            for (int rr = 0; rr < R; ++rr) {
                double pb = 0.0;
                const double *w = wb + (i64)rr * g.nzb;
                for (int q = 0; q < g.nzb; ++q) pb += par(s_b & zb[q]) ? -w[q] : w[q];
                vt += spa[rr] * pb;
            }
            const i64 di = drow + b, si = srow + sb;
            if (OP == kExpm) {
                // expm_update, core/math.hpp:132-146: c0 = cos-1, c1 = sin
                const double vd = 1.0 + ang.c0 * (vt * vt), vo = ang.c1 * vt;
                const double vi = l[si], vj = l[di];
                l[si] = vi * vd - vj * vo;
                l[di] = vj * vd + vi * vo;
            } else if (OP == kGrad) {
                // grad_update, core/math.hpp:148-162: c0 = -sin, c1 = cos
                const double vd = ang.c0 * (vt * vt), vo = ang.c1 * vt;
                const double rvi = r[si], rvj = r[di];
                acc += l[si] * (rvi * vd + rvj * vo) + l[di] * (rvj * vd - rvi * vo);
            } else if (OP == kPairTvec) {
                // tvec_update, core/math.hpp:165-170: l = src, r = dst; a diagonal
                // group has si == di and the second store leaves dst = src * vt
                const double ss = l[si], sd = l[di];
                r[si] = sd * (-vt);
                r[di] = ss * vt;
            } else if (OP == kPairBacktran) {
                if (g.type == 0) {   // op/backtran.hpp:7-70: the diagonal exponential is 1
                    X.b[di] = l[di] * vt;
                } else {             // backtran_update, core/math.hpp:217-226
                    const double vd = 1.0 + ang.c0 * (vt * vt), vo = ang.c1 * vt;
                    const double li = l[si], lj = l[di], ri = r[si], rj = r[di];
                    const double ls = li * vd - lj * vo, ld = lj * vd + li * vo;
                    l[si] = ls;
                    l[di] = ld;
                    r[si] = ri * vd - rj * vo;
                    r[di] = rj * vd + ri * vo;
                    X.b[si] = ld * (-vt);
                    X.b[di] = ls * vt;
                }
            } else if (OP == kPairTran) {
                // tran_update, core/math.hpp:180-184; diagonal groups l_i vt r_i (op/batchtran.hpp:7-81)
                acc += g.type == 0 ? l[di] * vt * r[di] : l[si] * vt * r[di] - l[di] * vt * r[si];
            } else if (OP == kPairBatchExpm) {
                // expm_batch_update_matrix, core/math.hpp:228-252: the first nv entries of rows si, di
                const double vd = 1.0 + ang.c0 * (vt * vt), vo = ang.c1 * vt;
                double *sp = l + si * X.ld, *dp = l + di * X.ld;
                for (int k = 0; k < X.nv; ++k) {
                    const double vi = sp[k], vj = dp[k];
                    sp[k] = vi * vd - vj * vo;
                    dp[k] = vj * vd + vi * vo;
                }
            } else {
                // backgrad_update, core/math.hpp:187-215
                const double evd = 1.0 + ang.c0 * (vt * vt), evo = ang.c1 * vt;
                const double gvd = ang.c2 * (vt * vt), gvo = ang.c3 * vt;
                const double lvi = l[si], lvj = l[di], rvi = r[si], rvj = r[di];
                const double els = lvi * evd - lvj * evo;
                const double eld = lvj * evd + lvi * evo;
                acc += els * (rvi * gvd + rvj * gvo) + eld * (rvj * gvd - rvi * gvo);
                l[si] = els;
                l[di] = eld;
                r[si] = rvi * evd - rvj * evo;
                r[di] = rvj * evd + rvi * evo;
            }
        }
    }
    if (!pair_reduces(OP)) return;
    // ---- deterministic reduction --------------------------------------------
    acc = warp_sum(acc);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = acc;
    __syncthreads();
    const unsigned nslots = gridDim.x * gridDim.y;
    const unsigned slot = blockIdx.y * gridDim.x + blockIdx.x;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
        partials[slot] = s;
        __threadfence();
        const unsigned long long t = atomicAdd(ticket, 1ull);
        last = (t == nslots - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double s = 0.0;
    for (unsigned i = threadIdx.x; i < nslots; i += blockDim.x) s += __ldcg(partials + i);
    s = warp_sum(s);
    if (lane == 0) red[wid] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) tot += red[i];
        out[0] = accumulate ? out[0] + tot : tot;
        *ticket = 0ull;   // ready for the next launch on this stream
    }
}

// ---- host side -----------------------------------------------------------------

template <typename Ti>
static int check_group(const DevNet<Ti> *N, i64 gidx)
{
    if (gidx < 0 || gidx >= N->ngs) {
        set_error("group index %lld out of range [0, %lld)", gidx, N->ngs);
        return BSIM_ERR_ARG;
    }
    return BSIM_OK;
}

// scratch layout: [nslots doubles][ticket]; the ticket must start at zero.
template <typename Ti>
static int pair_scratch(const DevBasis<Ti> *B, double **part, unsigned long long **ticket, cudaStream_t s)
{
    (void)s;
    const size_t nslots = (size_t)pair_grid(B);
    Workspace &ws = workspace_for(B);
    // [nslots partials][ticket][result slot of the synchronous legacy calls]
    int st = ws.partials(nslots + 2, part);
    if (st != BSIM_OK) return st;
    *ticket = reinterpret_cast<unsigned long long *>(*part + nslots);
    return BSIM_OK;
}

template <typename Ti, int OP>
static int launch_pair(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, PairAngles ang, double *l, double *r,
                       double *out, bool accumulate, cudaStream_t s, double *ext_part, size_t ext_n,
                       PairExtra X = PairExtra{nullptr, 0, 0})
{
    int st = check_group(N, gidx);
    if (st != BSIM_OK) return st;
    if (B->num_blocks == 0 || B->max_na == 0) {
        if (pair_reduces(OP) && !accumulate) BSIM_CUDA(cudaMemsetAsync(out, 0, sizeof(double), s));
        return BSIM_OK;
    }
    double *part = nullptr;
    unsigned long long *ticket = nullptr;
    if (pair_reduces(OP)) {
        if (ext_part) {
            if (ext_n < (size_t)pair_grid(B) + 1) { set_error("scratch too small"); return BSIM_ERR_TOO_LARGE; }
            part = ext_part;
            ticket = reinterpret_cast<unsigned long long *>(part + pair_grid(B));
        } else {
            st = pair_scratch(B, &part, &ticket, s);
            if (st != BSIM_OK) return st;
        }
    }
    if constexpr (OP <= kPairBackgrad) {   // the pair-list kernels serve expm, grad, backgrad
        bool used = false;
        // with caller-provided scratch (the no-allocation entry point) the
        // lists are used only if an earlier call built them
        st = pair_list_launch<Ti, OP>(B, N, gidx, ang, l, r, part, ticket, pair_grid(B), out, accumulate, s, &used,
                                      ext_part == nullptr);
        if (st != BSIM_OK || used) return st;
    }
    dim3 grid(B->max_na, B->num_blocks);
    pair_row_kernel<Ti, OP><<<grid, kPairThreads, 0, s>>>(B->view, N->view, (int)gidx, ang, l, r, part, ticket, out,
                                                         accumulate ? 1 : 0, X);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename Ti>
int expm(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, double theta, double *v, cudaStream_t s)
{
    PairAngles a{cos(theta) - 1.0, sin(theta), 0.0, 0.0};
    return launch_pair<Ti, kExpm>(B, N, gidx, a, v, nullptr, nullptr, false, s, nullptr, 0);
}

template <typename Ti>
int grad(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, double theta, const double *l, const double *r,
         double *out_dev, bool accumulate, cudaStream_t s, double *scratch, size_t scratch_n)
{
    PairAngles a{-sin(theta), cos(theta), 0.0, 0.0};
    return launch_pair<Ti, kGrad>(B, N, gidx, a, const_cast<double *>(l), const_cast<double *>(r), out_dev, accumulate,
                                  s, scratch, scratch_n);
}

template <typename Ti>
int backgrad(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, double theta, double *l, double *r,
             double *out_dev, bool accumulate, cudaStream_t s)
{
    // exp(-theta G) with the gradient at +theta (reference op/backgrad.hpp:81-84)
    PairAngles a{cos(theta) - 1.0, -sin(theta), -sin(theta), cos(theta)};
    return launch_pair<Ti, kBackgrad>(B, N, gidx, a, l, r, out_dev, accumulate, s, nullptr, 0);
}

template <typename Ti>
int tvec(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, const double *src, double *dst, cudaStream_t s)
{
    if (B->dim > 0) BSIM_CUDA(cudaMemsetAsync(dst, 0, sizeof(double) * B->dim, s));   // op/tvec.hpp: dst zeroed
    return launch_pair<Ti, kPairTvec>(B, N, gidx, PairAngles{0, 0, 0, 0}, const_cast<double *>(src), dst, nullptr,
                                      false, s, nullptr, 0);
}

template <typename Ti>
int backtran(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, double theta, double *l, double *r, double *b,
             cudaStream_t s)
{
    if (B->dim > 0) BSIM_CUDA(cudaMemsetAsync(b, 0, sizeof(double) * B->dim, s));     // op/backtran.hpp: b zeroed
    PairAngles a{cos(theta) - 1.0, sin(theta), 0.0, 0.0};                            // backtran.hpp:75-76
    return launch_pair<Ti, kPairBacktran>(B, N, gidx, a, l, r, nullptr, false, s, nullptr, 0, PairExtra{b, 0, 0});
}

template <typename Ti>
int batchexpm(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, double theta, double *matrix, int ld, int nv,
              cudaStream_t s)
{
    if (nv < 0 || ld < nv) { set_error("batchexpm needs 0 <= num_vecs <= ld (got %d, %d)", nv, ld); return BSIM_ERR_ARG; }
    int st = check_group(N, gidx);
    if (st != BSIM_OK) return st;
    if (nv == 0 || N->groups[gidx].type == 0) return BSIM_OK;   // diagonal groups: identity for real vectors
    PairAngles a{cos(theta) - 1.0, sin(theta), 0.0, 0.0};
    return launch_pair<Ti, kPairBatchExpm>(B, N, gidx, a, matrix, nullptr, nullptr, false, s, nullptr, 0,
                                           PairExtra{nullptr, ld, nv});
}

// trans[orig] = <l|T_g|r> for every group (op/batchtran.hpp:514-528): the
// off-diagonal groups through the pool-gradient kernels at theta = 0 (the
// update rules coincide there), the diagonal groups through the row kernel.
template <typename Ti>
int batchtran(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *l, const double *r, double *trans,
              cudaStream_t s)
{
    if (N->ngs == 0) return BSIM_OK;
    double *zeros = nullptr;
    BSIM_CUDA(dmalloc_async(&zeros, sizeof(double) * N->ngs, s));
    cudaError_t e = cudaMemsetAsync(zeros, 0, sizeof(double) * N->ngs, s);
    int st = e == cudaSuccess ? BSIM_OK : cuda_status(e, "batchtran");
    if (st == BSIM_OK) e = cudaMemsetAsync(trans, 0, sizeof(double) * N->ngs, s);
    if (st == BSIM_OK && e != cudaSuccess) st = cuda_status(e, "batchtran");
    if (st == BSIM_OK) st = batchgrad(B, N, zeros, l, r, trans, s);
    cudaFreeAsync(zeros, s);
    if (st != BSIM_OK) return st;
    for (i64 g = 0; g < N->ngs; ++g) {
        const GroupDev &G = N->groups[g];
        if (G.type != 0) continue;
        st = launch_pair<Ti, kPairTran>(B, N, g, PairAngles{0, 0, 0, 0}, const_cast<double *>(l),
                                        const_cast<double *>(r), trans + G.orig, true, s, nullptr, 0);
        if (st != BSIM_OK) return st;
    }
    return BSIM_OK;
}

template int tvec<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, i64, const double *, double *,
                            cudaStream_t);
template int backtran<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, i64, double, double *, double *,
                                double *, cudaStream_t);
template int batchexpm<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, i64, double, double *, int,
                                 int, cudaStream_t);
template int batchtran<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, const double *, const double *,
                                 double *, cudaStream_t);
template int tvec<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, i64,
                                      const double *, double *, cudaStream_t);
template int backtran<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *,
                                          i64, double, double *, double *, double *, cudaStream_t);
template int batchexpm<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *,
                                           i64, double, double *, int, int, cudaStream_t);
template int batchtran<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *,
                                           const double *, const double *, double *, cudaStream_t);

template int expm<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, i64, double, double *, cudaStream_t);
template int grad<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, i64, double, const double *,
                            const double *, double *, bool, cudaStream_t, double *, size_t);
template int backgrad<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, i64, double, double *, double *,
                                double *, bool, cudaStream_t);
template int expm<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, i64, double, double *, cudaStream_t);
template int grad<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, i64, double, const double *,
                            const double *, double *, bool, cudaStream_t, double *, size_t);
template int backgrad<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, i64, double, double *, double *,
                                double *, bool, cudaStream_t);

}  // namespace bsim
