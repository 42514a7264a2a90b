// Complex (c64) operators: the reference CPU library's _c64 entry points
// (src/extern/otf_native.cpp:4,6 with Tv = complex<double>; op/hvec.hpp,
// op/expm.hpp, op/grad.hpp, op/backgrad.hpp, op/tvec.hpp, op/backtran.hpp,
// op/batchexpm.hpp, op/batchgrad.hpp, op/batchtran.hpp) on device vectors of
// interleaved (re, im) doubles.  The reference has no GPU counterpart.
//
// The update rules are those of core/math.hpp:7-252 for complex Tv, diagonal
// groups included: e^{theta G} multiplies by exp(i theta Im vt), its gradient
// weight is vt exp(i theta Im vt) (fast_diag_exp / fast_diag_grad).
//
// Kernels: one CTA per destination alpha row of every block, lanes over the
// row's beta columns (the row-pair scheme of the real operators in
// pairops.cu, with the reference's once-per-pair rule); sigma loops over all
// groups inside the CTA, so each CTA owns its destination row and needs no
// atomics.  Scalar results reduce deterministically through per-CTA partials
// summed in slot order by the last CTA.
#include "../../include/binsim_cuotf.h"
#include "ops.h"

#include <cmath>

namespace bsim {

namespace {

struct cx {
    double x, y;
};
__device__ __forceinline__ cx cadd(cx a, cx b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cx csub(cx a, cx b) { return {a.x - b.x, a.y - b.y}; }
__device__ __forceinline__ cx cmul(cx a, cx b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ cx cconj(cx a) { return {a.x, -a.y}; }
__device__ __forceinline__ cx cscale(double s, cx a) { return {s * a.x, s * a.y}; }
__device__ __forceinline__ double cnorm2(cx a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ cx cexpi(double t) { return {cos(t), sin(t)}; }

enum C64Op { cExpm = 0, cGrad, cBackgrad, cTvec, cBacktran, cBatchExpm, cTran, cDiag };
__host__ __device__ constexpr bool c64_reduces(int op) { return op == cGrad || op == cBackgrad || op == cTran; }

constexpr int kC64Threads = 256;

// P_r(s) = sum_k (-1)^{popc(s & z_k)} w[r][k] for r < R (precompute_phase,
// core/math.hpp:37-78), the group's weights column-major [nz x R]
template <typename Ti>
__device__ __forceinline__ cx cphase(u64 s, const Ti *z, int nz, const cx *w)
{
    cx v = {0.0, 0.0};
    for (int q = 0; q < nz; ++q) v = par(s & (u64)z[q]) ? csub(v, w[q]) : cadd(v, w[q]);
    return v;
}

// Source block and source alpha row of destination row a of block kd for group
// g, with the once-per-pair rule of op/expm.hpp:93-351 when `once`; false when
// the row has no partner.
template <typename Ti>
__device__ __forceinline__ bool source_row(const BasisView<Ti> &B, const GroupDev &g, int kd, int a, bool once,
                                           int *ks_out, int *sa_out, Ti *s_a)
{
    if (a >= B.blk_na[kd]) return false;
    const int nirr = B.num_irreps;
    const int as = B.blk_asym[kd] ^ g.asym, bs = B.blk_bsym[kd] ^ g.bsym;
    const int ks = (as < nirr && bs < nirr) ? B.block_map[as * nirr + bs] : -1;
    if (ks < 0 || (once && ks < kd)) return false;
    *s_a = B.astrs[B.blk_astart[kd] + a] ^ (Ti)g.ax;
    const int sa = g.ax ? string_index(B, B.amap, B.nel_a, *s_a) : a;
    if (sa < 0 || (once && ks == kd && g.type != 2 && sa < a)) return false;
    *ks_out = ks;
    *sa_out = sa;
    return true;
}

// ---- sigma: dst = H src over all groups (op/hvec.hpp:481-496, every ordered pair) ----
template <typename Ti>
__global__ void __launch_bounds__(kC64Threads)
c64_hvec_kernel(const BasisView<Ti> B, const NetView<Ti> N, const cx *__restrict__ src, cx *__restrict__ dst)
{
    __shared__ cx spa[kMaxRank];
    const int kd = blockIdx.y, a = blockIdx.x;
    if (a >= B.blk_na[kd]) return;   // uniform across the CTA
    const int nb = B.blk_nb[kd];
    const i64 drow = B.blk_off[kd] + (i64)a * nb;
    const cx *W = reinterpret_cast<const cx *>(N.w);
    const Ti *bstrs = B.bstrs + B.blk_bstart[kd];
    for (int b0 = 0; b0 < nb; b0 += blockDim.x) {
        const int b = b0 + threadIdx.x;
        cx acc = {0.0, 0.0};
        for (int gi = 0; gi < N.ngs; ++gi) {
            const GroupDev g = N.g[gi];
            int ks = -1, sa = -1;
            Ti s_a = 0;
            if (!source_row(B, g, kd, a, false, &ks, &sa, &s_a)) continue;   // uniform
            __syncthreads();   // the previous group's phases are consumed
            if (threadIdx.x < g.rank) spa[threadIdx.x] = cphase(s_a, N.z + g.za_off, g.nza, W + g.wa_off + (i64)threadIdx.x * g.nza);
            __syncthreads();
            if (b >= nb) continue;
            const Ti s_b = bstrs[b] ^ (Ti)g.bx;
            const int sb = g.bx ? string_index(B, B.bmap, B.nel_b, s_b) : b;
            if (sb < 0) continue;
            cx vt = {0.0, 0.0};
            for (int rr = 0; rr < g.rank; ++rr)
                vt = cadd(vt, cmul(spa[rr], cphase(s_b, N.z + g.zb_off, g.nzb, W + g.wb_off + (i64)rr * g.nzb)));
            const i64 si = B.blk_off[ks] + (i64)sa * B.blk_nb[ks] + sb;
            acc = cadd(acc, cmul(src[si], vt));   // hvec_update, core/math.hpp:126-130
        }
        if (b < nb) dst[drow + b] = acc;
    }
}

// ---- one group: the pair operators ---------------------------------------------
struct C64Angles { double c0, c1, c2, c3, th_exp, th_grad; };

template <typename Ti, int OP>
__global__ void __launch_bounds__(kC64Threads)
c64_pair_kernel(const BasisView<Ti> B, const NetView<Ti> N, int gid, C64Angles ang, cx *__restrict__ l,
                cx *__restrict__ r, cx *__restrict__ b3, int ld, int nv, double *__restrict__ partials,
                unsigned long long *__restrict__ ticket, double *__restrict__ out, int accumulate)
{
    __shared__ cx spa[kMaxRank];
    __shared__ double red[2][32];
    __shared__ bool last;
    const int kd = blockIdx.y, a = blockIdx.x;
    const GroupDev g = N.g[gid];
    const cx *W = reinterpret_cast<const cx *>(N.w);
    int ks = -1, sa = -1;
    Ti s_a = 0;
    const bool active = source_row(B, g, kd, a, OP != cDiag, &ks, &sa, &s_a);
    cx acc = {0.0, 0.0};
    if (active) {   // uniform across the CTA
        if (threadIdx.x < g.rank) spa[threadIdx.x] = cphase(s_a, N.z + g.za_off, g.nza, W + g.wa_off + (i64)threadIdx.x * g.nza);
        __syncthreads();
        const int nb = B.blk_nb[kd], nbs = B.blk_nb[ks];
        const bool same = (ks == kd);
        const i64 drow = B.blk_off[kd] + (i64)a * nb;
        const i64 srow = B.blk_off[ks] + (i64)sa * nbs;
        const Ti *bstrs = B.bstrs + B.blk_bstart[kd];
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            const Ti s_b = bstrs[b] ^ (Ti)g.bx;
            const int sb = g.bx ? string_index(B, B.bmap, B.nel_b, s_b) : b;
            if (sb < 0 || (OP != cDiag && same && g.type == 2 && sb < b)) continue;
            cx vt = {0.0, 0.0};
            for (int rr = 0; rr < g.rank; ++rr)
                vt = cadd(vt, cmul(spa[rr], cphase(s_b, N.z + g.zb_off, g.nzb, W + g.wb_off + (i64)rr * g.nzb)));
            const i64 di = drow + b, si = srow + sb;
            const double n2 = cnorm2(vt);
            const cx vtc = cconj(vt);
            if (OP == cDiag) {   // get_diags_elements: diag += vt (op/hvec.hpp:498-554)
                l[di] = cadd(l[di], vt);
            } else if (g.type == 0) {
                // diagonal groups, core/math.hpp:7-35 (si == di)
                const cx ue = cexpi(vt.y * ang.th_exp);            // fast_diag_exp
                const cx du = cmul(vt, cexpi(vt.y * ang.th_grad));  // fast_diag_grad
                if (OP == cExpm) {
                    l[di] = cmul(l[di], ue);
                } else if (OP == cGrad) {
                    acc = cadd(acc, cmul(cconj(cmul(l[di], du)), r[di]));
                } else if (OP == cBackgrad) {
                    const cx ln = cmul(l[di], ue);
                    l[di] = ln;
                    acc = cadd(acc, cmul(cconj(cmul(ln, du)), r[di]));
                    r[di] = cmul(r[di], ue);
                } else if (OP == cTvec) {
                    r[di] = cmul(l[di], vt);
                } else if (OP == cBacktran) {
                    const cx ln = cmul(l[di], ue);
                    l[di] = ln;
                    r[di] = cmul(r[di], ue);
                    b3[di] = cmul(ln, vt);
                } else if (OP == cBatchExpm) {
                    cx *row = l + di * ld;
                    for (int k = 0; k < nv; ++k) row[k] = cmul(row[k], ue);
                } else if (OP == cTran) {
                    acc = cadd(acc, cmul(cconj(cmul(l[di], vt)), r[di]));
                }
            } else if (OP == cExpm || OP == cBatchExpm || OP == cBacktran) {
                // expm_update, core/math.hpp:132-146
                const double vd = 1.0 + ang.c0 * n2;
                const cx vf = cscale(ang.c1, vt), vr = cscale(ang.c1, vtc);
                if (OP == cBatchExpm) {
                    cx *sp = l + si * ld, *dp = l + di * ld;
                    for (int k = 0; k < nv; ++k) {
                        const cx vi = sp[k], vj = dp[k];
                        sp[k] = csub(cscale(vd, vi), cmul(vj, vr));
                        dp[k] = cadd(cscale(vd, vj), cmul(vi, vf));
                    }
                } else {
                    const cx li = l[si], lj = l[di];
                    const cx ls = csub(cscale(vd, li), cmul(lj, vr)), ldn = cadd(cscale(vd, lj), cmul(li, vf));
                    l[si] = ls;
                    l[di] = ldn;
                    if (OP == cBacktran) {   // backtran_update, core/math.hpp:217-226
                        const cx ri = r[si], rj = r[di];
                        r[si] = csub(cscale(vd, ri), cmul(rj, vr));
                        r[di] = cadd(cscale(vd, rj), cmul(ri, vf));
                        b3[si] = cmul(ldn, cscale(-1.0, vtc));   // tvec_update, :165-170
                        b3[di] = cmul(ls, vt);
                    }
                }
            } else if (OP == cGrad) {
                // grad_update, core/math.hpp:148-162
                const double vd = ang.c0 * n2;
                const cx vf = cscale(ang.c1, vt), vr = cscale(ang.c1, vtc);
                const cx rvi = r[si], rvj = r[di];
                acc = cadd(acc, cadd(cmul(cconj(l[si]), cadd(cscale(vd, rvi), cmul(rvj, vr))),
                                     cmul(cconj(l[di]), csub(cscale(vd, rvj), cmul(rvi, vf)))));
            } else if (OP == cBackgrad) {
                // backgrad_update, core/math.hpp:187-215
                const double evd = 1.0 + ang.c0 * n2, gvd = ang.c2 * n2;
                const cx ef = cscale(ang.c1, vt), er = cscale(ang.c1, vtc);
                const cx gf = cscale(ang.c3, vt), gr = cscale(ang.c3, vtc);
                const cx lvi = l[si], lvj = l[di], rvi = r[si], rvj = r[di];
                const cx els = csub(cscale(evd, lvi), cmul(lvj, er));
                const cx eld = cadd(cscale(evd, lvj), cmul(lvi, ef));
                acc = cadd(acc, cadd(cmul(cconj(els), cadd(cscale(gvd, rvi), cmul(rvj, gr))),
                                     cmul(cconj(eld), csub(cscale(gvd, rvj), cmul(rvi, gf)))));
                l[si] = els;
                l[di] = eld;
                r[si] = csub(cscale(evd, rvi), cmul(rvj, er));
                r[di] = cadd(cscale(evd, rvj), cmul(rvi, ef));
            } else if (OP == cTvec) {
                // tvec_update, core/math.hpp:165-170: l = src, r = dst
                const cx ss = l[si], sd = l[di];
                r[si] = cmul(sd, cscale(-1.0, vtc));
                r[di] = cmul(ss, vt);
            } else if (OP == cTran) {
                // tran_update, core/math.hpp:180-184
                acc = cadd(acc, csub(cmul(cconj(cmul(l[si], vt)), r[di]), cmul(cmul(cconj(l[di]), vt), r[si])));
            }
        }
    }
    if (!c64_reduces(OP)) return;
    // ---- deterministic reduction of the complex partial sums
    double re = warp_sum(acc.x), im = warp_sum(acc.y);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) { red[0][wid] = re; red[1][wid] = im; }
    __syncthreads();
    const unsigned nslots = gridDim.x * gridDim.y;
    const unsigned slot = blockIdx.y * gridDim.x + blockIdx.x;
    if (threadIdx.x == 0) {
        double sr = 0.0, si2 = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { sr += red[0][i]; si2 += red[1][i]; }
        partials[2 * slot] = sr;
        partials[2 * slot + 1] = si2;
        __threadfence();
        const unsigned long long t = atomicAdd(ticket, 1ull);
        last = (t == nslots - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double sr = 0.0, si2 = 0.0;
    for (unsigned i = threadIdx.x; i < nslots; i += blockDim.x) {
        sr += __ldcg(partials + 2 * i);
        si2 += __ldcg(partials + 2 * i + 1);
    }
    sr = warp_sum(sr);
    si2 = warp_sum(si2);
    if (lane == 0) { red[0][wid] = sr; red[1][wid] = si2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tr = 0.0, ti = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { tr += red[0][i]; ti += red[1][i]; }
        out[0] = accumulate ? out[0] + tr : tr;
        out[1] = accumulate ? out[1] + ti : ti;
        *ticket = 0ull;
    }
}

}  // namespace

namespace {

template <typename Ti>
int c64_scratch(const DevBasis<Ti> *B, double **part, unsigned long long **ticket, cudaStream_t s)
{
    const size_t nslots = (size_t)pair_grid(B);
    // The basis workspace starts with the real operators' [nslots partials][ticket]
    // [result slot], whose ticket word must stay zero between their launches; the
    // complex partials [2 * nslots][ticket] follow it.  The ticket is cleared
    // before every launch.
    double *base = nullptr;
    int st = B->ws.partials(3 * nslots + 3, &base);
    if (st != BSIM_OK) return st;
    *part = base + nslots + 2;
    *ticket = reinterpret_cast<unsigned long long *>(*part + 2 * nslots);
    BSIM_CUDA(cudaMemsetAsync(*ticket, 0, sizeof(unsigned long long), s));
    return BSIM_OK;
}

template <int OP, typename Ti>
int c64_launch(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, C64Angles ang, double *l, double *r, double *b3,
               int ld, int nv, double *out, bool accumulate, cudaStream_t s)
{
    if (gidx < 0 || gidx >= N->ngs) { set_error("group index %lld out of range [0, %lld)", (long long)gidx, (long long)N->ngs); return BSIM_ERR_ARG; }
    if (B->num_blocks == 0 || B->max_na == 0) {
        if (c64_reduces(OP) && !accumulate) BSIM_CUDA(cudaMemsetAsync(out, 0, 2 * sizeof(double), s));
        return BSIM_OK;
    }
    double *part = nullptr;
    unsigned long long *ticket = nullptr;
    if (c64_reduces(OP)) {
        int st = c64_scratch(B, &part, &ticket, s);
        if (st != BSIM_OK) return st;
    }
    dim3 grid(B->max_na, B->num_blocks);
    c64_pair_kernel<Ti, OP><<<grid, kC64Threads, 0, s>>>(B->view, N->view, (int)gidx, ang, reinterpret_cast<cx *>(l),
                                                         reinterpret_cast<cx *>(r), reinterpret_cast<cx *>(b3), ld, nv,
                                                         part, ticket, out, accumulate ? 1 : 0);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

// f(basis, complex network) for handles of one string type
template <class F>
int with_c64(void *basis, void *net, F &&f)
{
    if (is_u64_basis(basis)) {
        auto *n = static_cast<DevNet<unsigned long long> *>(net);
        if (!valid_c64(n)) { set_error("network handle is not a UInt64 c64 network of this library"); return BSIM_ERR_ARG; }
        return f(static_cast<DevBasis<unsigned long long> *>(basis), n);
    }
    auto *b = static_cast<DevBasis<unsigned> *>(basis);
    if (!valid(b)) { set_error("invalid basis handle"); return BSIM_ERR_ARG; }
    auto *n = static_cast<DevNet<unsigned> *>(net);
    if (!valid_c64(n)) { set_error("network handle is not a UInt32 c64 network of this library"); return BSIM_ERR_ARG; }
    return f(b, n);
}

#define NEED64(p) do { if (!(p)) { ::bsim::set_error("null pointer: " #p); return BSIM_ERR_NULL; } } while (0)

}  // namespace
}  // namespace bsim

using bsim::i64;

extern "C" {

int bsim_network_create_c64(const int64_t *orbsym, int64_t norb, int64_t ngs, const uint32_t *axs,
                            const uint32_t *bxs, const int64_t *ranks, const int64_t *num_zas,
                            const int64_t *num_zbs, const uint32_t *flat_zas, const uint32_t *flat_zbs,
                            const double *flat_wa, const double *flat_wb, void **out)
{
    if (!out) { bsim::set_error("null out"); return BSIM_ERR_NULL; }
    bsim::DevNet<unsigned> *n = nullptr;
    int st = bsim::make_network<unsigned>((const i64 *)orbsym, norb, ngs, axs, bxs, (const i64 *)ranks,
                                          (const i64 *)num_zas, (const i64 *)num_zbs, flat_zas, flat_zbs, flat_wa,
                                          flat_wb, &n, true);
    *out = n;
    return st;
}

int bsim_network_create_c64_u64(const int64_t *orbsym, int64_t norb, int64_t ngs, const uint64_t *axs,
                                const uint64_t *bxs, const int64_t *ranks, const int64_t *num_zas,
                                const int64_t *num_zbs, const uint64_t *flat_zas, const uint64_t *flat_zbs,
                                const double *flat_wa, const double *flat_wb, void **out)
{
    if (!out) { bsim::set_error("null out"); return BSIM_ERR_NULL; }
    using U = unsigned long long;
    bsim::DevNet<U> *n = nullptr;
    int st = bsim::make_network<U>((const i64 *)orbsym, norb, ngs, (const U *)axs, (const U *)bxs, (const i64 *)ranks,
                                   (const i64 *)num_zas, (const i64 *)num_zbs, (const U *)flat_zas,
                                   (const U *)flat_zbs, flat_wa, flat_wb, &n, true);
    *out = n;
    return st;
}

int bsim_hvec_c64(void *basis, void *net, const double *src, double *dst, bsim_stream_t stream)
{
    return bsim::with_c64(basis, net, [&](auto *b, auto *n) -> int {
        NEED64(src); NEED64(dst);
        if (b->dim == 0) return BSIM_OK;
        dim3 grid(b->max_na, b->num_blocks);
        bsim::c64_hvec_kernel<<<grid, bsim::kC64Threads, 0, stream>>>(b->view, n->view, reinterpret_cast<const bsim::cx *>(src),
                                                          reinterpret_cast<bsim::cx *>(dst));
        BSIM_CUDA(cudaGetLastError());
        return BSIM_OK;
    });
}

int bsim_diag_c64(void *basis, void *net, double *diag, bsim_stream_t stream)
{
    return bsim::with_c64(basis, net, [&](auto *b, auto *n) -> int {
        NEED64(diag);
        if (n->diag_group < 0) return BSIM_OK;   // accumulates; nothing to add
        return bsim::c64_launch<bsim::cDiag>(b, n, n->diag_group, bsim::C64Angles{}, diag, nullptr, nullptr, 0, 0, nullptr, false,
                                 stream);
    });
}

int bsim_expm_c64(void *basis, void *net, int64_t idx, double theta, double *vec, bsim_stream_t stream)
{
    return bsim::with_c64(basis, net, [&](auto *b, auto *n) -> int {
        NEED64(vec);
        bsim::C64Angles a{cos(theta) - 1.0, sin(theta), 0.0, 0.0, theta, 0.0};   // op/expm.hpp:71-72
        return bsim::c64_launch<bsim::cExpm>(b, n, idx, a, vec, nullptr, nullptr, 0, 0, nullptr, false, stream);
    });
}

int bsim_grad_c64(void *basis, void *net, int64_t idx, double theta, const double *l, const double *r,
                  double *out_dev, bsim_stream_t stream)
{
    return bsim::with_c64(basis, net, [&](auto *b, auto *n) -> int {
        NEED64(l); NEED64(r); NEED64(out_dev);
        bsim::C64Angles a{-sin(theta), cos(theta), 0.0, 0.0, 0.0, theta};   // op/grad.hpp:76-77
        return bsim::c64_launch<bsim::cGrad>(b, n, idx, a, const_cast<double *>(l), const_cast<double *>(r), nullptr, 0, 0,
                                 out_dev, false, stream);
    });
}

int bsim_backgrad_c64(void *basis, void *net, int64_t idx, double theta, double *l, double *r, double *out_dev,
                      bsim_stream_t stream)
{
    return bsim::with_c64(basis, net, [&](auto *b, auto *n) -> int {
        NEED64(l); NEED64(r); NEED64(out_dev);
        // exp(-theta G) with the gradient at +theta (op/backgrad.hpp:81-84; diagonal groups :61-62)
        bsim::C64Angles a{cos(theta) - 1.0, -sin(theta), -sin(theta), cos(theta), -theta, theta};
        return bsim::c64_launch<bsim::cBackgrad>(b, n, idx, a, l, r, nullptr, 0, 0, out_dev, false, stream);
    });
}

int bsim_tvec_c64(void *basis, void *net, int64_t idx, const double *src, double *dst, bsim_stream_t stream)
{
    return bsim::with_c64(basis, net, [&](auto *b, auto *n) -> int {
        NEED64(src); NEED64(dst);
        if (b->dim > 0) BSIM_CUDA(cudaMemsetAsync(dst, 0, 2 * sizeof(double) * b->dim, stream));
        return bsim::c64_launch<bsim::cTvec>(b, n, idx, bsim::C64Angles{}, const_cast<double *>(src), dst, nullptr, 0, 0, nullptr,
                                 false, stream);
    });
}

int bsim_backtran_c64(void *basis, void *net, int64_t idx, double theta, double *l, double *r, double *bvec,
                      bsim_stream_t stream)
{
    return bsim::with_c64(basis, net, [&](auto *b, auto *n) -> int {
        NEED64(l); NEED64(r); NEED64(bvec);
        if (b->dim > 0) BSIM_CUDA(cudaMemsetAsync(bvec, 0, 2 * sizeof(double) * b->dim, stream));
        bsim::C64Angles a{cos(theta) - 1.0, sin(theta), 0.0, 0.0, theta, 0.0};   // op/backtran.hpp:75-76
        return bsim::c64_launch<bsim::cBacktran>(b, n, idx, a, l, r, bvec, 0, 0, nullptr, false, stream);
    });
}

int bsim_batchexpm_c64(void *basis, void *net, int64_t idx, double theta, double *matrix, int ld, int num_vecs,
                       bsim_stream_t stream)
{
    return bsim::with_c64(basis, net, [&](auto *b, auto *n) -> int {
        NEED64(matrix);
        if (num_vecs < 0 || ld < num_vecs) { bsim::set_error("batchexpm needs 0 <= num_vecs <= ld (got %d, %d)", num_vecs, ld); return BSIM_ERR_ARG; }
        if (num_vecs == 0) return BSIM_OK;
        bsim::C64Angles a{cos(theta) - 1.0, sin(theta), 0.0, 0.0, theta, 0.0};   // op/batchexpm.hpp:73-74
        return bsim::c64_launch<bsim::cBatchExpm>(b, n, idx, a, matrix, nullptr, nullptr, ld, num_vecs, nullptr, false, stream);
    });
}

// grads[orig] (complex) = <l| G e^{theta G} |r> for every group at thetas[orig]
// (op/batchgrad.hpp:529-540); one launch per group.
int bsim_batchgrad_c64(void *basis, void *net, const double *thetas_host, const double *l, const double *r,
                       double *grads, bsim_stream_t stream)
{
    return bsim::with_c64(basis, net, [&](auto *b, auto *n) -> int {
        NEED64(l); NEED64(r); NEED64(grads);
        if (n->ngs > 0) NEED64(thetas_host);
        for (i64 g = 0; g < n->ngs; ++g) {
            const double t = thetas_host[g];
            bsim::C64Angles a{-sin(t), cos(t), 0.0, 0.0, 0.0, t};
            int st = bsim::c64_launch<bsim::cGrad>(b, n, g, a, const_cast<double *>(l), const_cast<double *>(r), nullptr, 0, 0,
                                       grads + 2 * g, false, stream);
            if (st != BSIM_OK) return st;
        }
        return (int)BSIM_OK;
    });
}

// trans[orig] (complex) = <l| T_g |r> for every group (op/batchtran.hpp:514-528)
int bsim_batchtran_c64(void *basis, void *net, const double *l, const double *r, double *trans, bsim_stream_t stream)
{
    return bsim::with_c64(basis, net, [&](auto *b, auto *n) -> int {
        NEED64(l); NEED64(r); NEED64(trans);
        for (i64 g = 0; g < n->ngs; ++g) {
            int st = bsim::c64_launch<bsim::cTran>(b, n, g, bsim::C64Angles{}, const_cast<double *>(l), const_cast<double *>(r),
                                       nullptr, 0, 0, trans + 2 * g, false, stream);
            if (st != BSIM_OK) return st;
        }
        return (int)BSIM_OK;
    });
}

}  // extern "C"
