// Pair operators (expm, grad, backgrad) over precomputed pair lists.
//
// The row kernel in pairops.cu gives every destination alpha row a CTA and
// finds each row's partner, each column's partner and both phases inside the
// CTA, one dependent global lookup after the other.  For single-block bases
// this file instead keeps, per X mask, the list of its connected string pairs
// (built once per basis and network on the host):
//   alpha half list of ax : (a, a^ax) with idx(a^ax) > a     (types 1 and 3)
//   beta list of bx       : (b, b^bx) for every connected b, the entries with
//                           idx(b^bx) > b first                (type 3 all, type 2 the first part)
// and the identity for the untouched spin.  A launch covers the group's pairs
// as tiles of (4 alpha entries) x (256 beta entries): each thread owns one beta
// entry, computes its beta phases, and updates its 4 pairs with all loads
// issued before the stores.  The pair ownership is the reference's (one update per unordered
// pair, op/expm.hpp:7-372), and the update formulas are those of
// core/math.hpp:132-215.  grad/backgrad reduce deterministically through
// per-CTA partials and a last-CTA ticket, like the row kernel.
#include "ops.h"

#include <algorithm>
#include <mutex>
#include <unordered_map>

namespace bsim {

namespace {

constexpr int kListCols = 256;     // beta entries per CTA (one per thread)
constexpr int kListMaxRank = 4;
constexpr int kListMaxZ = 64;      // Z masks per spin staged in shared memory

// One group's work for the batched gradient: its pair lists, phase data and
// tile count (tiles of kBatchRows alpha entries x kListCols beta entries).
struct BGroup {
    int aoff, acnt, boff, bcnt;   // list offsets (-1: identity) and lengths
    int R, nza, nzb, orig;
    int ntx, pad;
    i64 za_off, zb_off, wa_off, wb_off;
};
constexpr int kBatchRows = 16;   // alpha entries per tile of the batched gradient (loads in groups of 4)

template <typename Ti>
struct PairPlan {
    const void *basis = nullptr;
    i64 basis_dim = -1;
    bool ok = false;
    std::vector<int4> desc;        // per group: {alpha offset or -1, alpha count, beta offset or -1, beta count}
    Arena arena;
    const int2 *d_alist = nullptr, *d_blist = nullptr;
    // batched gradient over the whole network (built on first use)
    int bg_state = 0;              // 0 not built, 1 usable, -1 a group needs the tile kernel
    i64 bg_tiles = 0;
    int bg_n = 0;
    BGroup *d_bg = nullptr;
    i64 *d_tstart = nullptr;
    ~PairPlan()
    {
        arena.release();
        if (d_bg) cudaFree(d_bg);
        if (d_tstart) cudaFree(d_tstart);
    }
};

std::mutex g_pair_mu;

template <typename Ti>
int build_pair_plan(const DevBasis<Ti> *B, const DevNet<Ti> *N, PairPlan<Ti> *P)
{
    P->basis = B;
    P->basis_dim = B->dim;
    P->ok = false;
    if (B->num_blocks != 1) return BSIM_OK;
    const int nA = B->na[0], nB = B->nb[0];
    std::unordered_map<u64, int> amap, bmap;
    amap.reserve((size_t)nA * 2);
    bmap.reserve((size_t)nB * 2);
    for (int a = 0; a < nA; ++a) amap[(u64)B->astrs[a]] = a;
    for (int b = 0; b < nB; ++b) bmap[(u64)B->bstrs[b]] = b;
    std::vector<int2> alist, blist;
    std::unordered_map<u64, int2> aidx, bidx;   // mask -> {offset, count} (beta: count of the whole list)
    std::unordered_map<u64, int> bhalf;         // beta mask -> entries with partner index above
    auto alpha_list = [&](u64 x) {
        auto it = aidx.find(x);
        if (it != aidx.end()) return it->second;
        const int off = (int)alist.size();
        for (int a = 0; a < nA; ++a) {
            auto f = amap.find((u64)B->astrs[a] ^ x);
            if (f != amap.end() && f->second > a) alist.push_back(make_int2(a, f->second));
        }
        const int2 r = make_int2(off, (int)alist.size() - off);
        aidx[x] = r;
        return r;
    };
    auto beta_list = [&](u64 x) {
        auto it = bidx.find(x);
        if (it != bidx.end()) return it->second;
        const int off = (int)blist.size();
        for (int b = 0; b < nB; ++b) {   // partner index above first: the pure-beta half
            auto f = bmap.find((u64)B->bstrs[b] ^ x);
            if (f != bmap.end() && f->second > b) blist.push_back(make_int2(b, f->second));
        }
        bhalf[x] = (int)blist.size() - off;
        for (int b = 0; b < nB; ++b) {
            auto f = bmap.find((u64)B->bstrs[b] ^ x);
            if (f != bmap.end() && f->second < b) blist.push_back(make_int2(b, f->second));
        }
        const int2 r = make_int2(off, (int)blist.size() - off);
        bidx[x] = r;
        return r;
    };
    P->desc.assign((size_t)N->ngs, make_int4(-1, 0, -1, 0));
    for (i64 g = 0; g < N->ngs; ++g) {
        const GroupDev &G = N->groups[g];
        if (G.type == 1) {
            const int2 a = alpha_list(G.ax);
            P->desc[g] = make_int4(a.x, a.y, -1, nB);
        } else if (G.type == 2) {
            const int2 b = beta_list(G.bx);
            P->desc[g] = make_int4(-1, nA, b.x, bhalf[G.bx]);
        } else if (G.type == 3) {
            const int2 a = alpha_list(G.ax), b = beta_list(G.bx);
            P->desc[g] = make_int4(a.x, a.y, b.x, b.y);
        }
    }
    const size_t bytes = (std::max<size_t>(alist.size(), 1) + std::max<size_t>(blist.size(), 1)) * sizeof(int2) + 1024;
    if (bytes > ((size_t)4 << 30)) return BSIM_OK;   // lists too large: the row kernel serves this network
    int st = P->arena.reserve(bytes);
    if (st != BSIM_OK) return st;
    int2 *da = P->arena.template take<int2>(std::max<size_t>(alist.size(), 1));
    int2 *db = P->arena.template take<int2>(std::max<size_t>(blist.size(), 1));
    if (!alist.empty()) BSIM_CUDA(cudaMemcpy(da, alist.data(), alist.size() * sizeof(int2), cudaMemcpyHostToDevice));
    if (!blist.empty()) BSIM_CUDA(cudaMemcpy(db, blist.data(), blist.size() * sizeof(int2), cudaMemcpyHostToDevice));
    P->d_alist = da;
    P->d_blist = db;
    P->ok = true;
    return BSIM_OK;
}

template <typename Ti>
int get_pair_plan(const DevBasis<Ti> *B, const DevNet<Ti> *N, PairPlan<Ti> **out)
{
    std::lock_guard<std::mutex> lk(g_pair_mu);
    auto *p = static_cast<PairPlan<Ti> *>(N->pair_state);
    if (p && p->basis == B && p->basis_dim == B->dim) { *out = p; return BSIM_OK; }
    if (p) { delete p; const_cast<DevNet<Ti> *>(N)->pair_state = nullptr; }
    p = new PairPlan<Ti>();
    int rc = build_pair_plan(B, N, p);
    if (rc != BSIM_OK) { delete p; return rc; }
    const_cast<DevNet<Ti> *>(N)->pair_state = p;
    const_cast<DevNet<Ti> *>(N)->pair_free = [](void *q) { delete static_cast<PairPlan<Ti> *>(q); };
    *out = p;
    return BSIM_OK;
}

// The cached plan of (B, N) if one exists; never builds one (no allocation).
template <typename Ti>
PairPlan<Ti> *find_pair_plan(const DevBasis<Ti> *B, const DevNet<Ti> *N)
{
    std::lock_guard<std::mutex> lk(g_pair_mu);
    auto *p = static_cast<PairPlan<Ti> *>(N->pair_state);
    return (p && p->basis == B && p->basis_dim == B->dim) ? p : nullptr;
}

struct ListArgs {
    int nB, acnt, bcnt, R, nza, nzb;
    const int2 *alist, *blist;   // nullptr: identity
    i64 za_off, zb_off, wa_off, wb_off;
};

template <typename Ti, int OP, int RT, int BATCH, int MINB>
__global__ void __launch_bounds__(kListCols, MINB)
pair_list_kernel(const Ti *__restrict__ astrs, const Ti *__restrict__ bstrs, const Ti *__restrict__ zall,
                 const double *__restrict__ wall, const ListArgs A, PairAngles ang, double *__restrict__ l,
                 double *__restrict__ r, double *__restrict__ partials, unsigned long long *__restrict__ ticket,
                 double *__restrict__ out, int accumulate)
{
    __shared__ double spa[RT][kListMaxRank];
    __shared__ long long arow[RT], asrc[RT];
    __shared__ double red[kListCols / 32];
    __shared__ bool last;
    // the group's Z masks and weights, staged once: the phase loops below then
    // run on shared memory instead of one global load per mask
    __shared__ unsigned long long zsa[kListMaxZ], zsb[kListMaxZ];
    __shared__ double wsa[kListMaxRank * kListMaxZ], wsb[kListMaxRank * kListMaxZ];
    const int t = threadIdx.x;
    const int R = A.R;
    for (int i = t; i < A.nza; i += kListCols) zsa[i] = (unsigned long long)zall[A.za_off + i];
    for (int i = t; i < A.nzb; i += kListCols) zsb[i] = (unsigned long long)zall[A.zb_off + i];
    for (int i = t; i < R * A.nza; i += kListCols) wsa[i] = wall[A.wa_off + i];
    for (int i = t; i < R * A.nzb; i += kListCols) wsb[i] = wall[A.wb_off + i];
    const int ntx = (A.acnt + RT - 1) / RT;
    const int ntiles = ntx * ((A.bcnt + kListCols - 1) / kListCols);
    double acc = 0.0;
    // grid-stride over (RT alpha entries) x (256 beta entries) tiles; the grid is
    // capped so the partial slots fit the basis' reduction scratch
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int tx = tile % ntx, ty = tile / ntx;
        __syncthreads();   // the previous tile's alpha entries are consumed
        if (t < RT) {
            const int i = tx * RT + t;
            long long ar = -1, as = -1;
            double p[kListMaxRank] = {0.0, 0.0, 0.0, 0.0};
            if (i < A.acnt) {
                const int2 e = A.alist ? A.alist[i] : make_int2(i, i);
                ar = (long long)e.x * A.nB;
                as = (long long)e.y * A.nB;
                const unsigned long long s = (unsigned long long)astrs[e.y];
                for (int q = 0; q < A.nza; ++q) {
                    const bool odd = par(s & zsa[q]);
#pragma unroll
                    for (int rr = 0; rr < kListMaxRank; ++rr)
                        if (rr < R) p[rr] += odd ? -wsa[rr * A.nza + q] : wsa[rr * A.nza + q];
                }
            }
            arow[t] = ar;
            asrc[t] = as;
#pragma unroll
            for (int rr = 0; rr < kListMaxRank; ++rr) spa[t][rr] = p[rr];
        }
        const int j = ty * kListCols + t;
        int b = -1, sb = -1;
        double pb[kListMaxRank] = {0.0, 0.0, 0.0, 0.0};
        if (j < A.bcnt) {
            const int2 e = A.blist ? A.blist[j] : make_int2(j, j);
            b = e.x;
            sb = e.y;
            const unsigned long long s = (unsigned long long)bstrs[sb];
            for (int q = 0; q < A.nzb; ++q) {
                const bool odd = par(s & zsb[q]);
#pragma unroll
                for (int rr = 0; rr < kListMaxRank; ++rr)
                    if (rr < R) pb[rr] += odd ? -wsb[rr * A.nzb + q] : wsb[rr * A.nzb + q];
            }
        }
        __syncthreads();
        if (b < 0) continue;
        // every pair of the tile is distinct: the loads of BATCH pairs are issued
        // before their stores
#pragma unroll
        for (int k0 = 0; k0 < RT; k0 += BATCH) {
            double lv_i[BATCH], lv_j[BATCH], rv_i[BATCH], rv_j[BATCH];
#pragma unroll
            for (int kk = 0; kk < BATCH; ++kk) {
                const int k = k0 + kk;
                lv_i[kk] = lv_j[kk] = rv_i[kk] = rv_j[kk] = 0.0;
                if (arow[k] < 0) continue;   // the tile's last alpha entries may run past the list
                const i64 di = arow[k] + b, si = asrc[k] + sb;
                if (OP == kPairGrad) {
                    lv_i[kk] = __ldg(l + si); lv_j[kk] = __ldg(l + di);
                    rv_i[kk] = __ldg(r + si); rv_j[kk] = __ldg(r + di);
                } else {
                    lv_i[kk] = l[si]; lv_j[kk] = l[di];
                    if (OP == kPairBackgrad) { rv_i[kk] = r[si]; rv_j[kk] = r[di]; }
                }
            }
#pragma unroll
            for (int kk = 0; kk < BATCH; ++kk) {
                const int k = k0 + kk;
                if (arow[k] < 0) continue;
                const i64 di = arow[k] + b, si = asrc[k] + sb;
                double t1 = 0.0;
#pragma unroll
                for (int rr = 0; rr < kListMaxRank; ++rr) t1 += spa[k][rr] * pb[rr];
                if (OP == kPairExpm) {
                    // expm_update, core/math.hpp:132-146: c0 = cos-1, c1 = sin
                    const double vd = 1.0 + ang.c0 * (t1 * t1), vo = ang.c1 * t1;
                    l[si] = lv_i[kk] * vd - lv_j[kk] * vo;
                    l[di] = lv_j[kk] * vd + lv_i[kk] * vo;
                } else if (OP == kPairGrad) {
                    // grad_update, core/math.hpp:148-162: c0 = -sin, c1 = cos
                    const double vd = ang.c0 * (t1 * t1), vo = ang.c1 * t1;
                    acc += lv_i[kk] * (rv_i[kk] * vd + rv_j[kk] * vo) + lv_j[kk] * (rv_j[kk] * vd - rv_i[kk] * vo);
                } else {
                    // backgrad_update, core/math.hpp:187-215
                    const double evd = 1.0 + ang.c0 * (t1 * t1), evo = ang.c1 * t1;
                    const double gvd = ang.c2 * (t1 * t1), gvo = ang.c3 * t1;
                    const double els = lv_i[kk] * evd - lv_j[kk] * evo;
                    const double eld = lv_j[kk] * evd + lv_i[kk] * evo;
                    acc += els * (rv_i[kk] * gvd + rv_j[kk] * gvo) + eld * (rv_j[kk] * gvd - rv_i[kk] * gvo);
                    l[si] = els;
                    l[di] = eld;
                    r[si] = rv_i[kk] * evd - rv_j[kk] * evo;
                    r[di] = rv_j[kk] * evd + rv_i[kk] * evo;
                }
            }
        }
    }
    if (OP == kPairExpm) return;
    // ---- deterministic reduction: CTA partials in slot order, summed by the last CTA
    acc = warp_sum(acc);
    const int lane = t & 31, wid = t >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = acc;
    __syncthreads();
    const unsigned nslots = gridDim.x;
    if (t == 0) {
        double s = 0.0;
        for (int i = 0; i < kListCols / 32; ++i) s += red[i];
        partials[blockIdx.x] = s;
        __threadfence();
        const unsigned long long tk = atomicAdd(ticket, 1ull);
        last = (tk == nslots - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double s = 0.0;
    for (unsigned i = t; i < nslots; i += kListCols) s += __ldcg(partials + i);
    s = warp_sum(s);
    if (lane == 0) red[wid] = s;
    __syncthreads();
    if (t == 0) {
        double tot = 0.0;
        for (int i = 0; i < kListCols / 32; ++i) tot += red[i];
        out[0] = accumulate ? out[0] + tot : tot;
        *ticket = 0ull;
    }
}

// Gradient of every group of a network at its own angle, one launch: the
// groups' tiles form one index space (prefix sums tstart); each CTA takes a
// contiguous range of tiles, so it meets few group boundaries, and adds its
// partial sum of a group into grads[orig] when it leaves the group.
template <typename Ti>
__global__ void __launch_bounds__(kListCols)
pair_list_batchgrad_kernel(const Ti *__restrict__ astrs, const Ti *__restrict__ bstrs, int nB,
                           const Ti *__restrict__ zall, const double *__restrict__ wall,
                           const int2 *__restrict__ alist_all, const int2 *__restrict__ blist_all,
                           const BGroup *__restrict__ groups, const i64 *__restrict__ tstart, int ngroups, i64 T,
                           const double *__restrict__ thetas, const double *__restrict__ l,
                           const double *__restrict__ r, double *__restrict__ grads,
                           const unsigned char *__restrict__ skip, const int *__restrict__ flag)
{
    __shared__ double spa[kBatchRows][kListMaxRank];
    __shared__ long long arow[kBatchRows], asrc[kBatchRows];
    __shared__ double red[kListCols / 32];
    __shared__ unsigned long long zsa[kListMaxZ], zsb[kListMaxZ];
    __shared__ double wsa[kListMaxRank * kListMaxZ], wsb[kListMaxRank * kListMaxZ];
    __shared__ BGroup G;
    __shared__ double ang0, ang1;
    __shared__ int gcur;
    __shared__ bool skipG;   // the current group is left to the theta = 0 density route
    const int t = threadIdx.x;
    const i64 t0 = (i64)blockIdx.x * T / gridDim.x, t1 = (i64)(blockIdx.x + 1) * T / gridDim.x;
    if (t0 >= t1) return;
    const bool route = skip && flag && *flag != 0;
    if (t == 0) {   // group of the first tile: last g with tstart[g] <= t0
        int lo = 0, hi = ngroups - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (tstart[mid] <= t0) lo = mid; else hi = mid - 1;
        }
        gcur = lo;
    }
    __syncthreads();
    int g = -1;
    double acc = 0.0;
    auto flush = [&]() {
        double v = warp_sum(acc);
        acc = 0.0;
        __syncthreads();
        if ((t & 31) == 0) red[t >> 5] = v;
        __syncthreads();
        if (t == 0 && !skipG) {
            double sum = 0.0;
            for (int i = 0; i < kListCols / 32; ++i) sum += red[i];
            atomicAdd(grads + G.orig, sum);
        }
    };
    for (i64 tile = t0; tile < t1; ++tile) {
        if (g < 0 || tile >= tstart[g + 1]) {   // entering a new group (uniform across the CTA)
            if (g >= 0) flush();
            __syncthreads();
            if (t == 0) {
                int gg = g < 0 ? gcur : g + 1;
                while (tile >= tstart[gg + 1]) ++gg;
                gcur = gg;
                G = groups[gg];
                const double th = thetas[G.orig];
                ang0 = -sin(th);   // grad_update, core/math.hpp:148-162
                ang1 = cos(th);
                skipG = route && skip[G.orig];
            }
            __syncthreads();
            g = gcur;
            if (skipG) {   // uniform: jump to the group's last tile in this CTA's range
                tile = min(t1, tstart[g + 1]) - 1;
                continue;
            }
            for (int i = t; i < G.nza; i += kListCols) zsa[i] = (unsigned long long)zall[G.za_off + i];
            for (int i = t; i < G.nzb; i += kListCols) zsb[i] = (unsigned long long)zall[G.zb_off + i];
            for (int i = t; i < G.R * G.nza; i += kListCols) wsa[i] = wall[G.wa_off + i];
            for (int i = t; i < G.R * G.nzb; i += kListCols) wsb[i] = wall[G.wb_off + i];
        }
        const i64 local = tile - tstart[g];
        const int tx = (int)(local % G.ntx), ty = (int)(local / G.ntx);
        const int2 *alist = G.aoff >= 0 ? alist_all + G.aoff : nullptr;
        const int2 *blist = G.boff >= 0 ? blist_all + G.boff : nullptr;
        const int R = G.R;
        __syncthreads();   // smem of the previous tile consumed, this group's masks staged
        if (t < kBatchRows) {
            const int i = tx * kBatchRows + t;
            long long ar = -1, as = -1;
            double p[kListMaxRank] = {0.0, 0.0, 0.0, 0.0};
            if (i < G.acnt) {
                const int2 e = alist ? alist[i] : make_int2(i, i);
                ar = (long long)e.x * nB;
                as = (long long)e.y * nB;
                const unsigned long long sv = (unsigned long long)astrs[e.y];
                for (int q = 0; q < G.nza; ++q) {
                    const bool odd = par(sv & zsa[q]);
#pragma unroll
                    for (int rr = 0; rr < kListMaxRank; ++rr)
                        if (rr < R) p[rr] += odd ? -wsa[rr * G.nza + q] : wsa[rr * G.nza + q];
                }
            }
            arow[t] = ar;
            asrc[t] = as;
#pragma unroll
            for (int rr = 0; rr < kListMaxRank; ++rr) spa[t][rr] = p[rr];
        }
        const int j = ty * kListCols + t;
        int b = -1, sb = -1;
        double pb[kListMaxRank] = {0.0, 0.0, 0.0, 0.0};
        if (j < G.bcnt) {
            const int2 e = blist ? blist[j] : make_int2(j, j);
            b = e.x;
            sb = e.y;
            const unsigned long long sv = (unsigned long long)bstrs[sb];
            for (int q = 0; q < G.nzb; ++q) {
                const bool odd = par(sv & zsb[q]);
#pragma unroll
                for (int rr = 0; rr < kListMaxRank; ++rr)
                    if (rr < R) pb[rr] += odd ? -wsb[rr * G.nzb + q] : wsb[rr * G.nzb + q];
            }
        }
        __syncthreads();
        if (b >= 0) {
#pragma unroll
            for (int k0 = 0; k0 < kBatchRows; k0 += 4) {
                double li[4], lj[4], ri[4], rj[4];
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    const int k = k0 + kk;
                    li[kk] = lj[kk] = ri[kk] = rj[kk] = 0.0;
                    if (arow[k] < 0) continue;
                    const i64 di = arow[k] + b, si = asrc[k] + sb;
                    li[kk] = __ldg(l + si); lj[kk] = __ldg(l + di);
                    ri[kk] = __ldg(r + si); rj[kk] = __ldg(r + di);
                }
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    const int k = k0 + kk;
                    if (arow[k] < 0) continue;
                    double vt = 0.0;
#pragma unroll
                    for (int rr = 0; rr < kListMaxRank; ++rr) vt += spa[k][rr] * pb[rr];
                    const double vd = ang0 * (vt * vt), vo = ang1 * vt;
                    acc += li[kk] * (ri[kk] * vd + rj[kk] * vo) + lj[kk] * (rj[kk] * vd - ri[kk] * vo);
                }
            }
        }
    }
    flush();
}

}  // namespace

template <typename Ti, int OP>
int pair_list_launch(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, PairAngles ang, double *l, double *r,
                     double *part, unsigned long long *ticket, i64 max_slots, double *out, bool accumulate,
                     cudaStream_t s, bool *used, bool may_build)
{
    *used = false;
    PairPlan<Ti> *P = nullptr;
    if (may_build) {
        int st = get_pair_plan(B, N, &P);
        if (st != BSIM_OK) return st;
    } else if (!(P = find_pair_plan(B, N))) {
        return BSIM_OK;   // no plan yet: the row kernel serves the call
    }
    const GroupDev &G = N->groups[gidx];
    if (!P->ok || G.rank > kListMaxRank || G.nza > kListMaxZ || G.nzb > kListMaxZ) return BSIM_OK;
    const int4 d = P->desc[gidx];
    *used = true;
    if (G.type == 0 || d.y == 0 || d.w == 0) {   // nothing to rotate; grad/backgrad still define the output
        if (OP != kPairExpm && !accumulate) BSIM_CUDA(cudaMemsetAsync(out, 0, sizeof(double), s));
        return BSIM_OK;
    }
    ListArgs A{B->nb[0], d.y, d.w, G.rank, G.nza, G.nzb, d.x >= 0 ? P->d_alist + d.x : nullptr,
               d.z >= 0 ? P->d_blist + d.z : nullptr, G.za_off, G.zb_off, G.wa_off, G.wb_off};
    // 32 alpha entries per tile (per pair of barriers), the loads of each group
    // of 4 pairs issued before their stores, 3 CTAs per SM
    constexpr int kRT = 32;
    const i64 cap = OP == kPairExpm ? (i64)148 * 64 : std::max<i64>(1, max_slots);
    const i64 tiles = (i64)((d.y + kRT - 1) / kRT) * ((d.w + kListCols - 1) / kListCols);
    const unsigned grid = (unsigned)std::min<i64>(tiles, cap);
    pair_list_kernel<Ti, OP, kRT, 4, 3><<<grid, kListCols, 0, s>>>(B->view.astrs, B->view.bstrs, N->view.z,
                                                                      N->view.w, A, ang, l, r, part, ticket, out,
                                                                      accumulate ? 1 : 0);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename Ti>
int pair_list_batchgrad(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *thetas, const double *l,
                        const double *r, double *grads, cudaStream_t s, bool *used, const unsigned char *skip,
                        const int *flag)
{
    *used = false;
    PairPlan<Ti> *P = nullptr;
    int st = get_pair_plan(B, N, &P);
    if (st != BSIM_OK) return st;
    if (!P->ok) return BSIM_OK;
    if (P->bg_state == 0) {
        std::vector<BGroup> bg;
        std::vector<i64> ts(1, 0);
        P->bg_state = 1;
        for (i64 g = 0; g < N->ngs; ++g) {
            const GroupDev &Gd = N->groups[g];
            if (Gd.type == 0) continue;   // diagonal groups contribute zero for real vectors
            if (Gd.rank > kListMaxRank || Gd.nza > kListMaxZ || Gd.nzb > kListMaxZ) { P->bg_state = -1; break; }
            const int4 d = P->desc[g];
            if (d.y == 0 || d.w == 0) continue;
            BGroup x{d.x, d.y, d.z, d.w, Gd.rank, Gd.nza, Gd.nzb, (int)g, (d.y + kBatchRows - 1) / kBatchRows, 0,
                     Gd.za_off, Gd.zb_off, Gd.wa_off, Gd.wb_off};
            bg.push_back(x);
            ts.push_back(ts.back() + (i64)x.ntx * ((d.w + kListCols - 1) / kListCols));
        }
        if (P->bg_state == 1 && !bg.empty()) {
            ts.push_back(ts.back());   // sentinel: tstart[n + 1] for the last group's boundary test
            BSIM_CUDA(dmalloc(&P->d_bg, bg.size() * sizeof(BGroup)));
            BSIM_CUDA(dmalloc(&P->d_tstart, ts.size() * sizeof(i64)));
            BSIM_CUDA(cudaMemcpy(P->d_bg, bg.data(), bg.size() * sizeof(BGroup), cudaMemcpyHostToDevice));
            BSIM_CUDA(cudaMemcpy(P->d_tstart, ts.data(), ts.size() * sizeof(i64), cudaMemcpyHostToDevice));
            P->bg_n = (int)bg.size();
            P->bg_tiles = ts[bg.size()];
        }
    }
    if (P->bg_state < 0) return BSIM_OK;
    *used = true;
    BSIM_CUDA(cudaMemsetAsync(grads, 0, sizeof(double) * N->ngs, s));
    if (P->bg_n == 0 || P->bg_tiles == 0) return BSIM_OK;
    const i64 grid = std::min<i64>(P->bg_tiles, (i64)148 * 32);
    pair_list_batchgrad_kernel<Ti><<<(unsigned)grid, kListCols, 0, s>>>(
        B->view.astrs, B->view.bstrs, B->nb[0], N->view.z, N->view.w, P->d_alist, P->d_blist, P->d_bg, P->d_tstart,
        P->bg_n, P->bg_tiles, thetas, l, r, grads, skip, flag);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template int pair_list_batchgrad<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, const double *,
                                           const double *, const double *, double *, cudaStream_t, bool *,
                                           const unsigned char *, const int *);
template int pair_list_batchgrad<unsigned long long>(const DevBasis<unsigned long long> *,
                                                     const DevNet<unsigned long long> *, const double *,
                                                     const double *, const double *, double *, cudaStream_t, bool *,
                                                     const unsigned char *, const int *);

#define PAIR_LIST_INST(OP)                                                                                   \
    template int pair_list_launch<unsigned, OP>(const DevBasis<unsigned> *, const DevNet<unsigned> *, i64,     \
                                                PairAngles, double *, double *, double *, unsigned long long *, \
                                                i64, double *, bool, cudaStream_t, bool *, bool);
#define PAIR_LIST_INST64(OP)                                                                                 \
    template int pair_list_launch<unsigned long long, OP>(const DevBasis<unsigned long long> *,                 \
                                                          const DevNet<unsigned long long> *, i64, PairAngles,  \
                                                          double *, double *, double *, unsigned long long *,   \
                                                          i64, double *, bool, cudaStream_t, bool *, bool);
PAIR_LIST_INST(kPairExpm)
PAIR_LIST_INST(kPairGrad)
PAIR_LIST_INST(kPairBackgrad)
PAIR_LIST_INST64(kPairExpm)
PAIR_LIST_INST64(kPairGrad)
PAIR_LIST_INST64(kPairBackgrad)

}  // namespace bsim
