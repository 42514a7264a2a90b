// Host-side construction of the structured sigma plan (see fastplan.h).
#include "fastplan.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <thread>
#include <unordered_map>

namespace bsim {

namespace {

inline int popc(u64 x) { return __builtin_popcountll(x); }

// Ma(bx): alpha orbitals with an odd number of bx bits strictly below them.
u64 mask_below_odd(u64 x, int norb)
{
    u64 m = 0;
    for (int i = 0; i < norb; ++i)
        if (popc(x & ((1ull << i) - 1)) & 1) m |= 1ull << i;
    return m;
}

// Mb(ax): beta orbitals with an odd number of ax bits strictly above them.
u64 mask_above_odd(u64 x, int norb)
{
    u64 m = 0;
    for (int j = 0; j < norb; ++j)
        if (popc(x >> (j + 1)) & 1) m |= 1ull << j;
    return m;
}

template <typename Ti>
double phase_r(u64 s, const Ti *z, int nz, const double *w, int r, u64 zxor)
{
    const double *wr = w + (i64)r * nz;
    double v = 0.0;
    for (int k = 0; k < nz; ++k) v += (popc(s & ((u64)z[k] ^ zxor)) & 1) ? -wr[k] : wr[k];
    return v;
}

u64 comb_count(int n, int k)
{
    if (k < 0 || k > n) return 0;
    u64 r = 1;
    for (int i = 1; i <= k; ++i) r = r * (u64)(n - k + i) / (u64)i;
    return r;
}

// String -> index of one spin's list: a dense table up to 24 orbitals, above
// that the colex rank of the string (Gosper order) indexing a table of
// C(norb, n) entries; -1 for strings outside the list.
struct StrIndex {
    int norb = 0, nel = 0;
    bool ranked = false;
    std::vector<int> tab;
    std::vector<u64> binom;   // [65 x 65]
    template <typename Ti>
    void build(int norb_, const std::vector<Ti> &strs)
    {
        norb = norb_;
        nel = strs.empty() ? 0 : popc((u64)strs[0]);
        ranked = norb > 24;
        binom.assign(65 * 65, 0);
        for (int n = 0; n <= 64; ++n) {
            binom[n * 65] = 1;
            for (int k = 1; k <= n; ++k) binom[n * 65 + k] = binom[(n - 1) * 65 + k - 1] + (k <= n - 1 ? binom[(n - 1) * 65 + k] : 0);
        }
        tab.assign(ranked ? (size_t)binom[norb * 65 + nel] : (size_t)1 << norb, -1);
        for (size_t i = 0; i < strs.size(); ++i) tab[slot((u64)strs[i])] = (int)i;
    }
    size_t slot(u64 s) const
    {
        if (!ranked) return (size_t)s;
        u64 r = 0;
        int i = 1;
        for (u64 y = s; y; y &= y - 1, ++i) r += binom[__builtin_ctzll(y) * 65 + i];
        return (size_t)r;
    }
    int operator()(u64 s) const
    {
        if (norb < 64 && (s >> norb)) return -1;
        if (ranked && popc(s) != nel) return -1;
        return tab[slot(s)];
    }
};

}  // namespace

template <typename Ti>
int build_fast_plan(const DevBasis<Ti> *B, const DevNet<Ti> *N, FastPlan<Ti> *P)
{
    P->ok = false;
    P->basis = B;
    P->basis_dim = B->dim;
    if (B->num_blocks != 1) { P->why = "more than one symmetry block"; return BSIM_OK; }
    const int norb = B->norb;
    const int nA = B->na[0], nB = B->nb[0];
    const auto &A = B->astrs;
    const auto &Bs = B->bstrs;
    const int nelA = popc((u64)A[0]), nelB = popc((u64)Bs[0]);
    if ((u64)nA != comb_count(norb, nelA) || (u64)nB != comb_count(norb, nelB)) {
        P->why = "string lists are not complete (symmetry-restricted)";
        return BSIM_OK;
    }
    if (norb > 63) { P->why = "norb > 63"; return BSIM_OK; }
    P->norb = norb; P->nA = nA; P->nB = nB; P->nelA = nelA; P->nelB = nelB;
    P->ldA = (nB + 7) & ~7;
    P->ldB = (nA + 7) & ~7;
    P->ldG = (nB + kMixCols - 1) / kMixCols * kMixCols;
    P->Ka.resize(nA);
    for (int a = 0; a < nA; ++a) {
        u64 k = 0, s = (u64)A[a];
        for (int i = 0; i < norb; ++i)
            if ((s >> i) & 1u) k ^= (1ull << i) - 1;
        P->Ka[a] = k;
    }

    const Ti *z = N->z.data();
    const double *w = N->w.data();
    std::vector<int> diag, pa, pb, mixed;
    for (i64 g = 0; g < N->ngs; ++g) {
        const GroupDev &G = N->groups[g];
        if (G.rank == 0) continue;
        if (G.type == 0) (diag.empty() ? diag : P->residual).push_back((int)g);
        else if (G.type == 1) (G.rank <= kSideMaxRank ? pa : P->residual).push_back((int)g);
        else if (G.type == 2) (G.rank <= kSideMaxRank ? pb : P->residual).push_back((int)g);
        else mixed.push_back((int)g);
    }

    // ---- diagonal tables --------------------------------------------------------
    std::vector<double> PAd, PBd;
    if (!diag.empty()) {
        const GroupDev &G = N->groups[diag[0]];
        P->rank_d = G.rank;
        PAd.resize((size_t)nA * G.rank);
        PBd.assign((size_t)G.rank * P->ldA, 0.0);
        for (int a = 0; a < nA; ++a)
            for (int r = 0; r < G.rank; ++r) PAd[(size_t)a * G.rank + r] = phase_r(A[a], z + G.za_off, G.nza, w + G.wa_off, r, 0);
        for (int b = 0; b < nB; ++b)
            for (int r = 0; r < G.rank; ++r) PBd[(size_t)r * P->ldA + b] = phase_r(Bs[b], z + G.zb_off, G.nzb, w + G.wb_off, r, 0);
    }

    // ---- pure sides: row-spin data + column factor in the alpha-first frame -----
    struct SideHost {
        std::vector<u64> x, zmask;
        std::vector<int> rank, nz, colmode;
        std::vector<i64> z_off, w_off, ctab_off;
        std::vector<double> wv, cconst, ctab;
    } sh[2];
    auto add_side = [&](int side, const std::vector<int> &gl) {
        SideHost &S = sh[side];
        const auto &colstr = side == 0 ? Bs : A;
        const int ncol = side == 0 ? nB : nA;
        const int ld = side == 0 ? P->ldA : P->ldB;
        for (int g : gl) {
            const GroupDev &G = N->groups[g];
            const u64 rowx = side == 0 ? G.ax : G.bx;
            const Ti *rz = z + (side == 0 ? G.za_off : G.zb_off);
            const int rnz = side == 0 ? G.nza : G.nzb;
            const double *rw = w + (side == 0 ? G.wa_off : G.wb_off);
            const Ti *cz = z + (side == 0 ? G.zb_off : G.za_off);
            const int cnz = side == 0 ? G.nzb : G.nza;
            const double *cw = w + (side == 0 ? G.wb_off : G.wa_off);
            // the frame flips the column factor by (-1)^{popc(col & M)}
            const u64 cm = side == 0 ? mask_above_odd(rowx, norb) : mask_below_odd(rowx, norb);
            std::vector<double> col((size_t)G.rank * ncol);
            bool constant = true;
            for (int r = 0; r < G.rank; ++r)
                for (int c = 0; c < ncol; ++c) {
                    double v = phase_r((u64)colstr[c], cz, cnz, cw, r, cm);
                    col[(size_t)r * ncol + c] = v;
                    if (std::fabs(v - col[(size_t)r * ncol]) > 1e-13 * std::max(1.0, std::fabs(col[(size_t)r * ncol])))
                        constant = false;
                }
            S.x.push_back(rowx);
            S.rank.push_back(G.rank);
            S.nz.push_back(rnz);
            S.z_off.push_back((i64)S.zmask.size());
            for (int k = 0; k < rnz; ++k) S.zmask.push_back((u64)rz[k]);
            S.w_off.push_back((i64)S.wv.size());
            S.wv.insert(S.wv.end(), rw, rw + (i64)rnz * G.rank);
            for (int r = 0; r < kSideMaxRank; ++r) S.cconst.push_back(r < G.rank ? col[(size_t)r * ncol] : 0.0);
            S.colmode.push_back(constant ? 0 : 1);
            S.ctab_off.push_back(constant ? -1 : (i64)S.ctab.size());
            if (!constant)
                for (int r = 0; r < G.rank; ++r) {
                    S.ctab.insert(S.ctab.end(), col.begin() + (size_t)r * ncol, col.begin() + (size_t)(r + 1) * ncol);
                    S.ctab.resize(S.ctab.size() + (ld - ncol), 0.0);
                }
        }
    };
    add_side(0, pa);
    add_side(1, pb);
    StrIndex amap, bmap;
    amap.build(norb, A);
    bmap.build(norb, Bs);
    const int nth_host = std::max(1, std::min(16, (int)std::thread::hardware_concurrency()));

    // ---- same-spin doubles through intermediate strings: extract and verify W ----
    const int nP = norb * (norb - 1) / 2;
    auto pair_id = [norb](int p, int q) { return p * (2 * norb - p - 1) / 2 + (q - p - 1); };
    auto spair = [](u64 m, int p, int q) { return (popc(m & ((1ull << p) - 1)) + popc(m & ((1ull << q) - 1))) & 1; };
    // which 2 of the 4 bits of x form pq, as a 4-bit pattern (one slot per split)
    auto split_id = [](u64 x, u64 pq) {
        int id = 0, k = 0;
        for (u64 y = x; y; y &= y - 1, ++k)
            if (pq & (y & (~y + 1))) id |= 1 << k;
        return id;
    };
    std::vector<char> ri_grp[2];
    std::vector<double> Wri[2];
    bool ri_on[2] = {false, false};
    for (int side = 0; side < 2; ++side) {
        const SideHost &S = sh[side];
        const int ng = (int)S.x.size();
        const int nel = side == 0 ? nelA : nelB;
        const int nU = (int)comb_count(norb - nel + 2, 2), npr = (int)comb_count(nel, 2);
        ri_grp[side].assign(ng, 0);
        const char *ri_env = getenv("BSIM_SIGMA_RI");   // BSIM_SIGMA_RI=0 keeps these groups in the row lists
        if (nel < 2 || norb - nel < 2 || nU > kRiMaxU || npr > 64 || (ri_env && ri_env[0] == '0')) continue;
        Wri[side].assign((size_t)nP * nP, 0.0);
        const auto &rows = side == 0 ? A : Bs;
        const StrIndex &rmap = side == 0 ? amap : bmap;
        const int nrows = side == 0 ? nA : nB;
        std::vector<int> cand;
        for (int g = 0; g < ng; ++g)
            if (popc(S.x[g]) == 4 && S.colmode[g] == 0) cand.push_back(g);
        auto work = [&](int t) {
            for (size_t ci = t; ci < cand.size(); ci += nth_host) {
                const int g = cand[ci];
                const u64 x = S.x[g];
                const int R = S.rank[g], nz = S.nz[g];
                double wv[16];
                bool have[16] = {false};
                bool ok = true;
                for (int r = 0; r < nrows && ok; ++r) {
                    const u64 d = (u64)rows[r];
                    if (popc(d & x) != 2) continue;
                    const u64 sv = d ^ x;
                    if (rmap(sv) < 0) { ok = false; break; }
                    double pa[kSideMaxRank] = {0, 0, 0, 0};
                    for (int q = 0; q < nz; ++q) {
                        const bool odd = popc(sv & S.zmask[S.z_off[g] + q]) & 1;
                        for (int rr = 0; rr < R; ++rr) {
                            const double v = S.wv[S.w_off[g] + (i64)rr * nz + q];
                            pa[rr] += odd ? -v : v;
                        }
                    }
                    double coef = 0.0;
                    for (int rr = 0; rr < R; ++rr) coef += pa[rr] * S.cconst[(size_t)g * kSideMaxRank + rr];
                    const u64 pq = d & x, rs = sv & x, m = d & ~x;
                    const int p = __builtin_ctzll(pq), q2 = 63 - __builtin_clzll(pq);
                    const int r1 = __builtin_ctzll(rs), s1 = 63 - __builtin_clzll(rs);
                    const double w = ((spair(m, p, q2) ^ spair(m, r1, s1)) ? -coef : coef);
                    const int id = split_id(x, pq);
                    if (!have[id]) { have[id] = true; wv[id] = w; }
                    else if (std::fabs(w - wv[id]) > 1e-12 * std::max(1.0, std::fabs(wv[id]))) ok = false;
                }
                if (!ok) continue;
                // record W for every split seen (each split maps to its own (pq, rs) entry)
                for (int r = 0; r < nrows; ++r) {
                    const u64 d = (u64)rows[r];
                    if (popc(d & x) != 2) continue;
                    const u64 pq = d & x, rs = (d ^ x) & x;
                    const int id = split_id(x, pq);
                    const int p = __builtin_ctzll(pq), q2 = 63 - __builtin_clzll(pq);
                    const int r1 = __builtin_ctzll(rs), s1 = 63 - __builtin_clzll(rs);
                    Wri[side][(size_t)pair_id(p, q2) * nP + pair_id(r1, s1)] = wv[id];
                }
                ri_grp[side][g] = 1;
            }
        };
        std::vector<std::thread> th;
        for (int t = 1; t < nth_host; ++t) th.emplace_back(work, t);
        work(0);
        for (auto &t : th) t.join();
        for (int g = 0; g < ng; ++g) ri_on[side] = ri_on[side] || ri_grp[side][g];
    }

    // per-row contribution lists (CSR), built with a few host threads: alpha
    // (without the intermediate-string groups when that side uses them), beta
    // with every group (column bands), beta without them (whole sigma)
    struct CSRHost {
        std::vector<i64> cptr, tptr;
        std::vector<CEnt> cent;
        std::vector<TEnt> tent;
    } csr[3];
    {
        for (int li = 0; li < 3; ++li) {
            const int side = li == 0 ? 0 : 1;
            const bool skip_ri = li == 0 ? ri_on[0] : (li == 2);
            if (li == 2 && !ri_on[1]) continue;
            const SideHost &S = sh[side];
            const auto &rows = side == 0 ? A : Bs;
            const StrIndex &rmap = side == 0 ? amap : bmap;
            const int nrows = side == 0 ? nA : nB;
            const int ng = (int)S.x.size();
            const int nth = std::max(1, std::min(16, (int)std::thread::hardware_concurrency()));
            const i64 ld_in = side == 0 ? P->ldA : P->ldB;
            struct Part {
                std::vector<i64> cn, tn;
                std::vector<CEnt> cent;
                std::vector<TEnt> tent;
            };
            std::vector<Part> parts(nth);
            auto work = [&](int t) {
                Part &pt = parts[t];
                const int r0 = (int)((i64)nrows * t / nth), r1 = (int)((i64)nrows * (t + 1) / nth);
                for (int r = r0; r < r1; ++r) {
                    const u64 s0 = (u64)rows[r];
                    i64 cc = 0, tc = 0;
                    for (int g = 0; g < ng; ++g) {
                        if (skip_ri && ri_grp[side][g]) continue;
                        const u64 x = S.x[g];
                        if (2 * popc(s0 & x) != popc(x)) continue;
                        const u64 sv = s0 ^ x;
                        if (sv >> norb) continue;
                        const int src = rmap(sv);
                        if (src < 0) continue;
                        double pa[kSideMaxRank] = {0, 0, 0, 0};
                        const int R = S.rank[g], nz = S.nz[g];
                        for (int q = 0; q < nz; ++q) {
                            const bool odd = popc(sv & S.zmask[S.z_off[g] + q]) & 1;
                            for (int rr = 0; rr < R; ++rr) {
                                const double v = S.wv[S.w_off[g] + (i64)rr * nz + q];
                                pa[rr] += odd ? -v : v;
                            }
                        }
                        if (S.colmode[g] == 0) {
                            double coef = 0.0;
                            for (int rr = 0; rr < R; ++rr) coef += pa[rr] * S.cconst[(size_t)g * kSideMaxRank + rr];
                            pt.cent.push_back(CEnt{(long long)src * ld_in, coef});
                            ++cc;
                        } else {
                            TEnt t{(long long)src * ld_in, (long long)S.ctab_off[g] | R, {0, 0, 0, 0}};
                            for (int rr = 0; rr < kSideMaxRank; ++rr) t.pa[rr] = pa[rr];
                            pt.tent.push_back(t);
                            ++tc;
                        }
                    }
                    pt.cn.push_back(cc);
                    pt.tn.push_back(tc);
                }
            };
            std::vector<std::thread> th;
            for (int t = 1; t < nth; ++t) th.emplace_back(work, t);
            work(0);
            for (auto &x : th) x.join();
            CSRHost &C = csr[li];
            C.cptr.assign(1, 0);
            C.tptr.assign(1, 0);
            for (auto &pt : parts) {
                for (i64 v : pt.cn) C.cptr.push_back(C.cptr.back() + v);
                for (i64 v : pt.tn) C.tptr.push_back(C.tptr.back() + v);
                C.cent.insert(C.cent.end(), pt.cent.begin(), pt.cent.end());
                C.tent.insert(C.tent.end(), pt.tent.begin(), pt.tent.end());
            }
        }
    }
    P->nnzA = (i64)csr[0].cent.size();
    P->nnzB = (i64)csr[1].cent.size();
    P->nPA = (int)pa.size();
    P->nPB = (int)pb.size();

    // ---- mixed single-single groups: Kronecker factorisation --------------------
    std::unordered_map<u64, int> eidx, fidx;
    struct MixedRec { int E, F; double coef; };
    std::vector<MixedRec> recs;
    std::vector<int> connA, connB;   // scratch: connected string indices
    for (int g : mixed) {
        const GroupDev &G = N->groups[g];
        if (G.rank != 1 || popc(G.ax) != 2 || popc(G.bx) != 2) { P->residual.push_back(g); continue; }
        const u64 ma = mask_below_odd(G.bx, norb), mb = mask_above_odd(G.ax, norb);
        const double csign = (popc(G.ax & ma) & 1) ? -1.0 : 1.0;
        auto ei = eidx.find(G.ax);
        auto fi = fidx.find(G.bx);
        // sign masks of a new excitation: the first transformed Z mask of this group
        const u64 mA = ei == eidx.end() ? ((u64)z[G.za_off] ^ ma) : P->mA[ei->second];
        const u64 mB = fi == fidx.end() ? ((u64)z[G.zb_off] ^ mb) : P->mB[fi->second];
        // lam / mu from one connected string each, then verified on all of them
        auto factor = [&](const auto &strs, int n, u64 x, const Ti *zz, int nz, const double *ww, u64 zx, u64 sm,
                          double *out) {
            double f = 0.0;
            bool have = false;
            for (int i = 0; i < n; ++i) {
                const u64 s = (u64)strs[i];
                if (popc(s & x) != 1) continue;
                const double v = phase_r(s, zz, nz, ww, 0, zx);
                const double sg = (popc(s & sm) & 1) ? -1.0 : 1.0;
                if (!have) { f = v * sg; have = true; continue; }
                if (std::fabs(v - f * sg) > 1e-12 * std::max(1.0, std::fabs(f))) return false;
            }
            *out = f;
            return have;
        };
        double lam = 0.0, mu = 0.0;
        if (!factor(A, nA, G.ax, z + G.za_off, G.nza, w + G.wa_off, ma, mA, &lam) ||
            !factor(Bs, nB, G.bx, z + G.zb_off, G.nzb, w + G.wb_off, mb, mB, &mu)) {
            P->residual.push_back(g);
            continue;
        }
        int E, F;
        if (ei == eidx.end()) {
            E = (int)P->Emask.size();
            eidx[G.ax] = E;
            P->Emask.push_back(G.ax);
            P->mA.push_back(mA);
        } else E = ei->second;
        if (fi == fidx.end()) {
            F = (int)P->Fmask.size();
            fidx[G.bx] = F;
            P->Fmask.push_back(G.bx);
            P->mB.push_back(mB);
        } else F = fi->second;
        recs.push_back({E, F, csign * lam * mu});
        P->mixed_pairs += 0;
    }
    P->nE = (int)P->Emask.size();
    P->nF = (int)P->Fmask.size();
    if (P->nE > 4096 || P->nF > 4096) {
        // too many excitations for the shared-memory tiles: everything generic
        for (auto &r : recs) (void)r;
        P->why = "too many single excitations for the structured mixed kernel";
        return BSIM_OK;
    }
    P->Lam.assign((size_t)P->nE * P->nF, 0.0);
    for (auto &r : recs) P->Lam[(size_t)r.E * P->nF + r.F] += r.coef;
    // M: connected alpha singles per source row (max over rows)
    int M = 0;
    for (int a = 0; a < nA; ++a) {
        int m = 0;
        for (int e = 0; e < P->nE; ++e) m += popc((u64)A[a] & P->Emask[e]) == 1;
        M = std::max(M, m);
    }
    P->M = M;
    if (M > kMaxConn && P->nE > 0) { P->why = "more than 128 connected alpha singles per string"; return BSIM_OK; }

    P->row64 = P->nE == 0 || !mixed_shape(nB, P->nF, 8, kSmemMax).grow;
    P->row32 = P->nE == 0 || !mixed_shape(nB, P->nF, 4, kSmemMax).grow;

    // ---- gather-index table of the mixed GEMM: X[F][b] = sB_F(b^F) c~[a', b^F] ------
    std::vector<int> gidx((size_t)P->nF * P->ldG, -1);
    {
        std::unordered_map<u64, int> bidx;
        bidx.reserve((size_t)nB * 2);
        for (int b = 0; b < nB; ++b) bidx[(u64)Bs[b]] = b;
        for (int f = 0; f < P->nF; ++f)
            for (int b = 0; b < nB; ++b) {
                const u64 s0 = (u64)Bs[b], fm = P->Fmask[f];
                if (popc(s0 & fm) != 1) continue;
                const u64 sv = s0 ^ fm;
                auto it = bidx.find(sv);
                if (it == bidx.end()) continue;
                gidx[(size_t)f * P->ldG + b] = (it->second << 1) | (popc(sv & P->mB[f]) & 1);
            }
    }

    // ---- intermediate-string tables ----------------------------------------------
    struct RIHost {
        int nM = 0, nU = 0, npr = 0;
        std::vector<int> src, pid;
        std::vector<int2> gath;
        std::vector<float> W32;
    } rih[2];
    for (int side = 0; side < 2; ++side) {
        if (!ri_on[side]) continue;
        RIHost &H = rih[side];
        const int nel = side == 0 ? nelA : nelB;
        const auto &rows = side == 0 ? A : Bs;
        const StrIndex &rmap = side == 0 ? amap : bmap;
        const int nrows = side == 0 ? nA : nB;
        H.nU = (int)comb_count(norb - nel + 2, 2);
        H.npr = (int)comb_count(nel, 2);
        // intermediates in colex order (Gosper), as the string lists
        std::vector<u64> Ms;
        std::unordered_map<u64, int> midx;
        const int k = nel - 2;
        if (k == 0) Ms.push_back(0);
        else
            for (u64 v = (1ull << k) - 1; v < (1ull << norb);) {
                Ms.push_back(v);
                const u64 t = v | (v - 1);
                v = (t + 1) | (((~t & (t + 1)) - 1) >> (__builtin_ctzll(v) + 1));
            }
        H.nM = (int)Ms.size();
        midx.reserve(Ms.size() * 2);
        for (int i = 0; i < H.nM; ++i) midx[Ms[i]] = i;
        H.src.assign((size_t)H.nM * H.nU, -1);
        H.pid.assign((size_t)H.nM * H.nU, 0);
        const u64 full = norb == 64 ? ~0ull : ((1ull << norb) - 1);
        for (int i = 0; i < H.nM; ++i) {
            const u64 m = Ms[i], comp = full & ~m;
            int slot = 0;
            for (u64 yp = comp; yp; yp &= yp - 1) {
                const int p = __builtin_ctzll(yp);
                for (u64 yq = yp & (yp - 1); yq; yq &= yq - 1) {
                    const int q = __builtin_ctzll(yq);
                    const int row = rmap(m | (1ull << p) | (1ull << q));
                    H.src[(size_t)i * H.nU + slot] = (row << 1) | spair(m, p, q);
                    H.pid[(size_t)i * H.nU + slot] = pair_id(p, q);
                    ++slot;
                }
            }
        }
        H.gath.assign((size_t)nrows * H.npr, make_int2(0, 0));
        for (int r = 0; r < nrows; ++r) {
            const u64 a = (u64)rows[r];
            int e = 0;
            for (u64 yp = a; yp; yp &= yp - 1) {
                const int p = __builtin_ctzll(yp);
                for (u64 yq = yp & (yp - 1); yq; yq &= yq - 1) {
                    const int q = __builtin_ctzll(yq);
                    const u64 m = a & ~((1ull << p) | (1ull << q));
                    const u64 comp = full & ~m;
                    const int pp = popc(comp & ((1ull << p) - 1)), qq = popc(comp & ((1ull << q) - 1));
                    const int nc = popc(comp);
                    const int slot = pp * (2 * nc - pp - 1) / 2 + (qq - pp - 1);
                    H.gath[(size_t)r * H.npr + e] = make_int2(midx[m] * H.nU + slot, spair(m, p, q));
                    ++e;
                }
            }
        }
        H.W32.assign(Wri[side].begin(), Wri[side].end());
    }

    // ---- upload -------------------------------------------------------------------
    auto bytes = [](size_t n, size_t sz) { return ((std::max<size_t>(n, 1) * sz) + 255) & ~size_t(255); };
    size_t tot = bytes(nA, sizeof(Ti)) + bytes(nB, sizeof(Ti)) + bytes(nA, 8) + bytes(PAd.size(), 8) +
                 bytes(PBd.size(), 8) + 2 * bytes(P->nE, 8) + 2 * bytes(P->Lam.size(), 8) + bytes(gidx.size(), 4) +
                 bytes(P->residual.size(), 4) + bytes(P->residual.size() + 1, 16);
    for (int li = 0; li < 3; ++li)
        tot += 2 * bytes(csr[li].cptr.size(), 8) + bytes(csr[li].cent.size(), sizeof(CEnt)) +
               bytes(csr[li].tent.size(), sizeof(TEnt)) + bytes(sh[li == 0 ? 0 : 1].ctab.size(), 8) +
               bytes(sh[li == 0 ? 0 : 1].ctab.size(), 4);
    for (int side = 0; side < 2; ++side)
        tot += 2 * bytes(rih[side].src.size(), 4) + bytes(rih[side].gath.size(), 8) + bytes(Wri[side].size(), 8) +
               bytes(rih[side].W32.size(), 4);
    int st = P->arena.reserve(tot);
    if (st != BSIM_OK) return st;
    auto put = [&](const auto &v) {
        using T = typename std::decay_t<decltype(v)>::value_type;
        T *d = P->arena.template take<T>(std::max<size_t>(v.size(), 1));
        if (!v.empty()) cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
        return (const T *)d;
    };
    P->d_astr = put(A);
    P->d_bstr = put(Bs);
    P->d_Ka = put(P->Ka);
    P->d_PAd = put(PAd);
    P->d_PBdT = put(PBd);
    P->d_Emask = put(P->Emask);
    P->d_mA = put(P->mA);
    P->d_Lam = put(P->Lam);
    std::vector<float> lam32(P->Lam.begin(), P->Lam.end());
    P->d_Lam32 = put(lam32);
    P->d_gidx = put(gidx);
    for (int li = 0; li < 3; ++li) {
        CSRHost &C = csr[li];
        if (li == 2 && !ri_on[1]) continue;
        SideCSR &D = li == 0 ? P->csrA : li == 1 ? P->csrB : P->csrBri;
        D.cptr = put(C.cptr);
        D.cent = put(C.cent);
        D.tptr = put(C.tptr);
        D.tent = put(C.tent);
        D.ctab = put(sh[li == 0 ? 0 : 1].ctab);
        D.ctab32 = put(std::vector<float>(sh[li == 0 ? 0 : 1].ctab.begin(), sh[li == 0 ? 0 : 1].ctab.end()));
    }
    for (int side = 0; side < 2; ++side) {
        RISide &R = side == 0 ? P->riA : P->riB;
        R = RISide{};
        if (!ri_on[side]) continue;
        const RIHost &H = rih[side];
        R.on = 1;
        R.nM = H.nM;
        R.nU = H.nU;
        R.npr = H.npr;
        R.nP = nP;
        R.src = put(H.src);
        R.pid = put(H.pid);
        R.gath = put(H.gath);
        R.W = put(Wri[side]);
        R.W32 = put(H.W32);
    }
    // residual groups through the generic tile kernel (chunks as in DevNet::finalize)
    std::vector<int> res = P->residual;
    std::stable_sort(res.begin(), res.end(), [&](int a, int b) {
        const GroupDev &x = N->groups[a], &y = N->groups[b];
        return x.type != y.type ? x.type < y.type : x.rank < y.rank;
    });
    std::vector<int4> ch;
    for (size_t i = 0; i < res.size();) {
        const int r = N->groups[res[i]].rank, ty = N->groups[res[i]].type;
        size_t j = i + 1;
        if (r <= 2)
            while (j < res.size() && j - i < 32 && N->groups[res[j]].rank == r && N->groups[res[j]].type == ty) ++j;
        ch.push_back(make_int4((int)i, (int)(j - i), r, ty));
        i = j;
    }
    P->d_resid = put(res);
    P->d_resid_chunks = put(ch);
    P->n_resid_chunks = (int)ch.size();
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_status(e, "fast plan upload");
    P->ok = true;
    return BSIM_OK;
}

template int build_fast_plan<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, FastPlan<unsigned> *);
template int build_fast_plan<unsigned long long>(const DevBasis<unsigned long long> *,
                                                 const DevNet<unsigned long long> *, FastPlan<unsigned long long> *);

}  // namespace bsim
