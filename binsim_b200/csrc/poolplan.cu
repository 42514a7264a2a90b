// Pool-gradient plan (host): recognises every group of a generator network as
// lam * (t - t^dagger) for one spin-orbital excitation t with at most two
// creators and two annihilators, the form of every pool component of
// jl/adapt.jl's generator pools (jl/network.jl:248-301 builds one group per
// component).  With that form the pool gradient at theta = 0
// (op/batchgrad.hpp:529-540, every theta zero) of all groups follows from five
// transition-density tables of the frame vectors l~ = eps l, r~ = eps r
// (eps(a, b) = (-1)^popc(b & K(a)), the interleaved -> alpha-first sign of the
// structured sigma):
//   D1a[p][q]       = <l~| a+_p a_q (alpha)            |r~>
//   D1b[p][q]       = <l~| a+_p a_q (beta)             |r~>
//   Tab[p][q][r][s] = <l~| a+_p a_q (alpha) a+_r a_s (beta) |r~>
//   Gaa[p][q][r][s] = <l~| a+_p a+_q a_r a_s (alpha)   |r~>
//   Gbb[p][q][r][s] = <l~| a+_p a+_q a_r a_s (beta)    |r~>
// and grad_g = coef_g * (X[dagger(idx_g)] - X[idx_g]) in batch_grad's
// orientation, X the table of the group's kind.
//
// Recognition uses only the network arrays: the group's Pauli sum
// sum_ij (wa wb^T)_ij X^x Z^{za_i (+) zb_j} (interleaved masks) is compared
// with the Jordan-Wigner expansion of each candidate excitation whose modes
// are the flipped modes (bits of x) plus the modes whose Z varies between
// terms and is not flipped (number modes).  Groups that match no candidate
// are reported as kind -1 and keep the pair-list gradient.
#include "../../include/binsim_cuotf.h"
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

namespace bsim {

namespace {

typedef unsigned __int128 u128;

struct Term {
    u128 x, z;
    double c;
};

inline int popc128(u128 v) { return __builtin_popcountll((u64)v) + __builtin_popcountll((u64)(v >> 64)); }

inline u128 interleave(u64 a, u64 b, int norb)
{
    u128 r = 0;
    for (int i = 0; i < norb; ++i) {
        if ((a >> i) & 1) r |= (u128)1 << (2 * i);
        if ((b >> i) & 1) r |= (u128)1 << (2 * i + 1);
    }
    return r;
}

bool term_less(const Term &u, const Term &v) { return u.x != v.x ? u.x < v.x : u.z < v.z; }

// Sums equal (x, z), drops |c| <= tol, sorted by (x, z).
void combine(std::vector<Term> &t, double tol)
{
    std::sort(t.begin(), t.end(), term_less);
    std::vector<Term> out;
    for (const Term &u : t) {
        if (!out.empty() && out.back().x == u.x && out.back().z == u.z) out.back().c += u.c;
        else out.push_back(u);
    }
    t.clear();
    for (const Term &u : out)
        if (std::fabs(u.c) > tol) t.push_back(u);
}

// Jordan-Wigner expansion of a product of ladder operators (leftmost first):
// each factor is 1/2 X_j Z^{below j} (+/-) 1/2 X_j Z^{below j | j} (+ for a
// creator), multiplied as X^x Z^z * X^e Z^w = (-1)^popc(z & e) X^(x^e) Z^(z^w).
void ladder_terms(const int *modes, const bool *cre, int k, double scale, std::vector<Term> &out)
{
    std::vector<Term> t{{0, 0, scale}};
    for (int i = 0; i < k; ++i) {
        const u128 e = (u128)1 << modes[i], m = e - 1;
        std::vector<Term> nt;
        nt.reserve(t.size() * 2);
        for (const Term &u : t) {
            const double flip = (popc128(u.z & e) & 1) ? -0.5 : 0.5;
            nt.push_back({u.x ^ e, u.z ^ m, u.c * flip});
            nt.push_back({u.x ^ e, u.z ^ (m | e), u.c * flip * (cre[i] ? 1.0 : -1.0)});
        }
        t.swap(nt);
    }
    out.insert(out.end(), t.begin(), t.end());
}

// Pauli terms of t - t^dagger, t = a+_{cre[0]} .. a_{ann[0]} ..
void generator_terms(const std::vector<int> &cre, const std::vector<int> &ann, std::vector<Term> &out)
{
    std::vector<int> m;
    std::vector<char> d;
    for (int c : cre) { m.push_back(c); d.push_back(1); }
    for (int a : ann) { m.push_back(a); d.push_back(0); }
    const int k = (int)m.size();
    bool dg[8], dd[8];
    int md[8];
    for (int i = 0; i < k; ++i) {
        dg[i] = d[i];
        md[i] = m[k - 1 - i];
        dd[i] = !d[k - 1 - i];
    }
    out.clear();
    ladder_terms(m.data(), dg, k, 1.0, out);
    ladder_terms(md, dd, k, -1.0, out);
    combine(out, 1e-14);
}

// lam with group == lam * cand on every term (relative tolerance), or 0.
double match(const std::vector<Term> &grp, const std::vector<Term> &cand, double cmax)
{
    if (grp.size() != cand.size() || cand.empty()) return 0.0;
    size_t k0 = 0;
    for (size_t i = 1; i < cand.size(); ++i)
        if (std::fabs(cand[i].c) > std::fabs(cand[k0].c)) k0 = i;
    for (size_t i = 0; i < grp.size(); ++i)
        if (grp[i].x != cand[i].x || grp[i].z != cand[i].z) return 0.0;
    const double lam = grp[k0].c / cand[k0].c;
    for (size_t i = 0; i < grp.size(); ++i)
        if (std::fabs(grp[i].c - lam * cand[i].c) > 1e-9 * cmax) return 0.0;
    return lam;
}

struct Plan {
    int kind = -1;
    int idx[4] = {0, 0, 0, 0};
    double coef = 0.0;
};

// Alpha-first normal form of t (creators then annihilators, spin orbital
// 2p + s): sign of the reordering that moves every alpha operator before
// every beta operator (keeping each spin's order), and the table kind/indices.
bool normal_form(const std::vector<int> &cre, const std::vector<int> &ann, double lam, Plan &P)
{
    std::vector<int> m(cre);
    m.insert(m.end(), ann.begin(), ann.end());
    std::vector<char> dg(cre.size(), 1);
    dg.insert(dg.end(), ann.size(), 0);
    int inv = 0;
    for (size_t i = 0; i < m.size(); ++i)
        for (size_t j = i + 1; j < m.size(); ++j)
            if ((m[i] & 1) && !(m[j] & 1)) ++inv;
    std::vector<int> oa, ob;
    std::vector<char> da, db;
    for (size_t i = 0; i < m.size(); ++i) {
        if (m[i] & 1) { ob.push_back(m[i] >> 1); db.push_back(dg[i]); }
        else { oa.push_back(m[i] >> 1); da.push_back(dg[i]); }
    }
    auto shape_ok = [](const std::vector<char> &d) {   // creators first, as many as annihilators
        const size_t h = d.size() / 2;
        if (d.size() % 2) return false;
        for (size_t i = 0; i < d.size(); ++i)
            if ((i < h) != (bool)d[i]) return false;
        return true;
    };
    if (!shape_ok(da) || !shape_ok(db)) return false;
    const size_t na = oa.size(), nb = ob.size();
    if (na == 2 && nb == 0) { P.kind = BSIM_POOL_D1A; P.idx[0] = oa[0]; P.idx[1] = oa[1]; }
    else if (na == 0 && nb == 2) { P.kind = BSIM_POOL_D1B; P.idx[0] = ob[0]; P.idx[1] = ob[1]; }
    else if (na == 2 && nb == 2) {
        P.kind = BSIM_POOL_TAB;
        P.idx[0] = oa[0]; P.idx[1] = oa[1]; P.idx[2] = ob[0]; P.idx[3] = ob[1];
    } else if (na == 4 && nb == 0) {
        P.kind = BSIM_POOL_GAA;
        for (int i = 0; i < 4; ++i) P.idx[i] = oa[i];
    } else if (na == 0 && nb == 4) {
        P.kind = BSIM_POOL_GBB;
        for (int i = 0; i < 4; ++i) P.idx[i] = ob[i];
    } else {
        return false;
    }
    P.coef = (inv & 1) ? -lam : lam;
    return true;
}

Plan classify(int norb, u64 ax, u64 bx, int rank, int nza, int nzb, const u64 *za, const u64 *zb,
              const double *wa, const double *wb)
{
    Plan P;
    // the group's Pauli sum
    std::vector<Term> g;
    double cmax = 0.0;
    const u128 x = interleave(ax, bx, norb);
    for (int i = 0; i < nza; ++i)
        for (int j = 0; j < nzb; ++j) {
            double c = 0.0;
            for (int k = 0; k < rank; ++k) c += wa[(size_t)k * nza + i] * wb[(size_t)k * nzb + j];
            g.push_back({x, interleave(za[i], zb[j], norb), c});
            cmax = std::max(cmax, std::fabs(c));
        }
    if (x == 0 || cmax == 0.0) {   // diagonal or empty: zero gradient for real vectors
        P.kind = BSIM_POOL_ZERO;
        return P;
    }
    combine(g, 1e-10 * cmax);
    if (g.empty()) { P.kind = BSIM_POOL_ZERO; return P; }
    u128 vary = 0;
    for (const Term &u : g) vary |= u.z ^ g[0].z;
    const u128 num = vary & ~x;
    std::vector<int> flip, nm;
    for (int b = 0; b < 2 * norb; ++b) {
        if ((x >> b) & 1) flip.push_back(b);
        if ((num >> b) & 1) nm.push_back(b);
    }
    std::vector<std::pair<std::vector<int>, std::vector<int>>> cands;
    if (flip.size() == 2 && nm.empty()) {
        cands.push_back({{flip[1]}, {flip[0]}});
    } else if (flip.size() == 2 && nm.size() == 1) {
        cands.push_back({{flip[1], nm[0]}, {nm[0], flip[0]}});
    } else if (flip.size() == 4 && nm.empty()) {
        const int f0 = flip[0], f1 = flip[1], f2 = flip[2], f3 = flip[3];
        cands.push_back({{f3, f2}, {f1, f0}});
        cands.push_back({{f3, f1}, {f2, f0}});
        cands.push_back({{f3, f0}, {f2, f1}});
    }
    std::vector<Term> ct;
    for (const auto &c : cands) {
        generator_terms(c.first, c.second, ct);
        const double lam = match(g, ct, cmax);
        if (lam != 0.0) {
            Plan Q;
            if (normal_form(c.first, c.second, lam, Q)) return Q;
            return P;
        }
    }
    return P;
}

}  // namespace

}  // namespace bsim

extern "C" {

int bsim_poolplan_classify(int64_t norb, int64_t ngs, const uint64_t *axs, const uint64_t *bxs,
                           const int64_t *ranks, const int64_t *num_zas, const int64_t *num_zbs,
                           const uint64_t *flat_zas, const uint64_t *flat_zbs, const double *flat_wa,
                           const double *flat_wb, int32_t *kind, int32_t *idx, double *coef)
{
    if (ngs < 0 || norb < 1 || norb > 64) return bsim::BSIM_ERR_ARG;
    if (ngs == 0) return bsim::BSIM_OK;
    if (!axs || !bxs || !ranks || !num_zas || !num_zbs || !flat_zas || !flat_zbs || !flat_wa || !flat_wb ||
        !kind || !idx || !coef)
        return bsim::BSIM_ERR_NULL;
    std::vector<int64_t> oza(ngs + 1, 0), ozb(ngs + 1, 0), owa(ngs + 1, 0), owb(ngs + 1, 0);
    for (int64_t g = 0; g < ngs; ++g) {
        if (ranks[g] < 0 || num_zas[g] < 0 || num_zbs[g] < 0) return bsim::BSIM_ERR_ARG;
        oza[g + 1] = oza[g] + num_zas[g];
        ozb[g + 1] = ozb[g] + num_zbs[g];
        owa[g + 1] = owa[g] + num_zas[g] * ranks[g];
        owb[g + 1] = owb[g] + num_zbs[g] * ranks[g];
    }
    const int nth = (int)std::max(1u, std::min(std::thread::hardware_concurrency(), 64u));
    auto work = [&](int t) {
        for (int64_t g = t; g < ngs; g += nth) {
            const bsim::Plan P = bsim::classify((int)norb, axs[g], bxs[g], (int)ranks[g], (int)num_zas[g],
                                                (int)num_zbs[g], reinterpret_cast<const bsim::u64 *>(flat_zas) + oza[g],
                                                reinterpret_cast<const bsim::u64 *>(flat_zbs) + ozb[g],
                                                flat_wa + owa[g], flat_wb + owb[g]);
            kind[g] = P.kind;
            for (int i = 0; i < 4; ++i) idx[4 * g + i] = P.idx[i];
            coef[g] = P.coef;
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nth; ++t) th.emplace_back(work, t);
    work(0);
    for (auto &t : th) t.join();
    return bsim::BSIM_OK;
}

}  // extern "C"
