/*
 * otf_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, OpenMP restatement of BinSim's on-the-fly (OTF) operator path,
 * used by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline
 * leg as the CHECKER of the CUDA library.  The product (binsim_b200) never
 * links, loads or calls this file.
 *
 * Each function cites the reference file:line it restates (paths are relative
 * to the reference project root).  Strings are carried as uint64 so the same
 * code serves the uint32 and uint64 string types; arithmetic is IEEE double
 * without fast-math so results are deterministic given the loop order below.
 *
 * The restatement is pinned against the reference's own compiled CPU
 * libraries (oracle/_ref, built by oracle/Makefile) in tests/test_oracle_pin.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t i64;
typedef uint64_t u64;

/* ------------------------------------------------------------------ */
/* string helpers: core/types.hpp:61-86                                */
/* ------------------------------------------------------------------ */

/* get_string_sym, core/types.hpp:61-76: XOR of orbital irreps over set bits. */
static i64 string_sym(u64 s, const i64 *orbsym)
{
    i64 sym = 0;
    for (int pos = 0; s; ++pos, s >>= 1)
        if (s & 1u)
            sym ^= orbsym[pos];
    return sym;
}

/* next_combination (Gosper's hack), core/types.hpp:78-86. */
static u64 next_comb(u64 v)
{
    if (v == 0)
        return 0;
    u64 c = v & (~v + 1);
    u64 r = v + c;
    return (((r ^ v) >> 2) / c) | r;
}

static int parity64(u64 x) { return __builtin_popcountll(x) & 1; }

/* ------------------------------------------------------------------ */
/* basis: basis/basis.hpp:118-296 (create_basis_manager_tmpl)          */
/* ------------------------------------------------------------------ */

typedef struct {
    i64 norb, num_irreps, num_blocks, dim;
    i64 *blk_asym, *blk_bsym, *blk_na, *blk_nb, *blk_off;
    u64 **blk_astrs, **blk_bstrs;   /* views into irrep string lists */
    u64 *all_a, *all_b;             /* strings grouped by irrep, Gosper order inside */
    i64 *na_irrep, *nb_irrep, *a_start, *b_start;
    i64 *block_map;                 /* [num_irreps^2] -> block or -1 */
} OBasis;

static void enum_strings(i64 norb, i64 ne, const i64 *orbsym, i64 nirr,
                         i64 *count, u64 **out, i64 *start)
{
    /* Pass 1 counts per irrep, pass 2 fills (basis.hpp:135-231). */
    u64 first = (ne >= 64) ? ~0ull : ((1ull << ne) - 1);
    u64 lim = 1ull << norb;
    i64 total = 0;
    for (i64 i = 0; i < nirr; ++i) count[i] = 0;
    for (u64 s = first; s < lim;) {
        i64 sym = string_sym(s, orbsym);
        if (sym < nirr) { count[sym]++; total++; }
        if (ne == 0) break;
        s = next_comb(s);
    }
    *out = (u64 *)malloc(sizeof(u64) * (total > 0 ? total : 1));
    i64 off = 0;
    for (i64 i = 0; i < nirr; ++i) { start[i] = off; off += count[i]; }
    i64 *fill = (i64 *)calloc(nirr, sizeof(i64));
    for (u64 s = first; s < lim;) {
        i64 sym = string_sym(s, orbsym);
        if (sym < nirr) (*out)[start[sym] + fill[sym]++] = s;
        if (ne == 0) break;
        s = next_comb(s);
    }
    free(fill);
}

void *oracle_basis_create(i64 norb, i64 na, i64 nb, i64 total_sym,
                          const i64 *orbsym, i64 num_irreps)
{
    OBasis *B = (OBasis *)calloc(1, sizeof(OBasis));
    B->norb = norb;
    B->num_irreps = num_irreps;
    B->na_irrep = (i64 *)calloc(num_irreps, sizeof(i64));
    B->nb_irrep = (i64 *)calloc(num_irreps, sizeof(i64));
    B->a_start = (i64 *)calloc(num_irreps, sizeof(i64));
    B->b_start = (i64 *)calloc(num_irreps, sizeof(i64));
    enum_strings(norb, na, orbsym, num_irreps, B->na_irrep, &B->all_a, B->a_start);
    enum_strings(norb, nb, orbsym, num_irreps, B->nb_irrep, &B->all_b, B->b_start);

    /* blocks: asym ascending, bsym = total_sym ^ asym (basis.hpp:154-161, 233-259) */
    i64 nblk = 0;
    for (i64 as = 0; as < num_irreps; ++as) {
        i64 bs = total_sym ^ as;
        if (bs < num_irreps && B->na_irrep[as] > 0 && B->nb_irrep[bs] > 0) nblk++;
    }
    B->num_blocks = nblk;
    B->blk_asym = (i64 *)calloc(nblk + 1, sizeof(i64));
    B->blk_bsym = (i64 *)calloc(nblk + 1, sizeof(i64));
    B->blk_na = (i64 *)calloc(nblk + 1, sizeof(i64));
    B->blk_nb = (i64 *)calloc(nblk + 1, sizeof(i64));
    B->blk_off = (i64 *)calloc(nblk + 1, sizeof(i64));
    B->blk_astrs = (u64 **)calloc(nblk + 1, sizeof(u64 *));
    B->blk_bstrs = (u64 **)calloc(nblk + 1, sizeof(u64 *));
    B->block_map = (i64 *)malloc(sizeof(i64) * num_irreps * num_irreps);
    for (i64 i = 0; i < num_irreps * num_irreps; ++i) B->block_map[i] = -1;
    i64 k = 0, dim = 0;
    for (i64 as = 0; as < num_irreps; ++as) {
        i64 bs = total_sym ^ as;
        if (bs >= num_irreps) continue;
        if (B->na_irrep[as] > 0 && B->nb_irrep[bs] > 0) {
            B->blk_asym[k] = as;
            B->blk_bsym[k] = bs;
            B->blk_na[k] = B->na_irrep[as];
            B->blk_nb[k] = B->nb_irrep[bs];
            B->blk_astrs[k] = B->all_a + B->a_start[as];
            B->blk_bstrs[k] = B->all_b + B->b_start[bs];
            B->blk_off[k] = dim;
            B->block_map[as * num_irreps + bs] = k;
            dim += B->blk_na[k] * B->blk_nb[k];
            k++;
        }
    }
    B->dim = dim;
    return B;
}

void oracle_basis_destroy(void *p)
{
    OBasis *B = (OBasis *)p;
    if (!B) return;
    free(B->blk_asym); free(B->blk_bsym); free(B->blk_na); free(B->blk_nb);
    free(B->blk_off); free(B->blk_astrs); free(B->blk_bstrs);
    free(B->all_a); free(B->all_b); free(B->na_irrep); free(B->nb_irrep);
    free(B->a_start); free(B->b_start); free(B->block_map);
    free(B);
}

i64 oracle_basis_dim(void *p) { return ((OBasis *)p)->dim; }
i64 oracle_basis_num_blocks(void *p) { return ((OBasis *)p)->num_blocks; }

/* Per block: asym, bsym, num_a, num_b, offset (5 int64 each). */
void oracle_basis_blocks(void *p, i64 *out)
{
    OBasis *B = (OBasis *)p;
    for (i64 k = 0; k < B->num_blocks; ++k) {
        out[5 * k + 0] = B->blk_asym[k];
        out[5 * k + 1] = B->blk_bsym[k];
        out[5 * k + 2] = B->blk_na[k];
        out[5 * k + 3] = B->blk_nb[k];
        out[5 * k + 4] = B->blk_off[k];
    }
}

/* Copy the alpha (spin=0) or beta (spin=1) string list of block k. */
void oracle_basis_strings(void *p, i64 k, int spin, u64 *out)
{
    OBasis *B = (OBasis *)p;
    i64 n = spin ? B->blk_nb[k] : B->blk_na[k];
    const u64 *s = spin ? B->blk_bstrs[k] : B->blk_astrs[k];
    memcpy(out, s, sizeof(u64) * n);
}

/* Index of string s inside its irrep list, or -1 (the a_idx_map/b_idx_map
 * lookup of basis.hpp:271-285, done by binary search as in find_index,
 * core/types.hpp:50-59).  Strings of an irrep that takes part in no block are
 * absent from the reference's map, so they are rejected here too. */
static i64 str_index(const OBasis *B, int spin, u64 s, const i64 *orbsym_unused)
{
    (void)orbsym_unused;
    /* find the irrep list containing s: search every block's list of that spin */
    for (i64 k = 0; k < B->num_blocks; ++k) {
        const u64 *arr = spin ? B->blk_bstrs[k] : B->blk_astrs[k];
        i64 n = spin ? B->blk_nb[k] : B->blk_na[k];
        i64 lo = 0, hi = n;
        while (lo < hi) {
            i64 mid = (lo + hi) >> 1;
            if (arr[mid] < s) lo = mid + 1; else hi = mid;
        }
        if (lo < n && arr[lo] == s) return lo;
    }
    return -1;
}

/* ------------------------------------------------------------------ */
/* network: ham/otf.hpp:224-349 (build_network_otf)                    */
/* ------------------------------------------------------------------ */

typedef struct {
    u64 ax, bx;
    int rank, nza, nzb, type;
    i64 asym, bsym, orig;
    u64 *za, *zb;
    double *wa, *wb;   /* column-major [num_z x rank]: w[r*num_z + k] (otf.hpp:84-85) */
} OGroup;

typedef struct {
    i64 ngs, norb;
    i64 *orbsym;
    OGroup *g;        /* in original order */
} ONet;

/* wm: doubles per weight (1 real, 2 complex (re, im) as ComplexF64 arrays) */
static void *net_create(const i64 *orbsym, i64 norb, i64 ngs,
                        const u64 *axs, const u64 *bxs, const i64 *ranks,
                        const i64 *nzas, const i64 *nzbs,
                        const u64 *flat_za, const u64 *flat_zb,
                        const double *flat_wa, const double *flat_wb, int wm)
{
    ONet *N = (ONet *)calloc(1, sizeof(ONet));
    N->ngs = ngs;
    N->norb = norb;
    N->orbsym = (i64 *)malloc(sizeof(i64) * (norb > 0 ? norb : 1));
    memcpy(N->orbsym, orbsym, sizeof(i64) * norb);
    N->g = (OGroup *)calloc(ngs > 0 ? ngs : 1, sizeof(OGroup));
    i64 oza = 0, ozb = 0, owa = 0, owb = 0;
    for (i64 i = 0; i < ngs; ++i) {
        OGroup *G = &N->g[i];
        G->ax = axs[i];
        G->bx = bxs[i];
        G->rank = (int)ranks[i];
        G->nza = (int)nzas[i];
        G->nzb = (int)nzbs[i];
        G->asym = string_sym(G->ax, orbsym);
        G->bsym = string_sym(G->bx, orbsym);
        G->orig = i;
        /* type code, otf.hpp:289-296 */
        G->type = (G->ax == 0 && G->bx == 0) ? 0 : (G->bx == 0) ? 1 : (G->ax == 0) ? 2 : 3;
        G->za = (u64 *)malloc(sizeof(u64) * (G->nza + 1));
        G->zb = (u64 *)malloc(sizeof(u64) * (G->nzb + 1));
        memcpy(G->za, flat_za + oza, sizeof(u64) * G->nza); oza += G->nza;
        memcpy(G->zb, flat_zb + ozb, sizeof(u64) * G->nzb); ozb += G->nzb;
        i64 swa = (i64)G->nza * G->rank * wm, swb = (i64)G->nzb * G->rank * wm;
        G->wa = (double *)malloc(sizeof(double) * (swa + 2));
        G->wb = (double *)malloc(sizeof(double) * (swb + 2));
        memcpy(G->wa, flat_wa + owa, sizeof(double) * swa); owa += swa;
        memcpy(G->wb, flat_wb + owb, sizeof(double) * swb); owb += swb;
    }
    return N;
}

void *oracle_net_create(const i64 *orbsym, i64 norb, i64 ngs,
                        const u64 *axs, const u64 *bxs, const i64 *ranks,
                        const i64 *nzas, const i64 *nzbs,
                        const u64 *flat_za, const u64 *flat_zb,
                        const double *flat_wa, const double *flat_wb)
{
    return net_create(orbsym, norb, ngs, axs, bxs, ranks, nzas, nzbs, flat_za, flat_zb, flat_wa, flat_wb, 1);
}

/* A network of the complex (Tv = complex<double>) interface, otf_native.cpp:4,6:
 * the weights are interleaved (re, im) pairs. */
void *oracle_net_create_c64(const i64 *orbsym, i64 norb, i64 ngs,
                            const u64 *axs, const u64 *bxs, const i64 *ranks,
                            const i64 *nzas, const i64 *nzbs,
                            const u64 *flat_za, const u64 *flat_zb,
                            const double *flat_wa, const double *flat_wb)
{
    return net_create(orbsym, norb, ngs, axs, bxs, ranks, nzas, nzbs, flat_za, flat_zb, flat_wa, flat_wb, 2);
}

void oracle_net_destroy(void *p)
{
    ONet *N = (ONet *)p;
    if (!N) return;
    for (i64 i = 0; i < N->ngs; ++i) {
        free(N->g[i].za); free(N->g[i].zb); free(N->g[i].wa); free(N->g[i].wb);
    }
    free(N->g); free(N->orbsym); free(N);
}

/* precompute_phase, core/math.hpp:37-78: P_r(s) = sum_k (-1)^{popc(s & z_k)} w[r,k]. */
static void phase(u64 s, const u64 *z, int nz, const double *w, int rank, double *p)
{
    for (int r = 0; r < rank; ++r) {
        const double *wr = w + (i64)r * nz;
        double v = 0.0;
        for (int k = 0; k < nz; ++k)
            v += parity64(s & z[k]) ? -wr[k] : wr[k];
        p[r] = v;
    }
}

/* compute_coeff, core/math.hpp:80-124: v = sum_r pa[r]*pb[r]. */
static double coeff(const double *pa, const double *pb, int rank)
{
    double v = 0.0;
    for (int r = 0; r < rank; ++r) v += pa[r] * pb[r];
    return v;
}

#define MAXR 256

/* Visit every connected (dst, src) determinant pair of group G.
 * dst = (a, b) in block kd, src = (a ^ ax, b ^ bx) in the block the group's
 * symmetry leads to (hvec.hpp:94-96, 190-192, 297-299).  When `once` is set
 * only one member of each unordered pair is visited, with the rule of
 * op/expm.hpp:93-123 (pure alpha), :194-224 (pure beta), :300-351 (mixed):
 * skip src_block < dst_block, and inside one block require the source alpha
 * (pure-beta: beta) index to exceed the destination's.
 * The visitor receives dst index di, src index si and vt = P_A(src_a)*P_B(src_b). */
typedef void (*pair_fn)(i64 di, i64 si, double vt, void *ctx, double *acc);

static double visit_pairs(const OBasis *B, const ONet *N, const OGroup *G, int once,
                          pair_fn fn, void *ctx)
{
    double total = 0.0;
    for (i64 kd = 0; kd < B->num_blocks; ++kd) {
        i64 sa_sym = B->blk_asym[kd] ^ G->asym;
        i64 sb_sym = B->blk_bsym[kd] ^ G->bsym;
        if (sa_sym >= B->num_irreps || sb_sym >= B->num_irreps) continue;
        i64 ks = B->block_map[sa_sym * B->num_irreps + sb_sym];
        if (ks < 0) continue;
        if (once && G->type != 0 && ks < kd) continue;
        const int same = (ks == kd);
        const i64 na = B->blk_na[kd], nb = B->blk_nb[kd];
        const i64 nbs = B->blk_nb[ks];
        const u64 *as = B->blk_astrs[kd], *bs = B->blk_bstrs[kd];
        /* beta side of the source: index and phases per dst beta column */
        i64 *sbi = (i64 *)malloc(sizeof(i64) * (nb + 1));
        double *pb = (double *)malloc(sizeof(double) * (nb + 1) * (G->rank + 1));
        for (i64 b = 0; b < nb; ++b) {
            u64 s = bs[b] ^ G->bx;
            sbi[b] = (G->bx == 0) ? b : str_index(B, 1, s, N->orbsym);
            if (sbi[b] >= 0) phase(s, G->zb, G->nzb, G->wb, G->rank, pb + b * G->rank);
        }
        double acc = 0.0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : acc)
        for (i64 a = 0; a < na; ++a) {
            u64 s = as[a] ^ G->ax;
            i64 sa = (G->ax == 0) ? a : str_index(B, 0, s, N->orbsym);
            if (sa < 0) continue;
            if (once && same && G->type != 2 && G->type != 0 && sa < a) continue;
            double pa[MAXR];
            phase(s, G->za, G->nza, G->wa, G->rank, pa);
            double local = 0.0;
            for (i64 b = 0; b < nb; ++b) {
                i64 sb = sbi[b];
                if (sb < 0) continue;
                if (once && same && G->type == 2 && sb < b) continue;
                double vt = coeff(pa, pb + b * G->rank, G->rank);
                i64 di = B->blk_off[kd] + a * nb + b;
                i64 si = B->blk_off[ks] + sa * nbs + sb;
                fn(di, si, vt, ctx, &local);
            }
            acc += local;
        }
        total += acc;
        free(sbi);
        free(pb);
    }
    return total;
}

/* ---------------- sigma: op/hvec.hpp:481-496 ---------------- */

typedef struct { const double *src; double *dst; } HvecCtx;

static void hvec_pair(i64 di, i64 si, double vt, void *ctx, double *acc)
{
    (void)acc;
    HvecCtx *c = (HvecCtx *)ctx;
    c->dst[di] += c->src[si] * vt;   /* hvec_update, core/math.hpp:126-130 */
}

/* dst = H src; dst is zeroed first (hvec.hpp:486-490).  Groups are applied in
 * original order; within one group every dst row is owned by one thread, so
 * there are no write races. */
void oracle_hvec(void *bp, void *np, const double *src, double *dst)
{
    OBasis *B = (OBasis *)bp;
    ONet *N = (ONet *)np;
    memset(dst, 0, sizeof(double) * B->dim);
    HvecCtx c = {src, dst};
    for (i64 g = 0; g < N->ngs; ++g)
        visit_pairs(B, N, &N->g[g], 0, hvec_pair, &c);
}

/* diag(H) += first diagonal group (hvec.hpp:498-554: uses diag_groups[0];
 * there is at most one group with ax = bx = 0).  Accumulates like the
 * reference (the caller zeroes). */
void oracle_diag(void *bp, void *np, double *diag)
{
    OBasis *B = (OBasis *)bp;
    ONet *N = (ONet *)np;
    for (i64 g = 0; g < N->ngs; ++g) {
        const OGroup *G = &N->g[g];
        if (G->type != 0) continue;
        for (i64 k = 0; k < B->num_blocks; ++k) {
            i64 na = B->blk_na[k], nb = B->blk_nb[k];
#pragma omp parallel for schedule(static)
            for (i64 a = 0; a < na; ++a) {
                double pa[MAXR], pb[MAXR];
                phase(B->blk_astrs[k][a], G->za, G->nza, G->wa, G->rank, pa);
                for (i64 b = 0; b < nb; ++b) {
                    phase(B->blk_bstrs[k][b], G->zb, G->nzb, G->wb, G->rank, pb);
                    diag[B->blk_off[k] + a * nb + b] += coeff(pa, pb, G->rank);
                }
            }
        }
        return;
    }
}

/* ---------------- expm / grad / backgrad ---------------- */

typedef struct { double *v; double cd, co; } ExpmCtx;

/* expm_update, core/math.hpp:132-146 (real Tv): sp = src, dp = dst. */
static void expm_pair(i64 di, i64 si, double vt, void *ctx, double *acc)
{
    (void)acc;
    ExpmCtx *c = (ExpmCtx *)ctx;
    double vd = 1.0 + c->cd * (vt * vt);
    double vi = c->v[si], vj = c->v[di];
    c->v[si] = vi * vd - vj * (c->co * vt);
    c->v[di] = vj * vd + vi * (c->co * vt);
}

/* v <- exp(theta G_idx) v, op/expm.hpp:374-438.  Diagonal groups are the
 * identity for real vectors (fast_diag_exp, core/math.hpp:7-20). */
void oracle_expm(void *bp, void *np, i64 idx, double theta, double *vec)
{
    OBasis *B = (OBasis *)bp;
    ONet *N = (ONet *)np;
    const OGroup *G = &N->g[idx];
    if (G->type == 0) return;
    ExpmCtx c = {vec, cos(theta) - 1.0, sin(theta)};
    visit_pairs(B, N, G, 1, expm_pair, &c);
}

typedef struct { const double *l, *r; double cd, co; } GradCtx;

/* grad_update, core/math.hpp:148-162 (real Tv). */
static void grad_pair(i64 di, i64 si, double vt, void *ctx, double *acc)
{
    GradCtx *c = (GradCtx *)ctx;
    double vd = c->cd * (vt * vt);
    double vo = c->co * vt;
    double rvi = c->r[si], rvj = c->r[di];
    *acc += c->l[si] * (rvi * vd + rvj * vo) + c->l[di] * (rvj * vd - rvi * vo);
}

/* <l| G e^{theta G} |r> in the reference's orientation, op/grad.hpp:397-465,
 * with cd = -sin(theta), co = cos(theta) (grad.hpp:76-77). */
double oracle_grad(void *bp, void *np, i64 idx, double theta, const double *l, const double *r)
{
    OBasis *B = (OBasis *)bp;
    ONet *N = (ONet *)np;
    const OGroup *G = &N->g[idx];
    if (G->type == 0) return 0.0;   /* fast_diag_grad is 0 for real Tv */
    GradCtx c = {l, r, -sin(theta), cos(theta)};
    return visit_pairs(B, N, G, 1, grad_pair, &c);
}

typedef struct { double *l, *r; double ecd, eco, gcd, gco; } BackCtx;

/* backgrad_update, core/math.hpp:187-215 (real Tv). */
static void back_pair(i64 di, i64 si, double vt, void *ctx, double *acc)
{
    BackCtx *c = (BackCtx *)ctx;
    double evd = 1.0 + c->ecd * (vt * vt), evo = c->eco * vt;
    double gvd = c->gcd * (vt * vt), gvo = c->gco * vt;
    double lvi = c->l[si], lvj = c->l[di], rvi = c->r[si], rvj = c->r[di];
    double els = lvi * evd - lvj * evo;
    double eld = lvj * evd + lvi * evo;
    *acc += els * (rvi * gvd + rvj * gvo) + eld * (rvj * gvd - rvi * gvo);
    c->l[si] = els;
    c->l[di] = eld;
    c->r[si] = rvi * evd - rvj * evo;
    c->r[di] = rvj * evd + rvi * evo;
}

/* Fused adjoint step, op/backgrad.hpp:406-474 with the angles of
 * backgrad.hpp:81-84: l <- e^{-theta G} l, g = <..>, r <- e^{-theta G} r. */
double oracle_backgrad(void *bp, void *np, i64 idx, double theta, double *l, double *r)
{
    OBasis *B = (OBasis *)bp;
    ONet *N = (ONet *)np;
    const OGroup *G = &N->g[idx];
    if (G->type == 0) return 0.0;
    BackCtx c = {l, r, cos(theta) - 1.0, -sin(theta), -sin(theta), cos(theta)};
    return visit_pairs(B, N, G, 1, back_pair, &c);
}

/* Pool gradient, op/batchgrad.hpp:529-540: grads[orig] = grad of every group
 * at thetas[orig]; grads is overwritten (std::fill at batchgrad.hpp:533). */
void oracle_batchgrad(void *bp, void *np, const double *thetas,
                      const double *l, const double *r, double *grads)
{
    ONet *N = (ONet *)np;
    for (i64 g = 0; g < N->ngs; ++g)
        grads[g] = oracle_grad(bp, np, g, thetas[g], l, r);
}

/* ---------------- tvec / backtran / batchexpm / batchtran ---------------- */

typedef struct { const double *src; double *dst; } TvecCtx;

/* tvec_update, core/math.hpp:165-170 (real Tv): ds = sd * (-vt), dd = ss * vt.
 * A diagonal group visits si == di, where the second store leaves
 * dst = src * vt, the diagonal rule of op/tvec.hpp:7-60. */
static void tvec_pair(i64 di, i64 si, double vt, void *ctx, double *acc)
{
    (void)acc;
    TvecCtx *c = (TvecCtx *)ctx;
    double ss = c->src[si], sd = c->src[di];
    c->dst[si] = sd * (-vt);
    c->dst[di] = ss * vt;
}

/* dst = T_idx src for one group, op/tvec.hpp (tvec_svd_network_otf):
 * dst is zeroed first. */
void oracle_tvec(void *bp, void *np, i64 idx, const double *src, double *dst)
{
    OBasis *B = (OBasis *)bp;
    ONet *N = (ONet *)np;
    memset(dst, 0, sizeof(double) * B->dim);
    TvecCtx c = {src, dst};
    visit_pairs(B, N, &N->g[idx], 1, tvec_pair, &c);
}

typedef struct { double *l, *r, *b; double cd, co; } BacktranCtx;

/* backtran_update, core/math.hpp:217-226 (real Tv): expm_update on l and on r,
 * then tvec_update from the rotated l into b. */
static void backtran_pair(i64 di, i64 si, double vt, void *ctx, double *acc)
{
    (void)acc;
    BacktranCtx *c = (BacktranCtx *)ctx;
    double vd = 1.0 + c->cd * (vt * vt), vo = c->co * vt;
    double li = c->l[si], lj = c->l[di], ri = c->r[si], rj = c->r[di];
    double ls = li * vd - lj * vo, ld = lj * vd + li * vo;
    c->l[si] = ls;
    c->l[di] = ld;
    c->r[si] = ri * vd - rj * vo;
    c->r[di] = rj * vd + ri * vo;
    c->b[si] = ld * (-vt);
    c->b[di] = ls * vt;
}

/* Diagonal group of backtran, op/backtran.hpp:7-70 (real Tv: the diagonal
 * exponential is 1): b = l * vt. */
static void backtran_diag(i64 di, i64 si, double vt, void *ctx, double *acc)
{
    (void)acc;
    (void)si;
    BacktranCtx *c = (BacktranCtx *)ctx;
    c->b[di] = c->l[di] * vt;
}

/* l <- e^{theta T} l, r <- e^{theta T} r, b = T l (rotated l); b zeroed first,
 * op/backtran.hpp (backtran_svd_network_otf, angles at :75-76). */
void oracle_backtran(void *bp, void *np, i64 idx, double theta, double *l, double *r, double *b)
{
    OBasis *B = (OBasis *)bp;
    ONet *N = (ONet *)np;
    const OGroup *G = &N->g[idx];
    memset(b, 0, sizeof(double) * B->dim);
    BacktranCtx c = {l, r, b, cos(theta) - 1.0, sin(theta)};
    visit_pairs(B, N, G, 1, G->type == 0 ? backtran_diag : backtran_pair, &c);
}

typedef struct { double *m; int ld, nv; double cd, co; } BatchExpmCtx;

/* expm_batch_update_matrix, core/math.hpp:228-252: expm_update on the first nv
 * entries of the rows si and di of a row-major matrix with row stride ld. */
static void batchexpm_pair(i64 di, i64 si, double vt, void *ctx, double *acc)
{
    (void)acc;
    BatchExpmCtx *c = (BatchExpmCtx *)ctx;
    double vd = 1.0 + c->cd * (vt * vt), vo = c->co * vt;
    double *sp = c->m + si * c->ld, *dp = c->m + di * c->ld;
    for (int k = 0; k < c->nv; ++k) {
        double vi = sp[k], vj = dp[k];
        sp[k] = vi * vd - vj * vo;
        dp[k] = vj * vd + vi * vo;
    }
}

/* e^{theta T_idx} on nv vectors stored as the columns of a dim x ld row-major
 * matrix, op/batchexpm.hpp (expm_svd_batched_network_otf); diagonal groups are
 * the identity for real vectors. */
void oracle_batchexpm(void *bp, void *np, i64 idx, double theta, double *matrix, int ld, int nv)
{
    OBasis *B = (OBasis *)bp;
    ONet *N = (ONet *)np;
    const OGroup *G = &N->g[idx];
    if (G->type == 0) return;
    BatchExpmCtx c = {matrix, ld, nv, cos(theta) - 1.0, sin(theta)};
    visit_pairs(B, N, G, 1, batchexpm_pair, &c);
}

typedef struct { const double *l, *r; } TranCtx;

/* tran_update, core/math.hpp:180-184 (real Tv): vt (l_s r_d - l_d r_s). */
static void tran_pair(i64 di, i64 si, double vt, void *ctx, double *acc)
{
    TranCtx *c = (TranCtx *)ctx;
    *acc += c->l[si] * vt * c->r[di] - c->l[di] * vt * c->r[si];
}

/* Diagonal group of batchtran, op/batchtran.hpp:7-81: l_i vt r_i. */
static void tran_diag(i64 di, i64 si, double vt, void *ctx, double *acc)
{
    (void)si;
    TranCtx *c = (TranCtx *)ctx;
    *acc += c->l[di] * vt * c->r[di];
}

/* trans[orig] = <l| T_g |r> for every group, op/batchtran.hpp:514-528
 * (tran_pool_network_batched_otf); trans is overwritten. */
void oracle_batchtran(void *bp, void *np, const double *l, const double *r, double *trans)
{
    OBasis *B = (OBasis *)bp;
    ONet *N = (ONet *)np;
    TranCtx c = {l, r};
    for (i64 g = 0; g < N->ngs; ++g) {
        const OGroup *G = &N->g[g];
        trans[g] = visit_pairs(B, N, G, 1, G->type == 0 ? tran_diag : tran_pair, &c);
    }
}

/* ------------------------------------------------------------------ */
/* Davidson vector helpers: diag/davidson.hpp:31-272 (real)            */
/* ------------------------------------------------------------------ */

/* build_ritz_and_residual, davidson.hpp:31-69: axt = sum c_j AV_j - e sum c_j V_j. */
double oracle_ritz_residual(i64 n, int dim, const double *c, double e,
                            const double *const *V, const double *const *AV, double *axt)
{
    double nrm = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : nrm)
    for (i64 i = 0; i < n; ++i) {
        double x = 0.0, ax = 0.0;
        for (int j = 0; j < dim; ++j) { x += c[j] * V[j][i]; ax += c[j] * AV[j][i]; }
        double rr = ax - e * x;
        axt[i] = rr;
        nrm += rr * rr;
    }
    return sqrt(nrm);
}

/* build_ritz_vector, davidson.hpp:71-95. */
void oracle_ritz_vector(i64 n, int dim, const double *c, const double *const *V, double *x)
{
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n; ++i) {
        double s = 0.0;
        for (int j = 0; j < dim; ++j) s += c[j] * V[j][i];
        x[i] = s;
    }
}

/* apply_preconditioner_inplace, davidson.hpp:97-117: r_i /= (d_i - e), the
 * denominator clamped to +-|shift| when smaller in magnitude. */
void oracle_precondition(i64 n, double *r, const double *d, double e, double shift)
{
    double s = fabs(shift);
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n; ++i) {
        double diff = d[i] - e;
        if (fabs(diff) < s) diff = (diff >= 0) ? s : -s;
        r[i] = r[i] / diff;
    }
}

/* mgs_orthogonalize, davidson.hpp:119-148: one modified Gram-Schmidt sweep,
 * returns the norm after it. */
double oracle_mgs(i64 n, int dim, const double *const *V, double *v)
{
    for (int j = 0; j < dim; ++j) {
        double p = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : p)
        for (i64 i = 0; i < n; ++i) p += V[j][i] * v[i];
#pragma omp parallel for schedule(static)
        for (i64 i = 0; i < n; ++i) v[i] -= p * V[j][i];
    }
    double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
    for (i64 i = 0; i < n; ++i) s += v[i] * v[i];
    return sqrt(s);
}

/* inplace_normalize, davidson.hpp:150-169. */
double oracle_normalize(i64 n, double *v)
{
    double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
    for (i64 i = 0; i < n; ++i) s += v[i] * v[i];
    double nrm = sqrt(s), inv = 1.0 / nrm;
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n; ++i) v[i] *= inv;
    return nrm;
}

/* fast_dot, davidson.hpp:171-184. */
double oracle_dot(i64 n, const double *a, const double *b)
{
    double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
    for (i64 i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* compute_heff_col, davidson.hpp:186-219: out_j = <V_j | AV_dim>. */
void oracle_heff_col(i64 n, int dim, const double *const *V, const double *av, double *out)
{
    for (int j = 0; j < dim; ++j) out[j] = oracle_dot(n, V[j], av);
}

/* ------------------------------------------------------------------ */
/* Complex (c64) operators: the Tv = complex<double> instantiation of  */
/* op/*.hpp with the rules of core/math.hpp:7-252 (conjugates, and the */
/* diagonal factors fast_diag_exp / fast_diag_grad).  Vectors are      */
/* interleaved (re, im) doubles.                                       */
/* ------------------------------------------------------------------ */
#include <complex.h>

typedef double complex zc;

static void phase_c(u64 s, const u64 *z, int nz, const zc *w, int rank, zc *p)
{
    for (int r = 0; r < rank; ++r) {
        const zc *wr = w + (i64)r * nz;
        zc v = 0.0;
        for (int k = 0; k < nz; ++k) v += parity64(s & z[k]) ? -wr[k] : wr[k];
        p[r] = v;
    }
}

typedef void (*pair_fn_c)(i64 di, i64 si, zc vt, int diag, void *ctx, zc *acc);

/* visit_pairs with complex phases; `diag` tells the visitor a diagonal group. */
static zc visit_pairs_c(const OBasis *B, const ONet *N, const OGroup *G, int once, pair_fn_c fn, void *ctx)
{
    double tre = 0.0, tim = 0.0;
    const zc *wa = (const zc *)G->wa, *wb = (const zc *)G->wb;
    for (i64 kd = 0; kd < B->num_blocks; ++kd) {
        i64 sa_sym = B->blk_asym[kd] ^ G->asym;
        i64 sb_sym = B->blk_bsym[kd] ^ G->bsym;
        if (sa_sym >= B->num_irreps || sb_sym >= B->num_irreps) continue;
        i64 ks = B->block_map[sa_sym * B->num_irreps + sb_sym];
        if (ks < 0) continue;
        if (once && G->type != 0 && ks < kd) continue;
        const int same = (ks == kd);
        const i64 na = B->blk_na[kd], nb = B->blk_nb[kd];
        const i64 nbs = B->blk_nb[ks];
        const u64 *as = B->blk_astrs[kd], *bs = B->blk_bstrs[kd];
        i64 *sbi = (i64 *)malloc(sizeof(i64) * (nb + 1));
        zc *pb = (zc *)malloc(sizeof(zc) * (nb + 1) * (G->rank + 1));
        for (i64 b = 0; b < nb; ++b) {
            u64 s = bs[b] ^ G->bx;
            sbi[b] = (G->bx == 0) ? b : str_index(B, 1, s, N->orbsym);
            if (sbi[b] >= 0) phase_c(s, G->zb, G->nzb, wb, G->rank, pb + b * G->rank);
        }
        double are = 0.0, aim = 0.0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : are, aim)
        for (i64 a = 0; a < na; ++a) {
            u64 s = as[a] ^ G->ax;
            i64 sa = (G->ax == 0) ? a : str_index(B, 0, s, N->orbsym);
            if (sa < 0) continue;
            if (once && same && G->type != 2 && G->type != 0 && sa < a) continue;
            zc pa[MAXR];
            phase_c(s, G->za, G->nza, wa, G->rank, pa);
            zc local = 0.0;
            for (i64 b = 0; b < nb; ++b) {
                i64 sb = sbi[b];
                if (sb < 0) continue;
                if (once && same && G->type == 2 && sb < b) continue;
                zc vt = 0.0;
                for (int r = 0; r < G->rank; ++r) vt += pa[r] * pb[b * G->rank + r];
                i64 di = B->blk_off[kd] + a * nb + b;
                i64 si = B->blk_off[ks] + sa * nbs + sb;
                fn(di, si, vt, G->type == 0, ctx, &local);
            }
            are += creal(local);
            aim += cimag(local);
        }
        tre += are;
        tim += aim;
        free(sbi);
        free(pb);
    }
    return tre + I * tim;
}

typedef struct { const zc *src; zc *dst; } HvecCtxC;

static void hvec_pair_c(i64 di, i64 si, zc vt, int diag, void *ctx, zc *acc)
{
    (void)diag; (void)acc;
    HvecCtxC *c = (HvecCtxC *)ctx;
    c->dst[di] += c->src[si] * vt;   /* hvec_update, core/math.hpp:126-130 */
}

/* dst = H src (op/hvec.hpp:481-496); dst zeroed first. */
void oracle_hvec_c64(void *bp, void *np, const double *src, double *dst)
{
    OBasis *B = (OBasis *)bp;
    ONet *N = (ONet *)np;
    memset(dst, 0, sizeof(zc) * B->dim);
    HvecCtxC c = {(const zc *)src, (zc *)dst};
    for (i64 g = 0; g < N->ngs; ++g) visit_pairs_c(B, N, &N->g[g], 0, hvec_pair_c, &c);
}

static void diag_pair_c(i64 di, i64 si, zc vt, int diag, void *ctx, zc *acc)
{
    (void)si; (void)diag; (void)acc;
    ((zc *)ctx)[di] += vt;
}

/* diag += the first diagonal group's values (op/hvec.hpp:498-554). */
void oracle_diag_c64(void *bp, void *np, double *diag)
{
    ONet *N = (ONet *)np;
    for (i64 g = 0; g < N->ngs; ++g)
        if (N->g[g].type == 0) { visit_pairs_c((OBasis *)bp, N, &N->g[g], 1, diag_pair_c, diag); return; }
}

typedef struct { zc *l, *r, *b; double cd, co, gcd, gco, th_e, th_g; int ld, nv; } OpCtxC;

static zc diag_exp(zc vt, double t) { return cexp(I * (cimag(vt) * t)); }      /* fast_diag_exp */
static zc diag_grad(zc vt, double t) { return vt * cexp(I * (cimag(vt) * t)); } /* fast_diag_grad */

static void expm_pair_c(i64 di, i64 si, zc vt, int diag, void *ctx, zc *acc)
{
    (void)acc;
    OpCtxC *c = (OpCtxC *)ctx;
    if (diag) { c->l[di] *= diag_exp(vt, c->th_e); return; }
    /* expm_update, core/math.hpp:132-146 */
    double vd = 1.0 + c->cd * creal(vt * conj(vt));
    zc vf = c->co * vt, vr = c->co * conj(vt);
    zc vi = c->l[si], vj = c->l[di];
    c->l[si] = vi * vd - vj * vr;
    c->l[di] = vj * vd + vi * vf;
}

void oracle_expm_c64(void *bp, void *np, i64 idx, double theta, double *vec)
{
    OpCtxC c = {(zc *)vec, 0, 0, cos(theta) - 1.0, sin(theta), 0, 0, theta, 0, 0, 0};
    visit_pairs_c((OBasis *)bp, (ONet *)np, &((ONet *)np)->g[idx], 1, expm_pair_c, &c);
}

static void grad_pair_c(i64 di, i64 si, zc vt, int diag, void *ctx, zc *acc)
{
    OpCtxC *c = (OpCtxC *)ctx;
    if (diag) { *acc += conj(c->l[di] * diag_grad(vt, c->th_g)) * c->r[di]; return; }
    /* grad_update, core/math.hpp:148-162 */
    double vd = c->cd * creal(vt * conj(vt));
    zc vf = c->co * vt, vr = c->co * conj(vt);
    zc rvi = c->r[si], rvj = c->r[di];
    *acc += conj(c->l[si]) * (rvi * vd + rvj * vr) + conj(c->l[di]) * (rvj * vd - rvi * vf);
}

/* <l| G e^{theta G} |r> (op/grad.hpp:397-465), written to out[0..1]. */
void oracle_grad_c64(void *bp, void *np, i64 idx, double theta, const double *l, const double *r, double *out)
{
    OpCtxC c = {(zc *)l, (zc *)r, 0, -sin(theta), cos(theta), 0, 0, 0, theta, 0, 0};
    zc g = visit_pairs_c((OBasis *)bp, (ONet *)np, &((ONet *)np)->g[idx], 1, grad_pair_c, &c);
    out[0] = creal(g);
    out[1] = cimag(g);
}

static void back_pair_c(i64 di, i64 si, zc vt, int diag, void *ctx, zc *acc)
{
    OpCtxC *c = (OpCtxC *)ctx;
    if (diag) {   /* op/backgrad.hpp:52-70 */
        zc u = diag_exp(vt, c->th_e);
        c->l[di] *= u;
        *acc += conj(c->l[di] * diag_grad(vt, c->th_g)) * c->r[di];
        c->r[di] *= u;
        return;
    }
    /* backgrad_update, core/math.hpp:187-215 */
    double n2 = creal(vt * conj(vt));
    double evd = 1.0 + c->cd * n2, gvd = c->gcd * n2;
    zc ef = c->co * vt, er = c->co * conj(vt), gf = c->gco * vt, gr = c->gco * conj(vt);
    zc lvi = c->l[si], lvj = c->l[di], rvi = c->r[si], rvj = c->r[di];
    zc els = lvi * evd - lvj * er, eld = lvj * evd + lvi * ef;
    *acc += conj(els) * (rvi * gvd + rvj * gr) + conj(eld) * (rvj * gvd - rvi * gf);
    c->l[si] = els;
    c->l[di] = eld;
    c->r[si] = rvi * evd - rvj * er;
    c->r[di] = rvj * evd + rvi * ef;
}

/* Fused adjoint step (op/backgrad.hpp:406-474, angles :81-84). */
void oracle_backgrad_c64(void *bp, void *np, i64 idx, double theta, double *l, double *r, double *out)
{
    OpCtxC c = {(zc *)l, (zc *)r, 0, cos(theta) - 1.0, -sin(theta), -sin(theta), cos(theta), -theta, theta, 0, 0};
    zc g = visit_pairs_c((OBasis *)bp, (ONet *)np, &((ONet *)np)->g[idx], 1, back_pair_c, &c);
    out[0] = creal(g);
    out[1] = cimag(g);
}

static void tvec_pair_c(i64 di, i64 si, zc vt, int diag, void *ctx, zc *acc)
{
    (void)acc;
    OpCtxC *c = (OpCtxC *)ctx;   /* l = src, r = dst */
    if (diag) { c->r[di] = c->l[di] * vt; return; }
    zc ss = c->l[si], sd = c->l[di];   /* tvec_update, core/math.hpp:165-170 */
    c->r[si] = sd * (-conj(vt));
    c->r[di] = ss * vt;
}

void oracle_tvec_c64(void *bp, void *np, i64 idx, const double *src, double *dst)
{
    memset(dst, 0, sizeof(zc) * ((OBasis *)bp)->dim);
    OpCtxC c = {(zc *)src, (zc *)dst, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    visit_pairs_c((OBasis *)bp, (ONet *)np, &((ONet *)np)->g[idx], 1, tvec_pair_c, &c);
}

static void backtran_pair_c(i64 di, i64 si, zc vt, int diag, void *ctx, zc *acc)
{
    (void)acc;
    OpCtxC *c = (OpCtxC *)ctx;
    if (diag) {   /* op/backtran.hpp:7-70 */
        zc u = diag_exp(vt, c->th_e);
        c->l[di] *= u;
        c->r[di] *= u;
        c->b[di] = c->l[di] * vt;
        return;
    }
    /* backtran_update, core/math.hpp:217-226 */
    double vd = 1.0 + c->cd * creal(vt * conj(vt));
    zc vf = c->co * vt, vr = c->co * conj(vt);
    zc li = c->l[si], lj = c->l[di], ri = c->r[si], rj = c->r[di];
    zc ls = li * vd - lj * vr, ld = lj * vd + li * vf;
    c->l[si] = ls;
    c->l[di] = ld;
    c->r[si] = ri * vd - rj * vr;
    c->r[di] = rj * vd + ri * vf;
    c->b[si] = ld * (-conj(vt));
    c->b[di] = ls * vt;
}

void oracle_backtran_c64(void *bp, void *np, i64 idx, double theta, double *l, double *r, double *b)
{
    memset(b, 0, sizeof(zc) * ((OBasis *)bp)->dim);
    OpCtxC c = {(zc *)l, (zc *)r, (zc *)b, cos(theta) - 1.0, sin(theta), 0, 0, theta, 0, 0, 0};
    visit_pairs_c((OBasis *)bp, (ONet *)np, &((ONet *)np)->g[idx], 1, backtran_pair_c, &c);
}

static void batchexpm_pair_c(i64 di, i64 si, zc vt, int diag, void *ctx, zc *acc)
{
    (void)acc;
    OpCtxC *c = (OpCtxC *)ctx;
    zc *sp = c->l + si * c->ld, *dp = c->l + di * c->ld;
    if (diag) {   /* expm_batch_update_diag */
        zc u = diag_exp(vt, c->th_e);
        for (int k = 0; k < c->nv; ++k) dp[k] *= u;
        return;
    }
    double vd = 1.0 + c->cd * creal(vt * conj(vt));   /* expm_batch_update_matrix, :228-252 */
    zc vf = c->co * vt, vr = c->co * conj(vt);
    for (int k = 0; k < c->nv; ++k) {
        zc vi = sp[k], vj = dp[k];
        sp[k] = vi * vd - vj * vr;
        dp[k] = vj * vd + vi * vf;
    }
}

void oracle_batchexpm_c64(void *bp, void *np, i64 idx, double theta, double *matrix, int ld, int nv)
{
    OpCtxC c = {(zc *)matrix, 0, 0, cos(theta) - 1.0, sin(theta), 0, 0, theta, 0, ld, nv};
    visit_pairs_c((OBasis *)bp, (ONet *)np, &((ONet *)np)->g[idx], 1, batchexpm_pair_c, &c);
}

/* grads[orig] = grad at thetas[orig] for every group (op/batchgrad.hpp:529-540). */
void oracle_batchgrad_c64(void *bp, void *np, const double *thetas, const double *l, const double *r, double *grads)
{
    ONet *N = (ONet *)np;
    for (i64 g = 0; g < N->ngs; ++g) oracle_grad_c64(bp, np, g, thetas[g], l, r, grads + 2 * g);
}

static void tran_pair_c(i64 di, i64 si, zc vt, int diag, void *ctx, zc *acc)
{
    OpCtxC *c = (OpCtxC *)ctx;
    if (diag) { *acc += conj(c->l[di] * vt) * c->r[di]; return; }   /* op/batchtran.hpp:7-81 */
    *acc += conj(c->l[si] * vt) * c->r[di] - conj(c->l[di]) * vt * c->r[si];   /* tran_update */
}

/* trans[orig] = <l|T_g|r> for every group (op/batchtran.hpp:514-528). */
void oracle_batchtran_c64(void *bp, void *np, const double *l, const double *r, double *trans)
{
    ONet *N = (ONet *)np;
    OpCtxC c = {(zc *)l, (zc *)r, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (i64 g = 0; g < N->ngs; ++g) {
        zc t = visit_pairs_c((OBasis *)bp, N, &N->g[g], 1, tran_pair_c, &c);
        trans[2 * g] = creal(t);
        trans[2 * g + 1] = cimag(t);
    }
}
