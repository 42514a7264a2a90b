// Construction and upload of the device basis and device OTF network.
#include "handles.h"
#include "refmirror.h"

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <numeric>

namespace bsim {

// ---- error bookkeeping --------------------------------------------------------
static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

const char *last_error() { return g_err; }

int cuda_status(cudaError_t e, const char *what)
{
    set_error("%s: %s", what, cudaGetErrorString(e));
    return BSIM_ERR_CUDA;
}

cudaError_t library_pool(cudaMemPool_t *pool)
{
    constexpr int kMaxDev = 64;
    static std::mutex mu;
    static cudaMemPool_t pools[kMaxDev] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p;
        if ((e = cudaMemPoolCreate(&p, &props)) != cudaSuccess) return e;
        unsigned long long keep = ~0ull;   // never hand freed memory back on synchronisation
        if ((e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
        pools[dev] = p;
    }
    *pool = pools[dev];
    return cudaSuccess;
}

cudaError_t trim_library_pool()
{
    cudaMemPool_t pool;
    cudaError_t e = library_pool(&pool);
    if (e != cudaSuccess) return e;
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return e;   // frees still queued on streams land first
    return cudaMemPoolTrimTo(pool, 0);
}

static std::atomic<long long> g_device_allocs{0};
void note_device_alloc() { g_device_allocs.fetch_add(1, std::memory_order_relaxed); }
long long device_alloc_count() { return g_device_allocs.load(std::memory_order_relaxed); }

// ---- arena --------------------------------------------------------------------
int Arena::reserve(size_t bytes)
{
    size = bytes + 4096;
    cudaError_t e = dmalloc(&base, size);
    if (e != cudaSuccess) {
        base = nullptr;
        set_error("device allocation of %zu bytes failed: %s", size, cudaGetErrorString(e));
        return BSIM_ERR_ALLOC;
    }
    used = 0;
    return BSIM_OK;
}

void Arena::release()
{
    if (base) cudaFree(base);
    base = nullptr;
    size = used = 0;
}

static size_t al(size_t n) { return (n + 255) & ~size_t(255); }

// ---- workspace ------------------------------------------------------------------
int Workspace::tile_table(const std::vector<i64> &pref, const i64 **out)
{
    if (tiles && pref == tiles_host) { *out = tiles; return BSIM_OK; }
    if (tiles) cudaFree(tiles);
    tiles = nullptr;
    cudaError_t e = dmalloc(&tiles, pref.size() * sizeof(i64));
    if (e != cudaSuccess) { tiles = nullptr; return cuda_status(e, "workspace tile table"); }
    e = cudaMemcpy(tiles, pref.data(), pref.size() * sizeof(i64), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_status(e, "workspace tile table copy");
    tiles_host = pref;
    tiles_n = pref.size();
    *out = tiles;
    return BSIM_OK;
}

int Workspace::f32_buffer(size_t n, float **out)
{
    if (f32_n < n) {
        if (f32) cudaFree(f32);
        f32 = nullptr;
        f32_n = 0;
        cudaError_t e = dmalloc(&f32, n * sizeof(float));
        if (e != cudaSuccess) { f32 = nullptr; return cuda_status(e, "workspace fp32 buffer"); }
        f32_n = n;
    }
    *out = f32;
    return BSIM_OK;
}

int Workspace::partials(size_t n, double **out)
{
    if (part_n < n) {
        if (part) cudaFree(part);
        part = nullptr;
        part_n = 0;
        cudaError_t e = dmalloc(&part, n * sizeof(double));
        if (e != cudaSuccess) { part = nullptr; return cuda_status(e, "workspace partials"); }
        // zeroed once: the tail holds the ticket counter of the last-CTA reductions
        e = cudaMemset(part, 0, n * sizeof(double));
        if (e != cudaSuccess) return cuda_status(e, "workspace partials");
        part_n = n;
    }
    *out = part;
    return BSIM_OK;
}

int Workspace::general(size_t bytes, void **out)
{
    if (gen_n < bytes) {
        if (gen) cudaFree(gen);
        gen = nullptr;
        gen_n = 0;
        cudaError_t e = dmalloc(&gen, bytes);
        if (e != cudaSuccess) { gen = nullptr; return cuda_status(e, "workspace general buffer"); }
        gen_n = bytes;
    }
    *out = gen;
    return BSIM_OK;
}

void Workspace::release()
{
    if (tiles) cudaFree(tiles);
    if (f32) cudaFree(f32);
    if (part) cudaFree(part);
    if (gen) cudaFree(gen);
    tiles = nullptr; f32 = nullptr; part = nullptr; gen = nullptr;
    tiles_n = f32_n = part_n = gen_n = 0;
    tiles_host.clear();
}

// ---- basis --------------------------------------------------------------------
static i64 sym_of(u64 s, const i64 *orbsym)
{
    i64 sym = 0;
    for (int p = 0; s; ++p, s >>= 1)
        if (s & 1u) sym ^= orbsym[p];
    return sym;
}

// Gosper's next combination (reference core/types.hpp:78-86).
static u64 next_comb(u64 v)
{
    if (v == 0) return 0;
    u64 c = v & (~v + 1);
    u64 r = v + c;
    return (((r ^ v) >> 2) / c) | r;
}

template <typename Ti>
static void strings_by_irrep(i64 norb, i64 ne, const i64 *orbsym, i64 nirr,
                             std::vector<std::vector<Ti>> &out)
{
    out.assign(nirr, {});
    const u64 lim = 1ull << norb;
    for (u64 s = (ne >= 64) ? ~0ull : ((1ull << ne) - 1); s < lim;) {
        i64 sym = sym_of(s, orbsym);
        if (sym < nirr) out[sym].push_back((Ti)s);
        if (ne == 0) break;
        s = next_comb(s);
    }
}

template <typename Ti>
int make_basis(i64 norb, i64 na, i64 nb, i64 total_sym, const i64 *orbsym, i64 num_irreps,
               DevBasis<Ti> **out)
{
    if (!out || (!orbsym && norb > 0)) { set_error("null argument"); return BSIM_ERR_NULL; }
    *out = nullptr;
    const i64 max_orb = sizeof(Ti) == 4 ? 32 : kMaxOrb64;
    if (norb < 1 || norb > max_orb) {
        set_error("norb=%lld unsupported (1..%lld for this string type)", norb, max_orb);
        return BSIM_ERR_UNSUPPORTED;
    }
    if (na < 0 || nb < 0 || na > norb || nb > norb || num_irreps < 1 || num_irreps > kMaxIrreps) {
        set_error("bad electron counts or irrep count");
        return BSIM_ERR_ARG;
    }
    for (i64 p = 0; p < norb; ++p)
        if (orbsym[p] < 0 || orbsym[p] >= kMaxIrreps) { set_error("orbsym out of range"); return BSIM_ERR_ARG; }
    auto *B = new DevBasis<Ti>();
    B->norb = (int)norb;
    B->num_irreps = (int)num_irreps;
    B->total_sym = total_sym;
    B->orbsym.assign(orbsym, orbsym + norb);
    std::vector<std::vector<Ti>> A, Bs;
    strings_by_irrep<Ti>(norb, na, orbsym, num_irreps, A);
    strings_by_irrep<Ti>(norb, nb, orbsym, num_irreps, Bs);
    // blocks: asym ascending, bsym = total_sym ^ asym (reference basis.hpp:233-259)
    B->block_map.assign(num_irreps * num_irreps, -1);
    i64 dim = 0;
    for (i64 as = 0; as < num_irreps; ++as) {
        i64 bs = total_sym ^ as;
        if (bs >= num_irreps || A[as].empty() || Bs[bs].empty()) continue;
        int k = (int)B->asym.size();
        B->asym.push_back((int)as);
        B->bsym.push_back((int)bs);
        B->na.push_back((int)A[as].size());
        B->nb.push_back((int)Bs[bs].size());
        B->astart.push_back((int)B->astrs.size());
        B->bstart.push_back((int)B->bstrs.size());
        B->astrs.insert(B->astrs.end(), A[as].begin(), A[as].end());
        B->bstrs.insert(B->bstrs.end(), Bs[bs].begin(), Bs[bs].end());
        B->off.push_back(dim);
        B->block_map[as * num_irreps + bs] = k;
        dim += (i64)A[as].size() * (i64)Bs[bs].size();
    }
    B->num_blocks = (int)B->asym.size();
    B->dim = dim;
    B->nel_a = (int)na;
    B->nel_b = (int)nb;
    int st = B->upload();
    if (st != BSIM_OK) { delete B; return st; }
    *out = B;
    return BSIM_OK;
}

template <typename Ti>
int DevBasis<Ti>::upload()
{
    max_na = max_nb = 0;
    for (int k = 0; k < num_blocks; ++k) {
        max_na = std::max(max_na, na[k]);
        max_nb = std::max(max_nb, nb[k]);
    }
    if (!astrs.empty()) nel_a = __builtin_popcountll((u64)astrs[0]);
    if (!bstrs.empty()) nel_b = __builtin_popcountll((u64)bstrs[0]);
    // index of a string inside its irrep list (reference basis.hpp:271-285): a
    // dense table up to 2^26 strings (the reference's map), else a table over
    // the colex rank of the string among all strings with its electron count
    std::vector<long long> binom(65 * 65, 0);
    for (int n = 0; n <= 64; ++n) {
        binom[n * 65] = 1;
        for (int k = 1; k <= n; ++k) {
            const unsigned long long a = (unsigned long long)binom[(n - 1) * 65 + k - 1];
            const unsigned long long b = k <= n - 1 ? (unsigned long long)binom[(n - 1) * 65 + k] : 0ull;
            const unsigned long long c = a + b;
            binom[n * 65 + k] = (c < a || c > 0x7fffffffffffffffull) ? 0x7fffffffffffffffll : (long long)c;
        }
    }
    const bool ranked = norb > kMaxDenseMapOrb;
    auto rank_of = [&](u64 x) {
        long long r = 0;
        int i = 1;
        for (u64 y = x; y; y &= y - 1, ++i) r += binom[__builtin_ctzll(y) * 65 + i];
        return r;
    };
    const size_t amap_n = ranked ? (size_t)binom[norb * 65 + nel_a] : size_t(1) << norb;
    const size_t bmap_n = ranked ? (size_t)binom[norb * 65 + nel_b] : size_t(1) << norb;
    if (amap_n > (size_t(1) << 30) || bmap_n > (size_t(1) << 30)) {
        set_error("string index tables of %zu / %zu entries are too large", amap_n, bmap_n);
        return BSIM_ERR_UNSUPPORTED;
    }
    std::vector<int> amap(amap_n, -1), bmap(bmap_n, -1);
    for (int k = 0; k < num_blocks; ++k) {
        for (int a = 0; a < na[k]; ++a) {
            const u64 x = (u64)astrs[astart[k] + a];
            amap[ranked ? (size_t)rank_of(x) : (size_t)x] = a;
        }
        for (int b = 0; b < nb[k]; ++b) {
            const u64 x = (u64)bstrs[bstart[k] + b];
            bmap[ranked ? (size_t)rank_of(x) : (size_t)x] = b;
        }
    }
    const int nbk = std::max(1, num_blocks);
    size_t bytes = 7 * al(nbk * sizeof(int)) + al(nbk * sizeof(i64)) +
                   al(std::max<size_t>(1, astrs.size()) * sizeof(Ti)) +
                   al(std::max<size_t>(1, bstrs.size()) * sizeof(Ti)) + al(amap_n * sizeof(int)) +
                   al(bmap_n * sizeof(int)) + al(block_map.size() * sizeof(int)) + al(binom.size() * 8);
    int st = arena.reserve(bytes);
    if (st != BSIM_OK) return st;
    auto put = [&](auto *dst, const auto &src) {
        using T = std::remove_reference_t<decltype(*dst)>;
        if (!src.empty()) cudaMemcpy((void *)dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
        return dst;
    };
    int *d_asym = put(arena.take<int>(nbk), asym);
    int *d_bsym = put(arena.take<int>(nbk), bsym);
    int *d_na = put(arena.take<int>(nbk), na);
    int *d_nb = put(arena.take<int>(nbk), nb);
    int *d_as = put(arena.take<int>(nbk), astart);
    int *d_bs = put(arena.take<int>(nbk), bstart);
    i64 *d_off = put(arena.take<i64>(nbk), off);
    Ti *d_astrs = put(arena.take<Ti>(std::max<size_t>(1, astrs.size())), astrs);
    Ti *d_bstrs = put(arena.take<Ti>(std::max<size_t>(1, bstrs.size())), bstrs);
    int *d_amap = put(arena.take<int>(amap_n), amap);
    int *d_bmap = put(arena.take<int>(bmap_n), bmap);
    int *d_bm = put(arena.take<int>(block_map.size()), block_map);
    long long *d_binom = put(arena.take<long long>(binom.size()), binom);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_status(e, "basis upload");
    view = BasisView<Ti>{num_blocks, num_irreps, norb, dim, d_asym, d_bsym, d_na, d_nb, d_as, d_bs,
                         d_off, d_astrs, d_bstrs, d_amap, d_bmap, d_bm, nel_a, nel_b, ranked ? 1 : 0, d_binom};
    return BSIM_OK;
}

template <typename Ti>
i64 DevBasis<Ti>::find_det(u64 astr, u64 bstr) const
{
    // set_det_coeff semantics (reference basis.hpp:298-330)
    i64 as = sym_of(astr, orbsym.data()), bs = sym_of(bstr, orbsym.data());
    if (as >= num_irreps || bs >= num_irreps) return -1;
    int k = block_map[as * num_irreps + bs];
    if (k < 0) return -1;
    auto fa = std::lower_bound(astrs.begin() + astart[k], astrs.begin() + astart[k] + na[k], (Ti)astr);
    auto fb = std::lower_bound(bstrs.begin() + bstart[k], bstrs.begin() + bstart[k] + nb[k], (Ti)bstr);
    if (fa == astrs.begin() + astart[k] + na[k] || *fa != (Ti)astr) return -1;
    if (fb == bstrs.begin() + bstart[k] + nb[k] || *fb != (Ti)bstr) return -1;
    return off[k] + (i64)(fa - (astrs.begin() + astart[k])) * nb[k] + (i64)(fb - (bstrs.begin() + bstart[k]));
}

// ---- network ------------------------------------------------------------------
template <typename Ti>
int make_network(const i64 *orbsym, i64 norb, i64 ngs, const Ti *axs, const Ti *bxs,
                 const i64 *ranks, const i64 *nzas, const i64 *nzbs, const Ti *flat_za,
                 const Ti *flat_zb, const double *flat_wa, const double *flat_wb,
                 DevNet<Ti> **out, bool wcomplex)
{
    if (!out) { set_error("null out"); return BSIM_ERR_NULL; }
    *out = nullptr;
    if (ngs < 0 || norb < 1 || norb > (i64)(8 * sizeof(Ti))) { set_error("bad ngs/norb"); return BSIM_ERR_ARG; }
    if (ngs > 0 && (!orbsym || !axs || !bxs || !ranks || !nzas || !nzbs)) {
        set_error("null network array");
        return BSIM_ERR_NULL;
    }
    auto *N = new DevNet<Ti>();
    N->norb = (int)norb;
    N->ngs = ngs;
    N->orbsym.assign(orbsym, orbsym + norb);
    i64 oza = 0, ozb = 0, owa = 0, owb = 0;
    // first all za, then all zb in z[]; first all wa, then all wb in w[]
    i64 tza = 0, tzb = 0, twa = 0, twb = 0;
    for (i64 g = 0; g < ngs; ++g) {
        if (ranks[g] < 0 || ranks[g] > kMaxRank || nzas[g] < 0 || nzbs[g] < 0) {
            set_error("group %lld: rank %lld or z counts out of range (max rank %d)", g, ranks[g], kMaxRank);
            delete N;
            return BSIM_ERR_UNSUPPORTED;
        }
        tza += nzas[g]; tzb += nzbs[g];
        twa += nzas[g] * ranks[g]; twb += nzbs[g] * ranks[g];
    }
    if ((tza + tzb > 0 && (!flat_za && tza) ) || (tzb && !flat_zb) || (twa && !flat_wa) || (twb && !flat_wb)) {
        set_error("null z/w arrays");
        delete N;
        return BSIM_ERR_NULL;
    }
    N->z.resize(tza + tzb);
    const i64 wm = wcomplex ? 2 : 1;   // doubles per weight
    N->w.resize(wm * (twa + twb));
    if (tza) memcpy(N->z.data(), flat_za, tza * sizeof(Ti));
    if (tzb) memcpy(N->z.data() + tza, flat_zb, tzb * sizeof(Ti));
    if (twa) memcpy(N->w.data(), flat_wa, wm * twa * sizeof(double));
    if (twb) memcpy(N->w.data() + wm * twa, flat_wb, wm * twb * sizeof(double));
    if (wcomplex) {
        N->cplx = 1;
        N->magic = HandleMagic<Ti>::net_c64;
    }
    N->groups.resize(ngs);
    for (i64 g = 0; g < ngs; ++g) {
        GroupDev &G = N->groups[g];
        G.ax = (u64)axs[g];
        G.bx = (u64)bxs[g];
        G.rank = (int)ranks[g];
        G.nza = (int)nzas[g];
        G.nzb = (int)nzbs[g];
        G.type = (G.ax == 0 && G.bx == 0) ? 0 : (G.bx == 0) ? 1 : (G.ax == 0) ? 2 : 3;
        G.asym = (int)sym_of(G.ax, orbsym);
        G.bsym = (int)sym_of(G.bx, orbsym);
        G.orig = (int)g;
        G.pad = 0;
        G.za_off = oza;
        G.zb_off = tza + ozb;
        G.wa_off = owa;
        G.wb_off = twa + owb;
        oza += G.nza; ozb += G.nzb;
        owa += (i64)G.nza * G.rank; owb += (i64)G.nzb * G.rank;
    }
    int st = N->finalize();
    if (st != BSIM_OK) { delete N; return st; }
    *out = N;
    return BSIM_OK;
}

template <typename Ti>
int DevNet<Ti>::finalize()
{
    excit_type.assign(ngs, 0);
    sorted_pos.assign(ngs, -1);
    for (auto &v : by_type) v.clear();
    max_rank = 0;
    for (i64 g = 0; g < ngs; ++g) {
        excit_type[g] = groups[g].type;
        by_type[groups[g].type].push_back((int)g);
        max_rank = std::max(max_rank, groups[g].rank);
    }
    // each type bucket sorted by rank (reference otf.hpp:305-313)
    for (auto &v : by_type)
        std::stable_sort(v.begin(), v.end(), [&](int a, int b) { return groups[a].rank < groups[b].rank; });
    for (auto &v : by_type)
        for (size_t i = 0; i < v.size(); ++i) sorted_pos[v[i]] = (i64)i;
    diag_group = by_type[0].empty() ? -1 : by_type[0][0];
    // sigma plan
    plan_groups.clear();
    plan_chunks.clear();
    for (auto &v : by_type) plan_groups.insert(plan_groups.end(), v.begin(), v.end());
    for (size_t i = 0; i < plan_groups.size();) {
        const int r = groups[plan_groups[i]].rank;
        size_t j = i + 1;
        const int ty = groups[plan_groups[i]].type;
        if (r <= 2)
            while (j < plan_groups.size() && j - i < 32 && groups[plan_groups[j]].rank == r &&
                   groups[plan_groups[j]].type == ty)
                ++j;
        if (r > 0) plan_chunks.push_back(make_int4((int)i, (int)(j - i), r, ty));
        i = j;
    }
    std::vector<float> w32(w.begin(), w.end());
    size_t bytes = al(std::max<size_t>(1, groups.size()) * sizeof(GroupDev)) +
                   al(std::max<size_t>(1, z.size()) * sizeof(Ti)) + al(std::max<size_t>(1, w.size()) * sizeof(double)) +
                   al(std::max<size_t>(1, w.size()) * sizeof(float)) +
                   al(std::max<size_t>(1, plan_groups.size()) * sizeof(int)) +
                   al(std::max<size_t>(1, plan_chunks.size()) * sizeof(int4));
    int st = arena.reserve(bytes);
    if (st != BSIM_OK) return st;
    auto put = [&](auto *dst, const auto &src) {
        using T = std::remove_reference_t<decltype(*dst)>;
        if (!src.empty()) cudaMemcpy((void *)dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
        return dst;
    };
    GroupDev *d_g = put(arena.take<GroupDev>(std::max<size_t>(1, groups.size())), groups);
    Ti *d_z = put(arena.take<Ti>(std::max<size_t>(1, z.size())), z);
    double *d_w = put(arena.take<double>(std::max<size_t>(1, w.size())), w);
    float *d_w32 = put(arena.take<float>(std::max<size_t>(1, w32.size())), w32);
    int *d_pg = put(arena.take<int>(std::max<size_t>(1, plan_groups.size())), plan_groups);
    int4 *d_pc = put(arena.take<int4>(std::max<size_t>(1, plan_chunks.size())), plan_chunks);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_status(e, "network upload");
    view = NetView<Ti>{(int)ngs, d_g, d_z, d_w, d_w32};
    d_plan_groups = d_pg;
    d_plan_chunks = d_pc;
    return BSIM_OK;
}

// ---- from the reference's host handles ---------------------------------------
int basis_from_ref_handle(const void *host_basis, DevBasis<unsigned> **out)
{
    if (!host_basis || !out) { set_error("null basis handle"); return BSIM_ERR_NULL; }
    *out = nullptr;
    const auto *H = static_cast<const refmirror::BasisManager32 *>(host_basis);
    if (H->norb < 1 || H->norb > kMaxDenseMapOrb || H->num_irreps < 1 || H->num_irreps > kMaxIrreps ||
        H->num_blocks < 0 || H->num_blocks > H->num_irreps) {
        set_error("host basis handle has out-of-range fields");
        return BSIM_ERR_ARG;
    }
    auto *B = new DevBasis<unsigned>();
    B->norb = (int)H->norb;
    B->num_irreps = (int)H->num_irreps;
    B->total_sym = H->total_sym;
    B->orbsym.assign(H->orbsym, H->orbsym + H->norb);
    B->block_map.assign(H->num_irreps * H->num_irreps, -1);
    i64 dim = 0;
    for (i64 k = 0; k < H->num_blocks; ++k) {
        const refmirror::BlockDesc32 &d = H->blocks[k];
        B->asym.push_back((int)d.asym);
        B->bsym.push_back((int)d.bsym);
        B->na.push_back((int)d.num_a);
        B->nb.push_back((int)d.num_b);
        B->astart.push_back((int)B->astrs.size());
        B->bstart.push_back((int)B->bstrs.size());
        B->astrs.insert(B->astrs.end(), d.astrs, d.astrs + d.num_a);
        B->bstrs.insert(B->bstrs.end(), d.bstrs, d.bstrs + d.num_b);
        B->off.push_back(d.offset);
        B->block_map[d.asym * H->num_irreps + d.bsym] = (int)k;
        dim = std::max<i64>(dim, d.offset + d.num_a * d.num_b);
    }
    B->num_blocks = (int)H->num_blocks;
    B->dim = dim;
    int st = B->upload();
    if (st != BSIM_OK) { delete B; return st; }
    *out = B;
    return BSIM_OK;
}

int network_from_ref_handle(const void *host_net, DevNet<unsigned> **out)
{
    if (!host_net || !out) { set_error("null network handle"); return BSIM_ERR_NULL; }
    *out = nullptr;
    const auto *H = static_cast<const refmirror::NetworkOTF32 *>(host_net);
    const refmirror::Vec<refmirror::SVDGroup32> *buckets[4] = {&H->diag_groups, &H->pure_a_groups,
                                                              &H->pure_b_groups, &H->mixed_groups};
    i64 total = 0;
    for (auto *b : buckets) total += b->size();
    if (total != H->num_groups || total < 0) {
        set_error("host network handle is inconsistent");
        return BSIM_ERR_ARG;
    }
    std::vector<const refmirror::SVDGroup32 *> byorig(total, nullptr);
    for (auto *b : buckets)
        for (const refmirror::SVDGroup32 *g = b->b; g != b->e; ++g) {
            if (g->original_idx < 0 || g->original_idx >= total || byorig[g->original_idx]) {
                set_error("host network handle has bad original indices");
                return BSIM_ERR_ARG;
            }
            byorig[g->original_idx] = g;
        }
    std::vector<unsigned> axs(total), bxs(total), za, zb;
    std::vector<i64> ranks(total), nza(total), nzb(total);
    std::vector<double> wa, wb;
    i64 norb = 32;
    for (i64 i = 0; i < total; ++i) {
        const auto *g = byorig[i];
        axs[i] = g->ax; bxs[i] = g->bx; ranks[i] = g->rank; nza[i] = g->num_za; nzb[i] = g->num_zb;
        za.insert(za.end(), g->unique_zas, g->unique_zas + g->num_za);
        zb.insert(zb.end(), g->unique_zbs, g->unique_zbs + g->num_zb);
        wa.insert(wa.end(), g->wa, g->wa + (i64)g->num_za * g->rank);
        wb.insert(wb.end(), g->wb, g->wb + (i64)g->num_zb * g->rank);
    }
    // The host network does not store norb; its orbsym has norb entries but no
    // length.  Symmetry of a mask only reads orbsym at set bits, so taking the
    // highest bit used by any X mask bounds the reads.
    unsigned used = 0;
    for (i64 i = 0; i < total; ++i) used |= axs[i] | bxs[i];
    norb = 1;
    while (norb < 32 && (used >> norb)) ++norb;
    std::vector<i64> orbsym(H->orbsym, H->orbsym + norb);
    return make_network<unsigned>(orbsym.data(), norb, total, axs.data(), bxs.data(), ranks.data(), nza.data(),
                                  nzb.data(), za.data(), zb.data(), wa.data(), wb.data(), out);
}

template int make_basis<unsigned>(i64, i64, i64, i64, const i64 *, i64, DevBasis<unsigned> **);
template int make_network<unsigned>(const i64 *, i64, i64, const unsigned *, const unsigned *, const i64 *,
                                    const i64 *, const i64 *, const unsigned *, const unsigned *,
                                    const double *, const double *, DevNet<unsigned> **, bool);
template struct DevBasis<unsigned>;
template struct DevNet<unsigned>;
template int make_basis<unsigned long long>(i64, i64, i64, i64, const i64 *, i64, DevBasis<unsigned long long> **);
template int make_network<unsigned long long>(const i64 *, i64, i64, const unsigned long long *,
                                              const unsigned long long *, const i64 *, const i64 *, const i64 *,
                                              const unsigned long long *, const unsigned long long *, const double *,
                                              const double *, DevNet<unsigned long long> **, bool);
template struct DevBasis<unsigned long long>;
template struct DevNet<unsigned long long>;

}  // namespace bsim
