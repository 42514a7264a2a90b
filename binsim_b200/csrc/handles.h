// Host-side handles of libcuotf: the device basis and the device OTF network.
//
// A handle owns one device arena (a single cudaMalloc) holding every table
// the kernels read.  Handles start with a magic word so that entry points can
// reject pointers that are not handles of the right kind.
#pragma once
#include "common.cuh"

namespace bsim {

// Magic words per string type: UInt32 handles (the reference's GPU library's
// type) and UInt64 handles (up to 63 spatial orbitals).
template <typename Ti> struct HandleMagic;
// Complex (c64) networks carry their own magic words, so the real operators
// reject them and the c64 operators reject real networks.
template <> struct HandleMagic<unsigned> {
    static constexpr unsigned basis = 0xB5B1A515u, net = 0xB5B1E7A1u, net_c64 = 0xB5B1C632u;
};
template <> struct HandleMagic<unsigned long long> {
    static constexpr unsigned basis = 0xB5B1A564u, net = 0xB5B1E764u, net_c64 = 0xB5B1C664u;
};
constexpr unsigned kBasisMagic = HandleMagic<unsigned>::basis;
constexpr unsigned kNetMagic = HandleMagic<unsigned>::net;
constexpr int kMaxDenseMapOrb = 26;   // dense string->index tables up to 2^26 entries; ranked above
constexpr int kMaxOrb64 = 63;         // UInt64 strings (Gosper enumeration needs one spare bit)

// Device arena: one allocation carved into aligned pieces.
struct Arena {
    char *base = nullptr;
    size_t size = 0, used = 0;
    int reserve(size_t bytes);
    template <typename T>
    T *take(size_t n) {
        size_t a = (used + 255) & ~size_t(255);
        used = a + n * sizeof(T);
        return reinterpret_cast<T *>(base + a);
    }
    void release();
};

// Grow-on-demand device scratch owned by a basis handle: the tile table of the
// tile kernels, an FP32 staging vector, reduction partials and result slots.
// Growth calls cudaMalloc (synchronous); steady-state calls allocate nothing.
// Calls that share one basis handle share this scratch, so they must not run
// concurrently on different streams.
struct Workspace {
    i64 *tiles = nullptr;
    size_t tiles_n = 0;
    std::vector<i64> tiles_host;
    float *f32 = nullptr;
    size_t f32_n = 0;
    double *part = nullptr;
    size_t part_n = 0;
    void *gen = nullptr;     // general scratch (the VQE sweep's checkpoints and terms)
    size_t gen_n = 0;
    int tile_table(const std::vector<i64> &pref, const i64 **out);
    int f32_buffer(size_t n, float **out);
    int partials(size_t n, double **out);
    int general(size_t bytes, void **out);
    void release();
};

template <typename Ti>
struct DevBasis {
    unsigned magic = HandleMagic<Ti>::basis;
    int norb = 0, num_irreps = 0, num_blocks = 0;
    int nel_a = 0, nel_b = 0;
    i64 dim = 0, total_sym = 0;
    int max_na = 0, max_nb = 0;
    // host mirrors
    std::vector<int> asym, bsym, na, nb, astart, bstart, block_map;
    std::vector<i64> off;
    std::vector<Ti> astrs, bstrs;
    std::vector<i64> orbsym;
    // device
    Arena arena;
    BasisView<Ti> view{};
    mutable Workspace ws;

    int upload();                       // builds dense maps + copies tables
    i64 find_det(u64 astr, u64 bstr) const;   // -1 when absent
    ~DevBasis() { ws.release(); arena.release(); magic = 0; }
};

template <typename Ti>
struct DevNet {
    unsigned magic = HandleMagic<Ti>::net;
    int norb = 0;
    i64 ngs = 0;
    std::vector<GroupDev> groups;        // original order
    std::vector<Ti> z;
    std::vector<double> w;               // complex networks: interleaved (re, im), offsets in complex units
    int cplx = 0;                        // 1: complex weights (the reference's Tv = complex<double>)
    std::vector<i64> orbsym;
    // reference-style bookkeeping (ham/otf.hpp:329-344)
    std::vector<int> excit_type;         // [ngs] original index -> type
    std::vector<i64> sorted_pos;         // [ngs] original index -> position inside its type list
    std::vector<int> by_type[4];         // original indices per type, stably sorted by rank
    int diag_group = -1;                 // first diagonal group (get_diags uses it)
    int max_rank = 0;
    // sigma chunk plan: groups in (type, rank) order cut into chunks with uniform
    // rank <= 2 and at most 32 groups, or a single group of larger rank
    std::vector<int> plan_groups;        // original indices in plan order
    std::vector<int4> plan_chunks;       // {start, count, rank, type-mask}
    // device
    Arena arena;
    NetView<Ti> view{};
    const int *d_plan_groups = nullptr;
    const int4 *d_plan_chunks = nullptr;

    // cached structured-sigma plan for the last basis it was used with
    void *fast_state = nullptr;
    void (*fast_free)(void *) = nullptr;
    // cached pair lists of the pair operators for the last basis they were used with
    void *pair_state = nullptr;
    void (*pair_free)(void *) = nullptr;
    // cached theta = 0 route of the pool gradient (transition densities) for the
    // last basis it was used with
    void *density_state = nullptr;
    void (*density_free)(void *) = nullptr;

    int finalize();   // derived tables + upload
    ~DevNet() {
        if (fast_state && fast_free) fast_free(fast_state);
        if (pair_state && pair_free) pair_free(pair_state);
        if (density_state && density_free) density_free(density_state);
        arena.release();
        magic = 0;
    }
};

// ---- constructors -----------------------------------------------------------
template <typename Ti>
int make_basis(i64 norb, i64 na, i64 nb, i64 total_sym, const i64 *orbsym, i64 num_irreps,
               DevBasis<Ti> **out);

// wcomplex: flat_wa / flat_wb hold interleaved complex weights (twice the
// doubles), the network gets the c64 magic word.
template <typename Ti>
int make_network(const i64 *orbsym, i64 norb, i64 ngs, const Ti *axs, const Ti *bxs,
                 const i64 *ranks, const i64 *nzas, const i64 *nzbs, const Ti *flat_za,
                 const Ti *flat_zb, const double *flat_wa, const double *flat_wb,
                 DevNet<Ti> **out, bool wcomplex = false);

// From the reference's own host handles (layout mirrors in refmirror.h).
int basis_from_ref_handle(const void *host_basis, DevBasis<unsigned> **out);
int network_from_ref_handle(const void *host_net, DevNet<unsigned> **out);

template <typename Ti>
inline bool valid(const DevBasis<Ti> *b) { return b && b->magic == HandleMagic<Ti>::basis; }
template <typename Ti>
inline bool valid(const DevNet<Ti> *n) { return n && n->magic == HandleMagic<Ti>::net; }
template <typename Ti>
inline bool valid_c64(const DevNet<Ti> *n) { return n && n->magic == HandleMagic<Ti>::net_c64; }
// The first word of a handle tells its string type.
inline bool is_u64_basis(const void *h) { return h && *static_cast<const unsigned *>(h) == HandleMagic<unsigned long long>::basis; }
inline bool is_u64_net(const void *h) { return h && *static_cast<const unsigned *>(h) == HandleMagic<unsigned long long>::net; }
inline bool is_c64_net(const void *h)
{
    if (!h) return false;
    const unsigned m = *static_cast<const unsigned *>(h);
    return m == HandleMagic<unsigned>::net_c64 || m == HandleMagic<unsigned long long>::net_c64;
}

}  // namespace bsim
