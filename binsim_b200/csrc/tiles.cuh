// Tile machinery shared by the sigma and pool-gradient kernels.
//
// A CTA owns a 32 x 32 destination tile (32 alpha rows x 32 beta columns) of one
// symmetry block.  Groups are processed in chunks (uniform rank <= 2, up to 32
// groups; or one group of larger rank).  For each chunk the CTA stages in
// shared memory, per group:
//   * for the 32 columns: the source beta index  sb = idx(b_str ^ bx)  and the
//     beta phases PB_r(b_str ^ bx)            (amortised over 32 rows)
//   * for the 32 rows:    the source row offset off[ks] + sa * nb[ks] and the
//     alpha phases PA_r(a_str ^ ax)           (amortised over 32 columns)
// and then every thread (lane = column, 4 rows per warp) accumulates
//   v = sum_r PA_r * PB_r ;  use(src[row + sb])
// Lanes take consecutive columns, so every destination access and every source
// access of a group with bx == 0 (diagonal, pure alpha) is a coalesced 256-byte
// row segment.  Semantics follow reference op/hvec.hpp:7-384 (all ordered
// pairs) or, with ONCE, the unordered-pair rule of op/expm.hpp:93-351.
#pragma once
#include "common.cuh"

namespace bsim {

constexpr int kTile = 32;
constexpr int kRowsPerWarp = 4;
constexpr int kTileThreads = 256;   // 8 warps x 4 rows = 32 rows
constexpr int kChunkSlots = 64;     // sum over a chunk of (groups x rank) <= 64

template <typename Tw>
struct TileSmem {
    Tw pa[kChunkSlots][kTile];   // [g*R + r][row]
    Tw pb[kChunkSlots][kTile];   // [g*R + r][col]
    i64 row[kTile][kTile];       // [g][row] source row base (element index), -1 invalid
    int col[kTile][kTile];       // [g][col] source column, -1 invalid
};

struct TileCoord {
    int k, ta, tb;      // block, tile row, tile column
    int na, nb;
};

// Decode a flat tile id using the per-block prefix of tile counts.
template <typename Ti>
__device__ __forceinline__ TileCoord decode_tile(const BasisView<Ti> &B, const i64 *__restrict__ tile_start,
                                                 i64 t)
{
    TileCoord c;
    int k = 0;
    while (k + 1 < B.num_blocks && tile_start[k + 1] <= t) ++k;
    c.k = k;
    c.na = B.blk_na[k];
    c.nb = B.blk_nb[k];
    const int ntb = (c.nb + kTile - 1) / kTile;
    const i64 lt = t - tile_start[k];
    c.ta = (int)(lt / ntb);
    c.tb = (int)(lt % ntb);
    return c;
}

// Stage the chunk's per-group column and row data.  `ONCE` applies the
// unordered-pair rule: source block >= destination block, and inside one block
// source alpha index > destination's (types 1, 3) or source beta index >
// destination's (type 2).
template <typename Ti, typename Tw, bool ONCE>
__device__ __forceinline__ void fill_chunk(const BasisView<Ti> &B, const NetView<Ti> &N,
                                           const int *__restrict__ plan_g, int start, int G, int R,
                                           const TileCoord &c, TileSmem<Tw> &S, const double *__restrict__ wsrc_unused)
{
    (void)wsrc_unused;
    const int nirr = B.num_irreps;
    const int dasym = B.blk_asym[c.k], dbsym = B.blk_bsym[c.k];
    for (int t = threadIdx.x; t < G * kTile; t += blockDim.x) {
        const int gl = t >> 5, j = t & 31;
        const GroupDev gd = N.g[plan_g[start + gl]];
        const int as = dasym ^ gd.asym, bs = dbsym ^ gd.bsym;
        int ks = (as < nirr && bs < nirr) ? B.block_map[as * nirr + bs] : -1;
        if (ONCE && ks >= 0 && ks < c.k) ks = -1;
        const bool same = (ks == c.k);
        const Tw *wz = nullptr;
        // ---- column j ----
        int sc = -1;
        const int b = c.tb * kTile + j;
        if (ks >= 0 && b < c.nb) {
            const Ti s = B.bstrs[B.blk_bstart[c.k] + b] ^ (Ti)gd.bx;
            sc = gd.bx ? string_index(B, B.bmap, B.nel_b, s) : b;
            if (ONCE && same && gd.type == 2 && sc >= 0 && sc < b) sc = -1;
            if (sc >= 0) {
                const Ti *z = N.z + gd.zb_off;
                if constexpr (sizeof(Tw) == 8) wz = (const Tw *)(N.w + gd.wb_off);
                else wz = (const Tw *)(N.w32 + gd.wb_off);
                for (int r = 0; r < R; ++r) {
                    Tw v = Tw(0);
                    const Tw *wr = wz + (i64)r * gd.nzb;
                    for (int q = 0; q < gd.nzb; ++q) v += par(s & z[q]) ? -wr[q] : wr[q];
                    S.pb[gl * R + r][j] = v;
                }
            }
        }
        S.col[gl][j] = sc;
        // ---- row j ----
        i64 row = -1;
        const int a = c.ta * kTile + j;
        if (ks >= 0 && a < c.na) {
            const Ti s = B.astrs[B.blk_astart[c.k] + a] ^ (Ti)gd.ax;
            int sa = gd.ax ? string_index(B, B.amap, B.nel_a, s) : a;
            if (ONCE && same && (gd.type == 1 || gd.type == 3) && sa >= 0 && sa < a) sa = -1;
            if (sa >= 0) {
                row = B.blk_off[ks] + (i64)sa * B.blk_nb[ks];
                const Ti *z = N.z + gd.za_off;
                if constexpr (sizeof(Tw) == 8) wz = (const Tw *)(N.w + gd.wa_off);
                else wz = (const Tw *)(N.w32 + gd.wa_off);
                for (int r = 0; r < R; ++r) {
                    Tw v = Tw(0);
                    const Tw *wr = wz + (i64)r * gd.nza;
                    for (int q = 0; q < gd.nza; ++q) v += par(s & z[q]) ? -wr[q] : wr[q];
                    S.pa[gl * R + r][j] = v;
                }
            }
        }
        S.row[gl][j] = row;
    }
}

}  // namespace bsim
