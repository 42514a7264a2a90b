// Layout mirrors of the reference's host objects, so that the legacy entry
// points build_basisdev_f64 / build_networkdev_f64 accept the very handles the
// reference's CPU libraries return (jl/cuda/cunetwork.jl:13-53 passes them
// straight through).  Only the leading members the device copy needs are
// mirrored; member types and order are those of the reference:
//   BlockDesc<uint32>       src/include/basis/basis.hpp:7-13
//   BasisManager<uint32>    src/include/basis/basis.hpp:29-60
//   SVDGroup_OTF<uint32,double>  src/include/ham/otf.hpp:67-85
//   Network_OTF<uint32,double>   src/include/ham/otf.hpp:114-126
// std::vector<T> is mirrored as libstdc++'s three pointers (begin, end,
// end-of-storage); both sides are built by the same g++ ABI on x86-64.
#pragma once
#include <cstdint>

namespace bsim {
namespace refmirror {

struct BlockDesc32 {
    int64_t asym, bsym, num_a, num_b;
    const uint32_t *astrs, *bstrs;
    int64_t offset;
};

struct BasisManager32 {
    uint32_t *all_astrs, *all_bstrs;
    uint32_t **astrs_vec, **bstrs_vec;
    int64_t *num_astrs, *num_bstrs;
    BlockDesc32 *blocks;
    int64_t num_blocks;
    int64_t *orbsym;
    int64_t *block_map;
    int64_t num_irreps, physical_num_irreps, total_sym, dim, norb;
    int max_a_count, max_b_count;
    int *a_idx_map, *b_idx_map;
};

struct SVDGroup32 {
    uint32_t ax, bx;
    int rank;
    int64_t original_idx, asym, bsym;
    int num_za;
    uint32_t *unique_zas;
    int num_zb;
    uint32_t *unique_zbs;
    double *wa, *wb;
};

template <typename T>
struct Vec {
    T *b, *e, *cap;
    int64_t size() const { return e - b; }
};

struct NetworkOTF32 {
    int64_t num_groups;
    Vec<SVDGroup32> diag_groups, pure_a_groups, pure_b_groups, mixed_groups;
    int64_t *sorted_idxs;
    uint8_t *excit_types;
    int64_t *orbsym;
};

static_assert(sizeof(BlockDesc32) == 56, "BlockDesc<uint32> layout");
static_assert(sizeof(SVDGroup32) == 88, "SVDGroup_OTF<uint32,double> layout");
static_assert(sizeof(Vec<SVDGroup32>) == 24, "std::vector layout");

}  // namespace refmirror
}  // namespace bsim
