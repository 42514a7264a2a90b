// Structured sigma plan ("fast path") for single-block bases.
//
// Frame.  Determinant phases of the interleaved spin-orbital order (alpha 2p,
// beta 2p+1, reference ham/ham.hpp:402-450) differ from the alpha-first order
// by eps(a, b) = (-1)^{#(alpha electron at i, beta electron at j < i)}
//             = (-1)^{popc(b & K(a))},  K(a) = XOR_{i in a} ((1 << i) - 1).
// With c~ = eps * c the operator becomes H~ = eps H eps; group by group this
// only XORs the Z masks (alpha masks with Ma(bx), beta masks with Mb(ax)) and
// flips the weight sign by (-1)^{popc(ax & Ma(bx))}, where
//   Ma(bx) = alpha orbitals with an odd number of bx bits below them,
//   Mb(ax) = beta orbitals with an odd number of ax bits above them.
// In that frame
//   * a mixed single-single group (ax, bx) factors as
//       PA~(a') = lam * (-1)^{popc(a' & mA[ax])},  PB~(b') = mu * (-1)^{popc(b' & mB[bx])}
//     on connected strings, so the mixed part of sigma is
//       sigma~[a,b] += sum_{E,F} Lam[E,F] sA_E(a^E) sB_F(b^F) c~[a^E, b^F];
//   * a pure-alpha double has a beta factor that is constant in b.
// Every factorisation is verified numerically on all connected strings when
// the plan is built; groups that fail go to the generic tile kernel.
#pragma once
#include "handles.h"

namespace bsim {

// Groups acting on one spin ("row" spin) with a factor on the other ("col")
// spin.  For pure-alpha groups the rows are alpha strings; for pure-beta groups
// the kernels run on the transposed vector, so rows are beta strings.
struct SideDev {
    int ng;              // groups on this side
    int ncols;           // length of the other-spin list
    const u64 *x;        // [ng] row-spin X mask
    const int *rank;     // [ng]
    const int *nz;       // [ng] row-spin Z count
    const i64 *z_off;    // [ng] into zmask
    const i64 *w_off;    // [ng] into w (column-major nz x rank)
    const int *colmode;  // [ng] 0: constant column factor, 1: table
    const double *cconst;  // [ng * kSideMaxRank]
    const i64 *ctab_off;   // [ng] into ctab ([rank][ncols])
    const u64 *zmask;
    const double *w;
    const double *ctab;
    const float *ctab32;
};

constexpr int kSideMaxRank = 4;

// Static list of the pure-spin contributions of every row (depends only on the
// basis and the network): constant-factor entries (source row, coefficient)
// and table entries (source row, group, row-spin phases).
struct SideCSR {
    const i64 *cptr;      // [nrows + 1]
    const int *csrc;      // [nnz_c]
    const double *ccoef;  // [nnz_c]
    const i64 *tptr;      // [nrows + 1]
    const int *tsrc, *tgid;   // [nnz_t]
    const double *tpa;    // [nnz_t * kSideMaxRank]
};

template <typename Ti>
struct FastPlan {
    bool ok = false;
    std::string why;           // reason when the fast path is off
    const void *basis = nullptr;
    i64 basis_dim = -1;
    int norb = 0, nA = 0, nB = 0, nelA = 0, nelB = 0;
    // frame
    std::vector<u64> Ka;       // [nA] eps masks K(a)
    // diagonal D = PAd * PBd^T (tables [n x rank])
    int rank_d = 0;
    // pure sides
    int nPA = 0, nPB = 0;
    // mixed
    int nE = 0, nF = 0, M = 0;         // M = connected alpha singles per row (uniform)
    std::vector<u64> Emask, Fmask, mA, mB;
    std::vector<double> Lam;           // [nE x nF]
    std::vector<int> residual;         // original group ids for the generic kernel
    i64 mixed_pairs = 0;
    bool fits64 = false, fits32 = false;   // mixed GEMM shared memory fits (FP64 / FP32 rows)
    // device
    Arena arena;
    const Ti *d_astr = nullptr, *d_bstr = nullptr;
    const u64 *d_Ka = nullptr;
    const double *d_PAd = nullptr, *d_PBd = nullptr;
    SideDev sideA{}, sideB{};
    SideCSR csrA{}, csrB{};
    i64 nnzA = 0, nnzB = 0;
    const u64 *d_Emask = nullptr, *d_Fmask = nullptr, *d_mA = nullptr, *d_mB = nullptr;
    const double *d_Lam = nullptr;
    const float *d_Lam32 = nullptr;
    const int *d_binom = nullptr;      // [33 x 33] binomials for string ranking
    const int *d_ranktab = nullptr;    // [kRankTabInts] byte tables for string ranking
    const int *d_resid = nullptr;      // residual group plan (for the generic kernel)
    const int4 *d_resid_chunks = nullptr;
    int n_resid_chunks = 0;
    ~FastPlan() { arena.release(); }
};

// Shared memory of the mixed GEMM kernel: source row, Lam_conn [K x 64], an
// X slice [32 x 64], the binomial table and the excitation lists.
// Byte tables for the colex rank of a string: table k covers bits 8k..8k+7
// and is indexed [byte][number of set bits below the byte].
constexpr int kRankTabInts = 256 + 256 * 9 + 256 * 17;   // up to 24 orbitals
constexpr int kMixCols = 128;                             // columns per GEMM chunk

inline size_t mixed_smem_bytes(int nB, int nF, size_t elem)
{
    return (((size_t)nB + 7) & ~size_t(7)) * elem + (size_t)nF * 64 * elem + 32 * (size_t)kMixCols * elem +
           (size_t)kRankTabInts * 4 + kMixCols * 8 + 128 * 4;
}

template <typename Ti>
int build_fast_plan(const DevBasis<Ti> *B, const DevNet<Ti> *N, FastPlan<Ti> *P);

}  // namespace bsim
