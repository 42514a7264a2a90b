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

// Pure groups act on one spin (the "row" spin) with a factor on the other
// (column) spin.  Pure-alpha rows are alpha strings; pure-beta groups run on the
// transposed vector, so their rows are beta strings.
constexpr int kSideMaxRank = 4;

// Static list of the pure-spin contributions of every row (depends only on the
// basis and the network).  Constant-factor entries carry the source row's
// element offset in the padded input and the combined coefficient; table
// entries carry the source offset, the offset of the group's column-factor
// table (rank in the low 3 bits, tables start on multiples of 8) and the
// row-spin phases.
struct CEnt {
    long long off;
    double coef;
};
struct TEnt {
    long long off;
    long long toff_rank;
    double pa[kSideMaxRank];
};

struct SideCSR {
    const i64 *cptr;      // [nrows + 1]
    const CEnt *cent;     // [nnz_c]
    const i64 *tptr;      // [nrows + 1]
    const TEnt *tent;     // [nnz_t]
    const double *ctab;   // column-factor tables, rows padded to ld_in
    const float *ctab32;  // the same in FP32 (FP32-bulk sigma)
};

// Same-spin double excitations through (n-2)-electron intermediate strings m
// (resolution of the identity on one spin):
//   sigma~[a, b] += sum_{pq in a} s(m, pq) sum_{rs not in m} W[pq][rs] s(m, rs) c~[m + rs, b],
//   m = a - pq,  s(m, pq) = <m + pq| a+_p a+_q |m> = (-1)^(#m below p + #m below q).
// Per m the inner sum is a dense (nU x nU) x (nU x columns) product over the nU
// pairs outside m; the outer sum gathers C(n, 2) rows of its result per string.
// W is extracted from the 4-orbital pure groups and verified on every connected
// string pair when the plan is built; a group that does not factor this way
// stays in the row lists.
struct RISide {
    int on = 0;           // the side uses the intermediate-string product
    int nM = 0;           // intermediate strings, C(norb, n - 2)
    int nU = 0;           // pairs outside an intermediate, C(norb - n + 2, 2)
    int npr = 0;          // pairs inside a string, C(n, 2)
    int nP = 0;           // all pairs, C(norb, 2)
    const int *src = nullptr;     // [nM x nU]: (row of m + pair) << 1 | sign
    const int *pid = nullptr;     // [nM x nU]: pair index of each slot
    const int2 *gath = nullptr;   // [nrows x npr]: {m * nU + slot, sign}
    const double *W = nullptr;    // [nP x nP]
    const float *W32 = nullptr;
};

template <typename Ti>
struct FastPlan {
    bool ok = false;
    std::string why;           // reason when the fast path is off
    const void *basis = nullptr;
    i64 basis_dim = -1;
    int norb = 0, nA = 0, nB = 0, nelA = 0, nelB = 0;
    // padded row strides: ldA for rows of c~ (alpha rows, beta columns), ldB for
    // rows of c~^T and of the beta-side result, ldG for the gather-index table
    int ldA = 0, ldB = 0, ldG = 0;
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
    bool row64 = false, row32 = false;     // the mixed GEMM stages the source row in shared memory (FP64 / FP32)
    // device
    Arena arena;
    const Ti *d_astr = nullptr, *d_bstr = nullptr;
    const u64 *d_Ka = nullptr;
    const double *d_PAd = nullptr;     // [nA x rank_d] alpha diagonal factors
    SideCSR csrA{}, csrB{};
    SideCSR csrBri{};                  // beta rows without the intermediate-string groups
    RISide riA{}, riB{};
    i64 nnzA = 0, nnzB = 0;
    const u64 *d_Emask = nullptr, *d_mA = nullptr;
    const double *d_Lam = nullptr;
    const float *d_Lam32 = nullptr;
    const double *d_PBdT = nullptr;    // [rank_d x ldA] beta diagonal factors, transposed
    const int *d_gidx = nullptr;       // [nF x ldG] (rank(b^F) << 1 | sign) or -1
    const int *d_resid = nullptr;      // residual group plan (for the generic kernel)
    const int4 *d_resid_chunks = nullptr;
    int n_resid_chunks = 0;
    ~FastPlan() { arena.release(); }
};

constexpr int kMixCols = 128;                             // columns per GEMM chunk

// Shared memory of the intermediate-string GEMM: W_m [nU x ri_ls] and a ring of
// X slices.
// Output rows past 64 (up to kRiMaxU) are computed by all threads with scalar
// FMAs next to the 64-row register tiles, so W_m rows are 8 elements wider
// than the mixed GEMM's Lam_conn rows (72 / 76 elements: 4 mod 16 doubles for
// the FP64 fragments' banks).
constexpr int kRiMaxU = 72;
inline size_t gemm_ls(size_t elem) { return elem == 8 ? 68 : 64; }
inline size_t gemm_xs(size_t elem) { return elem == 8 ? kMixCols + 4 : kMixCols; }
inline size_t ri_ls(size_t elem) { return gemm_ls(elem) + 8; }
constexpr int kRiStagesHost = 3;   // X slices in the cp.async ring of the intermediate-string GEMM
inline size_t ri_smem_bytes(int nU, size_t elem)
{
    return (((size_t)nU + 7) & ~size_t(7)) * ri_ls(elem) * elem + kRiStagesHost * 32 * gemm_xs(elem) * elem +
           kRiMaxU * 8;
}

// Shared memory of the mixed GEMM kernel: source row (unless it is read from
// global memory), Lam_conn [K x 64] (or one 32-row F chunk of it), an X slice
// [32 x kMixCols] and the connected-excitation lists.
constexpr int kMaxConn = 128;   // connected alpha singles per string: up to two 64-row GEMM passes
constexpr size_t kSmemMax = 227 * 1024;

// rows: connected excitations per GEMM pass (64, or 80 for the FP32 80-row tile,
// whose Lam_conn rows are 80 elements long)
inline size_t mixed_smem_bytes(int nB, int nF, size_t elem, bool stream, bool grow, int rows = 64)
{
    const size_t lam_rows = stream ? 32 : (((size_t)nF + 7) & ~size_t(7));
    const size_t ls = rows > 64 ? (size_t)rows : gemm_ls(elem);
    return (grow ? 0 : (((size_t)nB + 7) & ~size_t(7)) * elem) + lam_rows * ls * elem +
           32 * gemm_xs(elem) * elem + 2 * kMaxConn * 4;
}

// Kernel shape of the mixed GEMM: the source row is staged in shared memory
// when it fits under row_limit (Lam_conn streamed per F chunk if needed), else
// the X gather reads it from global memory (an 18-orbital FP64 row is 350 KB).
struct MixedShape {
    bool stream, grow;
    size_t smem;
};
inline MixedShape mixed_shape(int nB, int nF, size_t elem, size_t row_limit, int rows = 64)
{
    const size_t lim = row_limit < kSmemMax ? row_limit : kSmemMax;
    for (int grow = 0; grow < 2; ++grow)
        for (int stream = 0; stream < 2; ++stream) {
            const size_t b = mixed_smem_bytes(nB, nF, elem, stream, grow, rows);
            if (b <= (grow ? kSmemMax : lim)) return MixedShape{stream != 0, grow != 0, b};
        }
    return MixedShape{true, true, mixed_smem_bytes(nB, nF, elem, true, true, rows)};
}

template <typename Ti>
int build_fast_plan(const DevBasis<Ti> *B, const DevNet<Ti> *N, FastPlan<Ti> *P);

}  // namespace bsim
