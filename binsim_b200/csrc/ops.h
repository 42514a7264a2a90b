// Internal operation entry points of libcuotf (the C-ABI in capi.cu wraps them).
#pragma once
#include "handles.h"

namespace bsim {

template <typename Ti>
inline Workspace &workspace_for(const DevBasis<Ti> *B) { return B->ws; }

// sigma = H src (dst overwritten).  mixed: FP32 bulk, FP64 accumulation; src32
// may carry an FP32 copy of the input (else one is made in the workspace).
template <typename Ti>
int sigma(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *src, const float *src32, double *dst,
          bool mixed, cudaStream_t s);

// As sigma, restricted to flat tiles [tile_lo, tile_hi) (32-row x 32-column
// destination tiles, block-major then row-major); other elements untouched.
template <typename Ti>
int sigma_tiles(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *src, const float *src32, double *dst,
                bool mixed, i64 tile_lo, i64 tile_hi, cudaStream_t s);
template <typename Ti>
i64 num_tiles(const DevBasis<Ti> *B);

// Structured sigma (single-block bases); *used tells whether it ran.
template <typename Ti>
int sigma_fast(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *src, const float *src32, double *dst,
               bool mixed, cudaStream_t s, bool *used);
// 1: structured path (FP64 and FP32), 2: structured for FP32 only, 0: generic.
// Columns [col_lo, col_hi) of sigma through the structured path (col_lo a
// multiple of 128): the unit of work of one rank when sigma is split by beta
// columns.  Every other element of dst is left untouched.
template <typename Ti>
int sigma_fast_cols(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *src, double *dst, bool mixed,
                    i64 col_lo, i64 col_hi, cudaStream_t s);

// One structured sigma with CUDA events around every launch: per-stage device
// milliseconds and launch counts (stages as in sigma_fast.cu's StageTimer).
template <typename Ti>
int sigma_fast_stages(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *src, double *dst, bool mixed,
                      cudaStream_t s, double *ms, int *launches, int nstages);

// Arithmetic peak of the CUDA cores (FMA chains), TFLOP/s, FP64 or FP32.
int fma_peak(int mode, double *tflops, cudaStream_t s);   // 0 FP32 FMA, 1 FP64 FMA, 2 FP64 DMMA

template <typename Ti>
int fast_sigma_info(const DevBasis<Ti> *B, const DevNet<Ti> *N, std::string *why, int *nresid);
template <typename Ti>
bool fast_sigma_available(const DevBasis<Ti> *B, const DevNet<Ti> *N);
// The generic tile kernel over an explicit chunk plan, adding into dst.
template <typename Ti>
int sigma_generic_accumulate(const DevBasis<Ti> *B, const DevNet<Ti> *N, const int *plan_g, const int4 *chunks,
                             int nchunks, const double *src, const float *src32, double *dst, bool mixed,
                             cudaStream_t s);

template <typename Ti>
int diag_elements(const DevBasis<Ti> *B, const DevNet<Ti> *N, double *diag, cudaStream_t s);

template <typename Ti>
int tile_prefix(const DevBasis<Ti> *B, Workspace &ws, const i64 **out_dev, i64 *ntiles);

// Single-generator pair operators (original group index gidx).
//   expm:     v <- exp(theta G) v
//   grad:     *out_dev = <l, G e^{theta G}>(r) in the reference orientation
//   backgrad: l <- e^{-theta G} l ; *out_dev = grad term ; r <- e^{-theta G} r
// out_dev is a device double; with accumulate the term is added to it.
template <typename Ti>
int expm(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, double theta, double *v, cudaStream_t s);
template <typename Ti>
int grad(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, double theta, const double *l, const double *r,
         double *out_dev, bool accumulate, cudaStream_t s, double *scratch = nullptr, size_t scratch_n = 0);
template <typename Ti>
int backgrad(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, double theta, double *l, double *r,
             double *out_dev, bool accumulate, cudaStream_t s);

// Pool gradient: grads[orig] = grad of every group at thetas[orig] (device arrays).
// Single-group operators of the reference CPU library without a GPU
// counterpart there (op/tvec.hpp, op/backtran.hpp, op/batchexpm.hpp,
// op/batchtran.hpp): dst = T src; l, r <- e^{theta T}; b = T l; e^{theta T} on
// nv columns of a row-major dim x ld matrix; <l|T_g|r> for every group.
template <typename Ti>
int tvec(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, const double *src, double *dst, cudaStream_t s);
template <typename Ti>
int backtran(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, double theta, double *l, double *r, double *b,
             cudaStream_t s);
template <typename Ti>
int batchexpm(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, double theta, double *matrix, int ld, int nv,
              cudaStream_t s);
template <typename Ti>
int batchtran(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *l, const double *r, double *trans,
              cudaStream_t s);
template <typename Ti>
int batchgrad(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *thetas, const double *l,
              const double *r, double *grads, cudaStream_t s);

// Number of CTAs the row-pair kernels launch (size of their partial-sum scratch).
template <typename Ti>
inline i64 pair_grid(const DevBasis<Ti> *B) { return (i64)B->max_na * B->num_blocks; }

// Angle terms of the pair updates (core/math.hpp:132-215).
struct PairAngles { double c0, c1, c2, c3; };
enum PairOpKind { kPairExpm = 0, kPairGrad = 1, kPairBackgrad = 2, kPairTvec = 3, kPairBacktran = 4, kPairTran = 5,
                  kPairBatchExpm = 6 };

// Gradients of every group of a pool network in one launch over the pair lists
// (single-block bases, ranks <= 4); *used = false when the tile kernel must run.
// skip / flag (device, may be null): when *flag is nonzero the groups with
// skip[orig] set are left out (the theta = 0 density route computes them).
template <typename Ti>
int pair_list_batchgrad(const DevBasis<Ti> *B, const DevNet<Ti> *N, const double *thetas, const double *l,
                        const double *r, double *grads, cudaStream_t s, bool *used,
                        const unsigned char *skip = nullptr, const int *flag = nullptr);

// Theta = 0 route of the pool gradient through transition densities
// (pooldensity.cu), built on first use for (basis, network) and cached on the
// network; *out = nullptr when it does not apply (complex weights, no groups
// of the planned forms, tables too large).  begin: device flag = every theta
// is zero; the flag and the per-group skip mask are then handed to the
// pair-list / tile kernels; finish: the density kernels, which run only when
// the flag is set, overwrite grads of the planned groups.
struct DensityRoute;
template <typename Ti>
int density_route(const DevBasis<Ti> *B, const DevNet<Ti> *N, DensityRoute **out);
int density_route_begin(DensityRoute *D, const double *thetas, cudaStream_t s);
template <typename Ti>
int density_route_finish(DensityRoute *D, const double *l, const double *r, double *grads, cudaStream_t s);
const unsigned char *density_route_skip(const DensityRoute *D);
const int *density_route_flag(const DensityRoute *D);

// Pair operator over the precomputed pair lists (single-block bases, rank <= 4).
// Sets *used = false (and launches nothing) when the row kernel must serve the
// call.  grad/backgrad write at most max_slots partials before the ticket.
// may_build = false: use the lists only if they exist already (building them
// allocates device memory); otherwise leave the call to the row kernel.
template <typename Ti, int OP>
int pair_list_launch(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, PairAngles ang, double *l, double *r,
                     double *part, unsigned long long *ticket, i64 max_slots, double *out, bool accumulate,
                     cudaStream_t s, bool *used, bool may_build = true);

}  // namespace bsim
