// Davidson vector operations and drivers (internal interface).
#pragma once
#include "ops.h"

namespace bsim {

constexpr int kMaxSub = 64;   // subspace limit, as the reference's 64-entry locals (diag/davidson.hpp:41)

struct Coeffs { double v[kMaxSub]; };

// Per-driver scratch for reductions: partials and small device result slots.
// Device scratch of the reductions: part [kDavPartDoubles] (per-CTA partial
// sums) and res [kDavResDoubles].  ensure() allocates it; attach() points it at
// memory the caller owns (then nothing is freed here).
constexpr int kDavPartDoubles = 148 * 8 * kMaxSub;
constexpr int kDavResDoubles = kMaxSub + 8;
struct DavScratch {
    double *part = nullptr;
    double *res = nullptr;
    bool owned = true;
    cudaStream_t stream = nullptr;   // stream of the allocation and of its release
    int ensure(cudaStream_t s = nullptr);
    void attach(double *part_mem, double *res_mem) { part = part_mem; res = res_mem; owned = false; }
    ~DavScratch();
};

template <typename TV>
int dav_ritz_residual(DavScratch &S, i64 n, int k, const double *coeffs, double e, const TV *const *V,
                      const TV *const *AV, double *axt, double *norm_dev, cudaStream_t s);
template <typename TV, typename TX>
int dav_combine(i64 n, int k, const double *coeffs, const TV *const *V, TX *x, cudaStream_t s);
int dav_precondition(DavScratch &S, i64 n, double *r, const double *d, double e, double shift, double *norm_dev,
                     cudaStream_t s);
int dav_precondition(DavScratch &S, i64 n, double *r, const float *d, double e, double shift, double *norm_dev,
                     cudaStream_t s);
template <typename TV>
int dav_mgs(DavScratch &S, i64 n, int k, const TV *const *V, double *v, double *norm_dev, cudaStream_t s);
int dav_normalize(DavScratch &S, i64 n, double *v, double *norm_dev, cudaStream_t s);
int dav_dot(DavScratch &S, i64 n, const double *a, const double *b, double *out_dev, cudaStream_t s);
template <typename TV, typename TW>
int dav_multidot(DavScratch &S, i64 n, int k, const TV *const *V, const TW *w, double *out_dev, cudaStream_t s);

void jacobi_eigh(int k, const double *A, int lda, double *evals, double *evecs);

// Device-scalar helpers of the device-resident drivers (davidson.cu): the
// Ritz coefficients, energy and norms stay on the device.
int dav_eigh_dev(int k, const double *h, int ldh, double *evals, double *evecs, cudaStream_t s);
template <typename TV>
int dav_ritz_residual_dev(DavScratch &S, i64 n, int k, const double *coeffs_dev, const double *e_dev,
                          const TV *const *V, const TV *const *AV, double *r, double *x, double *norm_dev,
                          cudaStream_t s);
template <typename TV, typename TX>
int dav_combine_dev(i64 n, int k, const double *coeffs_dev, const TV *const *V, TX *x, cudaStream_t s);
template <typename TD>
int dav_precondition_dev(DavScratch &S, i64 n, double *r, const TD *d, const double *e_dev,
                         const double *rnorm_dev, double *norm_dev, cudaStream_t s);
template <typename TV>
int dav_cgs2_dev(DavScratch &S, i64 n, int k, const TV *const *V, double *v, double *nrm, double *proj,
                 cudaStream_t s);
template <typename TO>
int dav_normalize_into(i64 n, const double *v, const double *nrm_dev, TO *out, double *breakdown_dev,
                       cudaStream_t s);
int dav_mirror_col(int dim, double *h, int ld, cudaStream_t s);
int dav_sym_avg(int dim, double *h, int ld, cudaStream_t s);
int dav_axpby_dev(i64 n, const double *a_dev, double *x, const double *t, cudaStream_t s);

// Result/statistics of a Davidson run.
struct DavStats {
    double energy;        // converged (or last) Ritz value
    double residual;      // final FP64 residual norm
    int iterations;       // subspace expansions (sigma applications after the first)
    int sigma_fp64;       // FP64 sigma applications
    int sigma_fp32;       // FP32-bulk sigma applications
    int converged;        // 1 if the tolerance was met
};

// Plain FP64 single-root Davidson, jl/davidson.jl:1-185 on device vectors.
// v0 (device, dim) is the start vector (normalised in place); diags (device)
// the Hamiltonian diagonal; x_out (device, dim) receives the Ritz vector.
template <typename Ti>
int davidson_fp64(const DevBasis<Ti> *B, const DevNet<Ti> *N, double *v0, const double *diags, double tol,
                  int maxiter, int ncv, int maxspace, double *x_out, DavStats *stats, int verbose, cudaStream_t s);

// Mixed precision: FP32 subspace storage and FP32-bulk sigma with FP64
// accumulation inside, wrapped in FP64 residual refinement (outer loop on the
// FP64 vector with an FP64 sigma).  Converges on the FP64 residual norm.
template <typename Ti>
int davidson_mixed(const DevBasis<Ti> *B, const DevNet<Ti> *N, double *v0, const double *diags, double tol,
                   int maxiter, int maxspace, double *x_out, DavStats *stats, int verbose, cudaStream_t s);

// Lowest nroots eigenpairs by block Davidson (the reference driver,
// jl/davidson.jl:1-185, generalised to a block of roots; the reference has a
// single-root driver only).  X (device, nroots x dim, root-major) holds the
// start vectors on entry and the Ritz vectors on exit; diag is FP64 or FP32.
constexpr int kMaxRoots = 8;
struct DavBlockStats {
    double energy[kMaxRoots];
    double residual[kMaxRoots];   // FP64 residual norms at exit
    int iterations;               // expansion steps (FP32 phase + refinement)
    int sigma_fp64, sigma_fp32;
    int converged;
};
template <typename Ti>
int davidson_block(const DevBasis<Ti> *B, const DevNet<Ti> *N, int nroots, double *X, const void *diag,
                   bool diag32, double tol, int maxiter, int ncv, int maxspace, bool mixed, DavBlockStats *stats,
                   int verbose, cudaStream_t s);

}  // namespace bsim
