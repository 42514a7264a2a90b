// Block Davidson for the lowest nroots eigenpairs, device resident.
//
// The reference driver (jl/davidson.jl:1-185, steps of diag/davidson.hpp:31-272)
// follows one root; this driver applies the same steps to a block of roots:
// Rayleigh-Ritz on the host (FP64 Jacobi, <= 64 x 64), per unconverged root the
// Ritz residual, the preconditioner r / (d - e_i) clamped at
// max(1e-2 |r_i|, 1e-4), modified Gram-Schmidt (repeated when the norm drops
// below 0.717 of its value), normalisation and one sigma, and a restart to ncv
// Ritz vectors when the subspace is full.  The restart rotates the subspace in
// place (one pass that reads every vector's element i and writes the ncv new
// elements i), so no second set of vectors is held.
//
// Mixed precision (FP32 subspace, FP32-bulk sigma with FP64 accumulation)
// runs the block loop on FP32 storage until every FP32 residual is below tol or
// the largest stops improving, forms the FP64 Ritz vectors, and refines them:
// FP64 sigma of each root, FP64 Rayleigh-Ritz among the roots, FP64 residuals,
// and while any is above tol an FP32 correction space whose couplings to the
// roots come from the FP64 sigmas.  The roots keep FP64 precision; only the
// corrections carry FP32 rounding.  The refinement's subspace is sized from
// the device memory left after the FP32 phase releases its vectors.
#include "dav.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace bsim {

namespace {

constexpr int kRotMax = kMaxRoots;   // vectors written by one in-place rotation

// Device vector from cudaMalloc (released eagerly between phases).
struct Vec {
    void *p = nullptr;
    Vec() = default;
    Vec(const Vec &) = delete;
    Vec &operator=(const Vec &) = delete;
    ~Vec() { reset(); }
    void reset()
    {
        if (p) cudaFree(p);
        p = nullptr;
    }
    int alloc(size_t bytes)
    {
        reset();
        cudaError_t e = dmalloc(&p, std::max<size_t>(bytes, 1));
        if (e != cudaSuccess) { p = nullptr; return cuda_status(e, "block davidson vector"); }
        return BSIM_OK;
    }
};

template <typename TV>
struct VP { TV *p[kMaxSub]; };

// V_c[i] <- sum_j Y[j + c * dim] V_j[i] for c < ncv (in place: each thread reads
// every input element i before it writes the outputs at i)
template <typename TV>
__global__ void rotate_kernel(i64 n, int dim, int ncv, const double *__restrict__ Y, VP<TV> V)
{
    __shared__ double sy[kMaxSub * kRotMax];
    for (int t = threadIdx.x; t < dim * ncv; t += blockDim.x) sy[t] = Y[t];
    __syncthreads();
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        double acc[kRotMax];
#pragma unroll
        for (int c = 0; c < kRotMax; ++c) acc[c] = 0.0;
        for (int j = 0; j < dim; ++j) {
            const double v = (double)V.p[j][i];
#pragma unroll
            for (int c = 0; c < kRotMax; ++c)
                if (c < ncv) acc[c] += sy[j + c * dim] * v;
        }
#pragma unroll
        for (int c = 0; c < kRotMax; ++c)
            if (c < ncv) V.p[c][i] = (TV)acc[c];
    }
}

__global__ void d2f_kernel(const double *__restrict__ x, float *__restrict__ y, i64 n)
{
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) y[i] = (float)x[i];
}

// Ritz residual in the refinement's space, FP64 roots and FP32 corrections:
// r = sum_{j<k} a_j (AX_j - e X_j) + sum_{j<m} b_j (AV_j - e V_j).  Near
// convergence the corrections' coefficients are small, so the FP32-bulk
// rounding of AV_j stays far below the residual.
struct RootPtrs { const double *x[kMaxRoots], *ax[kMaxRoots]; double a[kMaxRoots]; };
struct CorrPtrs { const float *v[kMaxSub], *av[kMaxSub]; double b[kMaxSub]; };
__global__ void split_residual_kernel(i64 n, int k, RootPtrs R, int m, CorrPtrs Cp, double e, double *__restrict__ r)
{
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int j = 0; j < k; ++j) acc += R.a[j] * (R.ax[j][i] - e * R.x[j][i]);
        double cor = 0.0;
        for (int j = 0; j < m; ++j) cor += Cp.b[j] * ((double)Cp.av[j][i] - e * (double)Cp.v[j][i]);
        r[i] = acc + cor;
    }
}

// x += t
__global__ void add_kernel(i64 n, double *__restrict__ x, const double *__restrict__ t)
{
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) x[i] += t[i];
}

constexpr int kGrid = 148 * 8;

#define TRY(...) do { int st__ = (__VA_ARGS__); if (st__ != BSIM_OK) return st__; } while (0)

int fetch(double *host, const double *dev, int n, cudaStream_t s)
{
    BSIM_CUDA(cudaMemcpyAsync(host, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    BSIM_CUDA(cudaStreamSynchronize(s));
    return BSIM_OK;
}

// Subspace of one block loop: vectors, projected matrix and its eigenpairs.
template <typename TV>
struct Space {
    std::vector<TV *> V, AV;
    int dim = 0;
    double h[kMaxSub * kMaxSub];
    double es[kMaxSub], vs[kMaxSub * kMaxSub];
    // the previous step's Ritz vectors in subspace coordinates (pdim rows), kept
    // at a restart next to the current ones
    int pdim = 0;
    double pvs[kMaxSub * kMaxRoots];
    void eig() { jacobi_eigh(dim, h, kMaxSub, es, vs); }
    void save(int k)
    {
        pdim = dim;
        for (int c = 0; c < k; ++c)
            for (int j = 0; j < dim; ++j) pvs[j + c * kMaxSub] = vs[j + (size_t)c * dim];
    }
    // Restart basis in subspace coordinates: the ncv lowest Ritz vectors, then
    // the previous step's k Ritz vectors orthogonalised against them (GD+k:
    // Stathopoulos & Saad, 1998), at most room columns.  Returns the count.
    int restart_basis(int ncv, int k, int room, double *Y) const
    {
        int nc = 0;
        for (int c = 0; c < std::min(ncv, dim); ++c, ++nc)
            for (int j = 0; j < dim; ++j) Y[j + nc * dim] = vs[j + (size_t)c * dim];
        for (int c = 0; c < k && pdim > 0 && nc < room; ++c) {
            double *y = Y + nc * dim;
            for (int j = 0; j < dim; ++j) y[j] = j < pdim ? pvs[j + c * kMaxSub] : 0.0;
            double nrm = 0.0;
            for (int pass = 0; pass < 2; ++pass)
                for (int q = 0; q < nc; ++q) {
                    double d = 0.0;
                    for (int j = 0; j < dim; ++j) d += Y[j + q * dim] * y[j];
                    for (int j = 0; j < dim; ++j) y[j] -= d * Y[j + q * dim];
                }
            for (int j = 0; j < dim; ++j) nrm += y[j] * y[j];
            nrm = std::sqrt(nrm);
            if (nrm < 1e-3) continue;   // the previous vector is (nearly) in the span already
            for (int j = 0; j < dim; ++j) y[j] /= nrm;
            ++nc;
        }
        return nc;
    }
};

// Shared state of one driver call.
template <typename Ti>
struct Ctx {
    const DevBasis<Ti> *B;
    const DevNet<Ti> *N;
    i64 n;
    int k;
    const void *diag;
    bool diag32;
    double tol;
    int verbose;
    cudaStream_t s;
    DavScratch S;
    double *dY = nullptr;   // rotation coefficients on the device
    DavBlockStats st{};
    ~Ctx() { if (dY) cudaFree(dY); }

    int precondition(double *t, double e, double shift, double *norm_dev)
    {
        return diag32 ? dav_precondition(S, n, t, static_cast<const float *>(diag), e, shift, norm_dev, s)
                      : dav_precondition(S, n, t, static_cast<const double *>(diag), e, shift, norm_dev, s);
    }

    // V[0..ncv) <- V[0..dim) Y[:, 0..ncv)  (Y column-major with leading dimension ldy)
    template <typename TV>
    int rotate(TV *const *V, int dim, int ncv, const double *Y, int ldy)
    {
        if (ncv > kRotMax) { set_error("in-place rotation of %d > %d vectors", ncv, kRotMax); return BSIM_ERR_ARG; }
        double y[kMaxSub * kRotMax];
        for (int c = 0; c < ncv; ++c)
            for (int j = 0; j < dim; ++j) y[j + c * dim] = Y[j + (size_t)c * ldy];
        if (!dY) BSIM_CUDA(dmalloc(&dY, sizeof(double) * kMaxSub * kRotMax));
        BSIM_CUDA(cudaMemcpyAsync(dY, y, sizeof(double) * dim * ncv, cudaMemcpyHostToDevice, s));
        BSIM_CUDA(cudaStreamSynchronize(s));   // y is a host local
        VP<TV> p{};
        for (int j = 0; j < dim; ++j) p.p[j] = V[j];
        rotate_kernel<TV><<<kGrid, 256, 0, s>>>(n, dim, ncv, dY, p);
        BSIM_CUDA(cudaGetLastError());
        return BSIM_OK;
    }

    // h[0..dim) x [0..dim) = <V_i | AV_j>, symmetrised (davidson.hpp:221-272)
    template <typename TV>
    int rebuild(Space<TV> &W)
    {
        double col[kMaxSub];
        for (int j = 0; j < W.dim; ++j) {
            TRY(dav_multidot<TV, TV>(S, n, W.dim, W.V.data(), W.AV[j], S.res, s));
            TRY(fetch(col, S.res, W.dim, s));
            for (int i = 0; i < W.dim; ++i) W.h[i + j * kMaxSub] = col[i];
        }
        for (int j = 0; j < W.dim; ++j)
            for (int i = 0; i < j; ++i)
                W.h[i + j * kMaxSub] = W.h[j + i * kMaxSub] = 0.5 * (W.h[i + j * kMaxSub] + W.h[j + i * kMaxSub]);
        return BSIM_OK;
    }

    // Ritz residual norms of the k lowest roots (the residual of the last root
    // stays in t)
    template <typename TV>
    int norms(Space<TV> &W, double *t, double *nr)
    {
        for (int i = 0; i < k; ++i) {
            TRY(dav_ritz_residual<TV>(S, n, W.dim, W.vs + (size_t)i * W.dim, W.es[i], W.V.data(), W.AV.data(), t,
                                      S.res + kMaxSub, s));
            TRY(fetch(&nr[i], S.res + kMaxSub, 1, s));
        }
        return BSIM_OK;
    }

    // Preconditions t for Ritz value e, orthogonalises it against V[0..dim) and
    // normalises it; returns whether a direction is left.
    template <typename TV>
    int correction(TV *const *V, int dim, double *t, double e, double rnorm, bool *ok)
    {
        double *sc = S.res + kMaxSub;
        double nrm[2];
        TRY(precondition(t, e, std::max(rnorm * 1e-2, 1e-4), sc));
        TRY(fetch(&nrm[0], sc, 1, s));
        TRY(dav_mgs<TV>(S, n, dim, V, t, sc + 1, s));
        TRY(fetch(&nrm[1], sc + 1, 1, s));
        if (nrm[1] < 0.717 * nrm[0]) {
            TRY(dav_mgs<TV>(S, n, dim, V, t, sc + 1, s));
            TRY(fetch(&nrm[1], sc + 1, 1, s));
        }
        *ok = nrm[1] >= 1e-12;
        if (*ok) TRY(dav_normalize(S, n, t, sc, s));
        return BSIM_OK;
    }

    // sigma of the new subspace vector V[dim] into AV[dim]; t is free (FP32
    // storage: it receives the FP64 sigma before the conversion)
    int apply(double *v, double *av, double *) { st.sigma_fp64++; return sigma(B, N, v, nullptr, av, false, s); }
    int apply(float *v, float *av, double *t)
    {
        st.sigma_fp32++;
        TRY(sigma(B, N, nullptr, v, t, true, s));
        d2f_kernel<<<kGrid, 256, 0, s>>>(t, av, n);
        BSIM_CUDA(cudaGetLastError());
        return BSIM_OK;
    }
    static int store(double *dst, const double *t, i64 n, cudaStream_t s)
    {
        BSIM_CUDA(cudaMemcpyAsync(dst, t, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        return BSIM_OK;
    }
    static int store(float *dst, const double *t, i64 n, cudaStream_t s)
    {
        d2f_kernel<<<kGrid, 256, 0, s>>>(t, dst, n);
        BSIM_CUDA(cudaGetLastError());
        return BSIM_OK;
    }

    // r (and its norm) of Ritz pair (y, e) of the refinement space W, whose first
    // k vectors stand for the FP64 roots X (sigmas AX)
    int split_residual(const Space<float> &W, const double *y, double e, double *const *X, double *const *AX,
                       double *r, double *norm)
    {
        RootPtrs R{};
        CorrPtrs Cp{};
        for (int j = 0; j < k; ++j) { R.x[j] = X[j]; R.ax[j] = AX[j]; R.a[j] = y[j]; }
        const int m = W.dim - k;
        for (int j = 0; j < m; ++j) { Cp.v[j] = W.V[k + j]; Cp.av[j] = W.AV[k + j]; Cp.b[j] = y[k + j]; }
        split_residual_kernel<<<kGrid, 256, 0, s>>>(n, k, R, m, Cp, e, r);
        BSIM_CUDA(cudaGetLastError());
        double *sc = S.res + kMaxSub;
        TRY(dav_dot(S, n, r, r, sc, s));
        double rr = 0.0;
        TRY(fetch(&rr, sc, 1, s));
        *norm = std::sqrt(std::max(rr, 0.0));
        return BSIM_OK;
    }

    // Appends V[dim] = t (normalised correction) and AV[dim] = H t, and extends h.
    template <typename TV>
    int append(Space<TV> &W, double *t)
    {
        TRY(store(W.V[W.dim], t, n, s));
        TRY(apply(W.V[W.dim], W.AV[W.dim], t));
        ++W.dim;
        double col[kMaxSub];
        TRY(dav_multidot<TV, TV>(S, n, W.dim, W.V.data(), W.AV[W.dim - 1], S.res, s));
        TRY(fetch(col, S.res, W.dim, s));
        for (int i = 0; i < W.dim; ++i) W.h[i + (W.dim - 1) * kMaxSub] = W.h[(W.dim - 1) + i * kMaxSub] = col[i];
        return BSIM_OK;
    }
};

}  // namespace

// The block loop on one subspace.  Returns when every root's residual is below
// tol, after maxiter expansion steps in total, when no correction direction is
// left, or (stall > 0) when the largest residual has not improved for `stall`
// steps (the FP32 noise floor).  nr receives the residual norms of the last
// Rayleigh-Ritz step.
template <typename Ti, typename TV>
static int block_loop(Ctx<Ti> &C, Space<TV> &W, int maxspace, int ncv, int maxiter, int stall, double *t, double *nr,
                      bool *converged, const char *tag)
{
    const int k = C.k;
    double best = 1e300;
    int since = 0;
    *converged = false;
    for (int iter = 1;; ++iter) {
        W.eig();
        TRY(C.norms(W, t, nr));
        double rmax = 0.0;
        int nnew = 0;
        for (int i = 0; i < k; ++i) {
            rmax = std::max(rmax, nr[i]);
            nnew += nr[i] >= C.tol;
        }
        if (C.verbose) {
            printf("  %s step %03d dim %2d:", tag, iter, W.dim);
            for (int i = 0; i < k; ++i) printf("  %.3e %.12f", nr[i], W.es[i]);
            printf("\n");
        }
        if (nnew == 0) { *converged = true; return BSIM_OK; }
        if (rmax < best) { best = rmax; since = 0; }
        else ++since;
        if (C.st.iterations >= maxiter || (stall > 0 && since >= stall)) return BSIM_OK;
        if (W.dim + nnew > maxspace) {   // restart: ncv Ritz vectors (the k roots among them) + previous ones
            double Y[kMaxSub * kRotMax];
            const int keep = W.restart_basis(ncv, k, std::min(maxspace - nnew, kRotMax), Y);
            TRY(C.rotate(W.V.data(), W.dim, keep, Y, W.dim));
            TRY(C.rotate(W.AV.data(), W.dim, keep, Y, W.dim));
            W.dim = keep;
            TRY(C.rebuild(W));
            W.eig();
        }
        W.save(k);
        const int d0 = W.dim;
        bool any = false;
        for (int i = 0; i < k; ++i) {
            if (nr[i] < C.tol) continue;
            TRY(dav_ritz_residual<TV>(C.S, C.n, d0, W.vs + (size_t)i * d0, W.es[i], W.V.data(), W.AV.data(), t,
                                      C.S.res + kMaxSub, C.s));
            bool ok = false;
            TRY(C.correction(W.V.data(), W.dim, t, W.es[i], nr[i], &ok));
            if (!ok) continue;
            TRY(C.append(W, t));
            any = true;
        }
        C.st.iterations++;
        if (!any) return BSIM_OK;
    }
}

template <typename Ti>
static int block_fp64(Ctx<Ti> &C, std::vector<double *> &Xp, int maxiter, int ncv, int maxspace)
{
    const i64 n = C.n;
    const int k = C.k;
    Space<double> W;
    W.V.assign(maxspace, nullptr);
    W.AV.assign(maxspace, nullptr);
    std::vector<Vec> own(2 * maxspace);
    for (int j = 0; j < maxspace; ++j) {
        if (j < k) W.V[j] = Xp[j];   // the roots live in the caller's buffers
        else { TRY(own[j].alloc(sizeof(double) * n)); W.V[j] = (double *)own[j].p; }
        TRY(own[maxspace + j].alloc(sizeof(double) * n));
        W.AV[j] = (double *)own[maxspace + j].p;
    }
    Vec tb;
    TRY(tb.alloc(sizeof(double) * n));
    double *t = (double *)tb.p;
    for (int j = 0; j < k; ++j) TRY(C.apply(W.V[j], W.AV[j], t));
    W.dim = k;
    TRY(C.rebuild(W));
    double nr[kMaxRoots];
    bool conv = false;
    TRY(block_loop(C, W, maxspace, ncv, maxiter, 0, t, nr, &conv, "fp64"));
    (void)conv;
    W.eig();
    TRY(C.norms(W, t, nr));
    TRY(C.rotate(W.V.data(), W.dim, k, W.vs, W.dim));   // Ritz vectors into X
    for (int i = 0; i < k; ++i) {
        C.st.energy[i] = W.es[i];
        C.st.residual[i] = nr[i];
    }
    C.st.converged = 1;
    for (int i = 0; i < k; ++i) C.st.converged &= nr[i] < C.tol;
    BSIM_CUDA(cudaStreamSynchronize(C.s));
    return BSIM_OK;
}

template <typename Ti>
static int block_mixed(Ctx<Ti> &C, std::vector<double *> &Xp, int maxiter, int ncv, int maxspace)
{
    const i64 n = C.n;
    const int k = C.k;
    double nr[kMaxRoots];
    // ---- phase A: block loop on FP32 storage with the FP32-bulk sigma ----
    std::vector<Vec> own(2 * maxspace);
    std::vector<float *> V32(maxspace), AV32(maxspace);
    for (int j = 0; j < maxspace; ++j) {
        TRY(own[j].alloc(sizeof(float) * n));
        TRY(own[maxspace + j].alloc(sizeof(float) * n));
        V32[j] = (float *)own[j].p;
        AV32[j] = (float *)own[maxspace + j].p;
    }
    {
        Space<float> W;
        W.V = V32;
        W.AV = AV32;
        double *t = Xp[0];   // the start vectors are copied out first; X is scratch until the Ritz vectors
        for (int j = 0; j < k; ++j) TRY(C.store(W.V[j], Xp[j], n, C.s));
        for (int j = 0; j < k; ++j) TRY(C.apply(W.V[j], W.AV[j], t));
        W.dim = k;
        TRY(C.rebuild(W));
        bool conv = false;
        TRY(block_loop(C, W, maxspace, ncv, maxiter, maxspace, t, nr, &conv, "fp32"));
        W.eig();
        for (int i = 0; i < k; ++i)
            TRY(dav_combine<float, double>(n, W.dim, W.vs + (size_t)i * W.dim, W.V.data(), Xp[i], C.s));
    }
    // ---- phase B: FP64 refinement of the block ----
    // The FP32 subspace is released; the correction space is sized after the
    // first FP64 sigmas, from the memory the FP64 vectors and the FP64 sigma's
    // scratch leave (a block that fits no correction space stops after the
    // FP64 residual check, with converged = 0 if a residual is above tol).
    BSIM_CUDA(cudaStreamSynchronize(C.s));
    for (auto &v : own) v.reset();
    int mB = 0;
    std::vector<Vec> axb(k);
    std::vector<double *> AX(k);
    for (int j = 0; j < k; ++j) { TRY(axb[j].alloc(sizeof(double) * n)); AX[j] = (double *)axb[j].p; }
    Vec tb;
    TRY(tb.alloc(sizeof(double) * n));
    double *t = (double *)tb.p;
    double *sc = C.S.res + kMaxSub;
    double hx[kMaxSub * kMaxSub], ex[kMaxSub], yx[kMaxSub * kMaxSub], col[kMaxSub], unit[kMaxRoots];
    bool conv = false;
    for (int outer = 0;; ++outer) {
        // orthonormal FP64 roots, their FP64 sigmas, Rayleigh-Ritz among them
        for (int j = 0; j < k; ++j) {
            double nrm = 0.0;
            TRY(dav_mgs<double>(C.S, n, j, Xp.data(), Xp[j], sc, C.s));
            TRY(fetch(&nrm, sc, 1, C.s));
            if (nrm < 1e-12) { set_error("refined roots became linearly dependent"); return BSIM_ERR_ARG; }
            TRY(dav_normalize(C.S, n, Xp[j], sc, C.s));
        }
        for (int j = 0; j < k; ++j) TRY(C.apply(Xp[j], AX[j], t));
        for (int j = 0; j < k; ++j) {
            TRY(dav_multidot<double, double>(C.S, n, k, Xp.data(), AX[j], C.S.res, C.s));
            TRY(fetch(col, C.S.res, k, C.s));
            for (int i = 0; i < k; ++i) hx[i + j * kMaxSub] = col[i];
        }
        for (int j = 0; j < k; ++j)
            for (int i = 0; i < j; ++i) hx[i + j * kMaxSub] = hx[j + i * kMaxSub] = 0.5 * (hx[i + j * kMaxSub] + hx[j + i * kMaxSub]);
        jacobi_eigh(k, hx, kMaxSub, ex, yx);
        TRY(C.rotate(Xp.data(), k, k, yx, k));
        TRY(C.rotate(AX.data(), k, k, yx, k));
        int nnew = 0;
        for (int i = 0; i < k; ++i) {
            for (int j = 0; j < k; ++j) unit[j] = i == j ? 1.0 : 0.0;
            TRY(dav_ritz_residual<double>(C.S, n, k, unit, ex[i], Xp.data(), AX.data(), t, sc, C.s));
            TRY(fetch(&nr[i], sc, 1, C.s));
            C.st.energy[i] = ex[i];
            C.st.residual[i] = nr[i];
            nnew += nr[i] >= C.tol;
        }
        if (C.verbose) {
            printf("  fp64 refinement %02d:", outer);
            for (int i = 0; i < k; ++i) printf("  %.3e %.12f", nr[i], ex[i]);
            printf("\n");
        }
        if (nnew == 0) { conv = true; break; }
        if (C.st.iterations >= maxiter) break;
        if (mB == 0) {
            BSIM_CUDA(cudaStreamSynchronize(C.s));
            size_t fr = 0, tot = 0;
            BSIM_CUDA(cudaMemGetInfo(&fr, &tot));
            const double pair = 8.0 * (double)n;   // one FP32 vector and its FP32 sigma
            mB = (int)std::min<double>(maxspace, std::floor(((double)fr - 1e9) / pair));
            if (mB < 2 * k) {
                if (C.verbose) printf("  no memory for the FP32 correction space (%d pairs)\n", mB);
                break;
            }
            for (int j = 0; j < mB; ++j) {
                TRY(own[j].alloc(sizeof(float) * n));
                TRY(own[maxspace + j].alloc(sizeof(float) * n));
                V32[j] = (float *)own[j].p;
                AV32[j] = (float *)own[maxspace + j].p;
            }
        }
        // ---- FP32 correction space around the FP64 roots ----
        Space<float> W;
        W.V.assign(V32.begin(), V32.begin() + mB);
        W.AV.assign(AV32.begin(), AV32.begin() + mB);
        for (int j = 0; j < k; ++j) {
            TRY(C.store(W.V[j], Xp[j], n, C.s));
            TRY(C.store(W.AV[j], AX[j], n, C.s));
        }
        W.dim = k;
        for (int j = 0; j < k; ++j)
            for (int i = 0; i < k; ++i) W.h[i + j * kMaxSub] = i == j ? ex[i] : 0.0;
        double rin[kMaxRoots], target[kMaxRoots];
        for (int i = 0; i < k; ++i) { rin[i] = nr[i]; target[i] = std::max(0.05 * nr[i], 0.5 * C.tol); }
        for (int pass = 0;; ++pass) {
            int want = 0;
            for (int i = 0; i < k; ++i) want += rin[i] >= target[i];
            if (want == 0 || W.dim + want > mB || (pass > 0 && C.st.iterations >= maxiter)) break;
            const int d0 = W.dim;
            bool any = false;
            for (int i = 0; i < k; ++i) {
                if (rin[i] < target[i]) continue;
                if (pass == 0) {   // the exact FP64 residual of root i
                    for (int j = 0; j < k; ++j) unit[j] = i == j ? 1.0 : 0.0;
                    TRY(dav_ritz_residual<double>(C.S, n, k, unit, ex[i], Xp.data(), AX.data(), t, sc, C.s));
                } else {
                    double rn = 0.0;
                    TRY(C.split_residual(W, W.vs + (size_t)i * d0, W.es[i], Xp.data(), AX.data(), t, &rn));
                }
                bool ok = false;
                TRY(C.correction(W.V.data(), W.dim, t, pass == 0 ? ex[i] : W.es[i], rin[i], &ok));
                if (!ok) continue;
                TRY(C.append(W, t));
                // couplings to the roots from their FP64 sigmas: <x_j|H|v> = <H x_j|v>
                for (int j = 0; j < k; ++j) {
                    TRY(dav_multidot<float, double>(C.S, n, 1, W.V.data() + (W.dim - 1), AX[j], sc, C.s));
                    double cj = 0.0;
                    TRY(fetch(&cj, sc, 1, C.s));
                    W.h[j + (W.dim - 1) * kMaxSub] = W.h[(W.dim - 1) + j * kMaxSub] = cj;
                }
                any = true;
            }
            C.st.iterations++;
            if (!any) break;
            W.eig();
            bool stalled = false;
            for (int i = 0; i < k; ++i) {
                const double prev = rin[i];
                TRY(C.split_residual(W, W.vs + (size_t)i * W.dim, W.es[i], Xp.data(), AX.data(), t, &rin[i]));
                stalled = stalled || (prev >= target[i] && rin[i] > 0.9 * prev);
            }
            if (C.verbose) {
                printf("    inner %02d dim %2d:", pass, W.dim);
                for (int i = 0; i < k; ++i) printf("  %.3e %.12f", rin[i], W.es[i]);
                printf("\n");
            }
            if (stalled) break;
        }
        if (W.dim == k) break;   // no correction direction left
        W.eig();
        // x_i <- sum_{j<k} Y[j,i] x_j (FP64, in place) + sum_{j>=k} Y[j,i] V_j (FP32 corrections)
        TRY(C.rotate(Xp.data(), k, k, W.vs, W.dim));
        for (int i = 0; i < k; ++i) {
            TRY(dav_combine<float, double>(n, W.dim - k, W.vs + (size_t)i * W.dim + k, W.V.data() + k, t, C.s));
            add_kernel<<<kGrid, 256, 0, C.s>>>(n, Xp[i], t);
            BSIM_CUDA(cudaGetLastError());
        }
    }
    C.st.converged = conv ? 1 : 0;
    BSIM_CUDA(cudaStreamSynchronize(C.s));
    return BSIM_OK;
}

template <typename Ti>
int davidson_block(const DevBasis<Ti> *B, const DevNet<Ti> *N, int nroots, double *X, const void *diag, bool diag32,
                   double tol, int maxiter, int ncv, int maxspace, bool mixed, DavBlockStats *stats, int verbose,
                   cudaStream_t s)
{
    const i64 n = B->dim;
    const int k = nroots;
    if (k < 1 || k > kMaxRoots || ncv < k || ncv > kRotMax || maxspace < ncv + k || maxspace > kMaxSub) {
        set_error("need 1 <= nroots <= ncv <= %d and ncv + nroots <= maxspace <= %d", kRotMax, kMaxSub);
        return BSIM_ERR_ARG;
    }
    if (n < maxspace) { set_error("subspace of %d vectors in a %lld-dimensional space", maxspace, (long long)n); return BSIM_ERR_ARG; }
    Ctx<Ti> C{B, N, n, k, diag, diag32, tol, verbose, s};
    TRY(C.S.ensure(s));
    std::vector<double *> Xp(k);
    for (int j = 0; j < k; ++j) Xp[j] = X + (i64)j * n;
    double *sc = C.S.res + kMaxSub;
    for (int j = 0; j < k; ++j) {   // orthonormal start block
        double nrm = 0.0;
        TRY(dav_mgs<double>(C.S, n, j, Xp.data(), Xp[j], sc, s));
        TRY(fetch(&nrm, sc, 1, s));
        if (nrm < 1e-12) { set_error("start vector %d is linearly dependent on the others", j); return BSIM_ERR_ARG; }
        TRY(dav_normalize(C.S, n, Xp[j], sc, s));
    }
    int rc = mixed ? block_mixed(C, Xp, maxiter, ncv, maxspace) : block_fp64(C, Xp, maxiter, ncv, maxspace);
    if (stats) *stats = C.st;
    return rc;
}

template int davidson_block<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, int, double *,
                                      const void *, bool, double, int, int, int, bool, DavBlockStats *, int,
                                      cudaStream_t);
template int davidson_block<unsigned long long>(const DevBasis<unsigned long long> *,
                                                const DevNet<unsigned long long> *, int, double *, const void *, bool,
                                                double, int, int, int, bool, DavBlockStats *, int, cudaStream_t);

}  // namespace bsim
