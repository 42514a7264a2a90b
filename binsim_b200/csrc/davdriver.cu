// Device-resident Davidson drivers.
//
// davidson_fp64 restates jl/davidson.jl:1-185 step for step: Rayleigh-Ritz on
// the host (FP64 Jacobi on <= 64 x 64), Ritz vector and residual, restart to
// ncv vectors when the subspace is full, preconditioner r/(d - e) clamped at
// max(1e-2 |r|, 1e-4), modified Gram-Schmidt repeated when the norm drops
// below 0.717 of its value, normalisation, one sigma per expansion.
// Vectors never leave the device; each iteration reads back a few scalars.
//
// davidson_mixed keeps the subspace V, AV in FP32 and expands it with the
// FP32-bulk sigma (FP64 accumulation inside), while every outer iteration
// recomputes the residual of the current FP64 vector with the FP64 sigma
// (FP64 residual refinement).  Rayleigh-Ritz, Gram-Schmidt projections,
// residual norms and energies are FP64 reductions over the FP32 data.
#include "dav.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace bsim {

namespace {

struct DevBuf {
    void *p = nullptr;
    cudaStream_t s = 0;
    ~DevBuf() { if (p) cudaFreeAsync(p, s); }
};

template <typename T>
int alloc(DevBuf &b, size_t n, cudaStream_t s)
{
    b.s = s;
    cudaError_t e = dmalloc_async(&b.p, std::max<size_t>(1, n) * sizeof(T), s);
    if (e != cudaSuccess) { b.p = nullptr; return cuda_status(e, "davidson buffer"); }
    return BSIM_OK;
}

int fetch(double *host, const double *dev, int n, cudaStream_t s)
{
    BSIM_CUDA(cudaMemcpyAsync(host, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    BSIM_CUDA(cudaStreamSynchronize(s));
    return BSIM_OK;
}

__global__ void cvt_kernel_d2f(const double *__restrict__ x, float *__restrict__ y, i64 n)
{
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) y[i] = (float)x[i];
}

// r = ax - e x (all FP64), partial |r|^2 written to part, final to out
__global__ void resid_kernel(i64 n, const double *__restrict__ x, const double *__restrict__ ax, double e,
                             double *__restrict__ r)
{
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        r[i] = ax[i] - e * x[i];
}

// x = a * x + t
__global__ void axpby_kernel(i64 n, double a, double *__restrict__ x, const double *__restrict__ t)
{
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        x[i] = a * x[i] + t[i];
}

}  // namespace

#define TRY(...) do { int st__ = (__VA_ARGS__); if (st__ != BSIM_OK) return st__; } while (0)

template <typename Ti>
int davidson_fp64(const DevBasis<Ti> *B, const DevNet<Ti> *N, double *v0, const double *diags, double tol,
                  int maxiter, int ncv, int maxspace, double *x_out, DavStats *stats, int verbose, cudaStream_t s)
{
    const i64 n = B->dim;
    if (maxspace > kMaxSub || maxspace <= ncv || ncv < 1) {
        set_error("need 1 <= ncv < maxspace <= %d", kMaxSub);
        return BSIM_ERR_ARG;
    }
    DavScratch S;
    TRY(S.ensure());
    std::vector<DevBuf> vb(maxspace), avb(maxspace), tb(ncv), tab(ncv);
    DevBuf axb;
    std::vector<double *> V(maxspace), AV(maxspace), Vt(ncv), AVt(ncv);
    for (int j = 0; j < maxspace; ++j) {
        TRY(alloc<double>(vb[j], n, s)); TRY(alloc<double>(avb[j], n, s));
        V[j] = (double *)vb[j].p; AV[j] = (double *)avb[j].p;
    }
    for (int j = 0; j < ncv; ++j) {
        TRY(alloc<double>(tb[j], n, s)); TRY(alloc<double>(tab[j], n, s));
        Vt[j] = (double *)tb[j].p; AVt[j] = (double *)tab[j].p;
    }
    TRY(alloc<double>(axb, n, s));
    double *axt = (double *)axb.p;
    double *sc = S.res + kMaxSub;   // scalar slots
    DavStats st{};

    BSIM_CUDA(cudaMemcpyAsync(V[0], v0, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    TRY(dav_normalize(S, n, V[0], sc, s));
    TRY(sigma(B, N, V[0], nullptr, AV[0], false, s));
    st.sigma_fp64++;
    TRY(dav_dot(S, n, V[0], AV[0], sc, s));
    double h[kMaxSub * kMaxSub] = {0};
    TRY(fetch(&h[0], sc, 1, s));
    int dim = 1;
    double es[kMaxSub], vs[kMaxSub * kMaxSub], col[kMaxSub];
    double e_best = h[0];
    for (int iter = 1; iter <= maxiter; ++iter) {
        jacobi_eigh(dim, h, kMaxSub, es, vs);
        const double min_e = es[0];
        TRY(dav_ritz_residual<double>(S, n, dim, vs, min_e, V.data(), AV.data(), axt, sc, s));
        double norm_r;
        TRY(fetch(&norm_r, sc, 1, s));
        if (verbose) printf("  Step %03d:  residual: %.4e,  e: %.14f\n", iter, norm_r, min_e);
        e_best = min_e;
        st.iterations = iter;
        st.residual = norm_r;
        if (norm_r < tol) {
            TRY(dav_combine<double, double>(n, dim, vs, V.data(), x_out, s));
            st.energy = e_best;
            st.converged = 1;
            if (stats) *stats = st;
            return BSIM_OK;
        }
        if (dim >= maxspace) {
            const int nsave = std::min(ncv, dim);
            for (int i = 0; i < nsave; ++i) {
                TRY(dav_combine<double, double>(n, dim, vs + (size_t)i * dim, V.data(), Vt[i], s));
                TRY(dav_combine<double, double>(n, dim, vs + (size_t)i * dim, AV.data(), AVt[i], s));
            }
            for (int i = 0; i < nsave; ++i) { std::swap(V[i], Vt[i]); std::swap(AV[i], AVt[i]); }
            dim = nsave;
            for (int j = 0; j < dim; ++j) {   // rebuild_heff, davidson.hpp:221-272
                TRY(dav_multidot<double, double>(S, n, dim, V.data(), AV[j], S.res, s));
                TRY(fetch(col, S.res, dim, s));
                for (int i = 0; i < dim; ++i) h[i + j * kMaxSub] = col[i];
            }
            for (int j = 0; j < dim; ++j)
                for (int i = 0; i < j; ++i) h[i + j * kMaxSub] = h[j + i * kMaxSub] = 0.5 * (h[i + j * kMaxSub] + h[j + i * kMaxSub]);
        }
        const double shift = std::max(norm_r * 1e-2, 1e-4);
        TRY(dav_precondition(S, n, axt, diags, min_e, shift, sc, s));
        double nrm[2];
        TRY(fetch(&nrm[0], sc, 1, s));
        TRY(dav_mgs<double>(S, n, dim, V.data(), axt, sc + 1, s));
        TRY(fetch(&nrm[1], sc + 1, 1, s));
        if (nrm[1] < 0.717 * nrm[0]) {
            TRY(dav_mgs<double>(S, n, dim, V.data(), axt, sc + 1, s));
            TRY(fetch(&nrm[1], sc + 1, 1, s));
        }
        if (nrm[1] < 1e-12) {   // breakdown: the new direction lies in the subspace
            TRY(dav_combine<double, double>(n, dim, vs, V.data(), x_out, s));
            st.energy = e_best;
            if (stats) *stats = st;
            return BSIM_OK;
        }
        TRY(dav_normalize(S, n, axt, sc, s));
        BSIM_CUDA(cudaMemcpyAsync(V[dim], axt, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        TRY(sigma(B, N, V[dim], nullptr, AV[dim], false, s));
        st.sigma_fp64++;
        ++dim;
        TRY(dav_multidot<double, double>(S, n, dim, V.data(), AV[dim - 1], S.res, s));
        TRY(fetch(col, S.res, dim, s));
        for (int i = 0; i < dim; ++i) h[i + (dim - 1) * kMaxSub] = h[(dim - 1) + i * kMaxSub] = col[i];
    }
    jacobi_eigh(dim, h, kMaxSub, es, vs);
    TRY(dav_combine<double, double>(n, dim, vs, V.data(), x_out, s));
    st.energy = e_best;
    if (stats) *stats = st;
    return BSIM_OK;
}

template <typename Ti>
int davidson_mixed(const DevBasis<Ti> *B, const DevNet<Ti> *N, double *v0, const double *diags, double tol,
                   int maxiter, int maxspace, double *x_out, DavStats *stats, int verbose, cudaStream_t s)
{
    const i64 n = B->dim;
    if (maxspace > kMaxSub || maxspace < 3) { set_error("need 3 <= maxspace <= %d", kMaxSub); return BSIM_ERR_ARG; }
    DavScratch S;
    TRY(S.ensure());
    std::vector<DevBuf> vb(maxspace), avb(maxspace);
    std::vector<float *> V(maxspace), AV(maxspace);
    for (int j = 0; j < maxspace; ++j) {
        TRY(alloc<float>(vb[j], n, s)); TRY(alloc<float>(avb[j], n, s));
        V[j] = (float *)vb[j].p; AV[j] = (float *)avb[j].p;
    }
    DevBuf xb, axb, rb, tb, ayb;
    TRY(alloc<double>(xb, n, s)); TRY(alloc<double>(axb, n, s)); TRY(alloc<double>(rb, n, s));
    TRY(alloc<double>(tb, n, s)); TRY(alloc<double>(ayb, n, s));
    // x: current FP64 vector, ax = H x (FP64), r = ax - E x, t: expansion vector,
    // ay: FP32-bulk sigma of the newest subspace vector
    double *x = (double *)xb.p, *ax = (double *)axb.p, *r = (double *)rb.p, *t = (double *)tb.p;
    double *ay = (double *)ayb.p;
    double *sc = S.res + kMaxSub;
    DavStats st{};
    const int grid = 1184;
    BSIM_CUDA(cudaMemcpyAsync(x, v0, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    TRY(dav_normalize(S, n, x, sc, s));
    double h[kMaxSub * kMaxSub], es[kMaxSub], vs[kMaxSub * kMaxSub], col[kMaxSub];
    int total_inner = 0;

    // ---- phase A: the reference driver's Davidson (restart to ncv Ritz vectors)
    // on FP32 subspace storage with the FP32-bulk sigma; it stops at the
    // tolerance or where the FP32 residual stalls, and the FP64 refinement below
    // takes over from its Ritz vector.
    {
        const int ncv = std::min(3, maxspace - 1);
        std::vector<DevBuf> tvb(ncv), tavb(ncv);
        std::vector<float *> Vt(ncv), AVt(ncv);
        for (int j = 0; j < ncv; ++j) {
            TRY(alloc<float>(tvb[j], n, s)); TRY(alloc<float>(tavb[j], n, s));
            Vt[j] = (float *)tvb[j].p; AVt[j] = (float *)tavb[j].p;
        }
        cvt_kernel_d2f<<<grid, 256, 0, s>>>(x, V[0], n);
        TRY(sigma(B, N, nullptr, V[0], ay, true, s));
        st.sigma_fp32++;
        cvt_kernel_d2f<<<grid, 256, 0, s>>>(ay, AV[0], n);
        TRY(dav_multidot<float, float>(S, n, 1, V.data(), AV[0], S.res, s));
        TRY(fetch(&h[0], S.res, 1, s));
        int dim = 1;
        double best = 1e300;   // smallest residual so far and the iterations since it
        int since_best = 0;
        for (int iter = 1; iter <= maxiter; ++iter) {
            jacobi_eigh(dim, h, kMaxSub, es, vs);
            const double e = es[0];
            double norm_r;
            TRY(dav_ritz_residual<float>(S, n, dim, vs, e, V.data(), AV.data(), t, sc, s));
            TRY(fetch(&norm_r, sc, 1, s));
            if (verbose) printf("  fp32 step %03d: residual %.4e e %.14f\n", iter, norm_r, e);
            // leave at the tolerance, or when the FP32 residual has stopped improving
            // (its noise floor) for a whole subspace cycle
            if (norm_r < best) { best = norm_r; since_best = 0; }
            else ++since_best;
            if (norm_r < tol || since_best >= maxspace || total_inner >= maxiter) break;
            if (dim >= maxspace) {
                const int nsave = std::min(ncv, dim);
                for (int i = 0; i < nsave; ++i) {
                    TRY(dav_combine<float, float>(n, dim, vs + (size_t)i * dim, V.data(), Vt[i], s));
                    TRY(dav_combine<float, float>(n, dim, vs + (size_t)i * dim, AV.data(), AVt[i], s));
                }
                for (int i = 0; i < nsave; ++i) { std::swap(V[i], Vt[i]); std::swap(AV[i], AVt[i]); }
                dim = nsave;
                for (int j = 0; j < dim; ++j) {
                    TRY(dav_multidot<float, float>(S, n, dim, V.data(), AV[j], S.res, s));
                    TRY(fetch(col, S.res, dim, s));
                    for (int i = 0; i < dim; ++i) h[i + j * kMaxSub] = col[i];
                }
                for (int j = 0; j < dim; ++j)
                    for (int i = 0; i < j; ++i)
                        h[i + j * kMaxSub] = h[j + i * kMaxSub] = 0.5 * (h[i + j * kMaxSub] + h[j + i * kMaxSub]);
            }
            const double shift = std::max(norm_r * 1e-2, 1e-4);
            double nrm[2];
            TRY(dav_precondition(S, n, t, diags, e, shift, sc, s));
            TRY(fetch(&nrm[0], sc, 1, s));
            TRY(dav_mgs<float>(S, n, dim, V.data(), t, sc + 1, s));
            TRY(fetch(&nrm[1], sc + 1, 1, s));
            if (nrm[1] < 0.717 * nrm[0]) {
                TRY(dav_mgs<float>(S, n, dim, V.data(), t, sc + 1, s));
                TRY(fetch(&nrm[1], sc + 1, 1, s));
            }
            if (nrm[1] < 1e-12) break;
            TRY(dav_normalize(S, n, t, sc, s));
            cvt_kernel_d2f<<<grid, 256, 0, s>>>(t, V[dim], n);
            TRY(sigma(B, N, nullptr, V[dim], ay, true, s));
            st.sigma_fp32++;
            ++total_inner;
            cvt_kernel_d2f<<<grid, 256, 0, s>>>(ay, AV[dim], n);
            ++dim;
            TRY(dav_multidot<float, float>(S, n, dim, V.data(), AV[dim - 1], S.res, s));
            TRY(fetch(col, S.res, dim, s));
            for (int i = 0; i < dim; ++i) h[i + (dim - 1) * kMaxSub] = h[(dim - 1) + i * kMaxSub] = col[i];
        }
        jacobi_eigh(dim, h, kMaxSub, es, vs);
        TRY(dav_combine<float, double>(n, dim, vs, V.data(), x, s));
        TRY(dav_normalize(S, n, x, sc, s));
        // restarts swapped subspace slots with the temporaries freed at the end of
        // this scope (stream-ordered, after the combine): point V/AV back at the
        // buffers that live through phase B
        for (int j = 0; j < maxspace; ++j) { V[j] = (float *)vb[j].p; AV[j] = (float *)avb[j].p; }
    }

    // ---- phase B: FP64 residual refinement ----
    for (int outer = 0; outer < maxiter; ++outer) {
        // ---- FP64 residual of the current vector ----
        TRY(sigma(B, N, x, nullptr, ax, false, s));
        st.sigma_fp64++;
        TRY(dav_dot(S, n, x, ax, sc, s));
        double E;
        TRY(fetch(&E, sc, 1, s));
        resid_kernel<<<grid, 256, 0, s>>>(n, x, ax, E, r);
        TRY(dav_dot(S, n, r, r, sc, s));
        double rr;
        TRY(fetch(&rr, sc, 1, s));
        const double rnorm = sqrt(std::max(rr, 0.0));
        st.energy = E;
        st.residual = rnorm;
        if (verbose) printf("  Outer %02d:  fp64 residual: %.4e,  e: %.14f\n", outer, rnorm, E);
        if (rnorm < tol) { st.converged = 1; break; }
        if (total_inner >= maxiter) break;
        // ---- inner FP32-storage Davidson on span{x, t1, t2, ...} ----
        cvt_kernel_d2f<<<grid, 256, 0, s>>>(x, V[0], n);
        cvt_kernel_d2f<<<grid, 256, 0, s>>>(ax, AV[0], n);
        int dim = 1;
        h[0] = E;
        BSIM_CUDA(cudaMemcpyAsync(t, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        double rin = rnorm, e_in = E;
        for (int it = 0; it < maxspace - 1; ++it) {
            const double shift = std::max(rin * 1e-2, 1e-4);
            double nrm[2];
            TRY(dav_precondition(S, n, t, diags, e_in, shift, sc, s));
            TRY(fetch(&nrm[0], sc, 1, s));
            TRY(dav_mgs<float>(S, n, dim, V.data(), t, sc + 1, s));
            TRY(fetch(&nrm[1], sc + 1, 1, s));
            if (nrm[1] < 0.717 * nrm[0]) {
                TRY(dav_mgs<float>(S, n, dim, V.data(), t, sc + 1, s));
                TRY(fetch(&nrm[1], sc + 1, 1, s));
            }
            if (nrm[1] < 1e-12) break;
            TRY(dav_normalize(S, n, t, sc, s));
            cvt_kernel_d2f<<<grid, 256, 0, s>>>(t, V[dim], n);
            // FP32-bulk sigma straight from the FP32 basis vector
            TRY(sigma(B, N, nullptr, V[dim], ay, true, s));
            st.sigma_fp32++;
            ++total_inner;
            cvt_kernel_d2f<<<grid, 256, 0, s>>>(ay, AV[dim], n);
            ++dim;
            TRY(dav_multidot<float, float>(S, n, dim, V.data(), AV[dim - 1], S.res, s));
            // the coupling to the current vector, <x|H|V_j> = <H x|V_j>, from the
            // FP64 sigma of x: near convergence it drives the correction, so it
            // must not carry the FP32-bulk sigma's rounding
            TRY(dav_multidot<float, double>(S, n, 1, V.data() + (dim - 1), ax, S.res + dim, s));
            TRY(fetch(col, S.res, dim + 1, s));
            col[0] = col[dim];
            for (int i = 0; i < dim; ++i) h[i + (dim - 1) * kMaxSub] = h[(dim - 1) + i * kMaxSub] = col[i];
            jacobi_eigh(dim, h, kMaxSub, es, vs);
            e_in = es[0];
            const double rprev = rin;
            TRY(dav_ritz_residual<float>(S, n, dim, vs, e_in, V.data(), AV.data(), t, sc, s));
            TRY(fetch(&rin, sc, 1, s));
            if (verbose) printf("    inner %02d: residual %.4e e %.14f\n", it, rin, e_in);
            // leave for an FP64 refinement once the inner residual dropped enough or
            // stalls at the FP32 noise floor
            if (rin < 0.05 * rnorm || rin < 0.5 * tol || (it >= 2 && rin > rprev) || total_inner >= maxiter)
                break;
        }
        jacobi_eigh(dim, h, kMaxSub, es, vs);
        // x <- y0 * x + sum_{j>=1} y_j V_j: the FP64 vector keeps its precision and
        // only the correction, small near convergence, carries FP32 rounding.
        if (dim > 1) {
            TRY(dav_combine<float, double>(n, dim - 1, vs + 1, V.data() + 1, t, s));
            axpby_kernel<<<grid, 256, 0, s>>>(n, vs[0], x, t);
        }
        TRY(dav_normalize(S, n, x, sc, s));
    }
    st.iterations = total_inner;
    BSIM_CUDA(cudaMemcpyAsync(x_out, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    if (stats) *stats = st;
    BSIM_CUDA(cudaStreamSynchronize(s));
    return BSIM_OK;
}

template int davidson_fp64<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, double *, const double *,
                                     double, int, int, int, double *, DavStats *, int, cudaStream_t);
template int davidson_mixed<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, double *, const double *,
                                      double, int, int, double *, DavStats *, int, cudaStream_t);
template int davidson_fp64<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, double *, const double *,
                                     double, int, int, int, double *, DavStats *, int, cudaStream_t);
template int davidson_mixed<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, double *, const double *,
                                      double, int, int, double *, DavStats *, int, cudaStream_t);

}  // namespace bsim
