// Device-resident Davidson drivers.
//
// davidson_fp64 restates jl/davidson.jl:1-185 step for step: Rayleigh-Ritz
// (Jacobi on the <= 64 x 64 projected matrix), Ritz vector and residual,
// restart to ncv vectors when the subspace is full, preconditioner r/(d - e)
// clamped at max(1e-2 |r|, 1e-4), Gram-Schmidt repeated when the norm drops
// below 0.717 of its value, normalisation, one sigma per expansion.  Every
// step runs on the device, the Jacobi eigensolve included (one warp), and the
// decisions that depend on scalars (the preconditioner's shift, the second
// Gram-Schmidt pass, breakdown) are taken there too: the host reads one
// residual norm per iteration for the convergence test, instead of a handful of
// scalars each followed by a synchronisation.  The orthogonalisation is
// classical Gram-Schmidt against the whole subspace at once (a few launches)
// where the reference uses modified Gram-Schmidt (one reduction per vector);
// with the 0.717 repetition both give an orthogonal direction to rounding.
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

}  // namespace

#define TRY(...) do { int st__ = (__VA_ARGS__); if (st__ != BSIM_OK) return st__; } while (0)

namespace {
// Device state of a driver: the projected matrix, its eigenpairs and the scalars
// the iteration reads on the device.  sc[0] residual norm, sc[1] breakdown flag
// of the last expansion, then the Ritz values (evals = sc + 2), so that the one
// read of an iteration is one copy; aux[0] / aux[1] norm before / after
// Gram-Schmidt, aux[2] the start vector's norm.
struct DavState {
    DevBuf buf;
    double *h = nullptr, *evals = nullptr, *evecs = nullptr, *proj = nullptr, *sc = nullptr, *aux = nullptr;
    int init(cudaStream_t s)
    {
        constexpr size_t kSq = (size_t)kMaxSub * kMaxSub, kAll = 2 * kSq + 2 * kMaxSub + 8;
        TRY(alloc<double>(buf, kAll, s));
        h = (double *)buf.p;
        evecs = h + kSq;
        sc = evecs + kSq;
        evals = sc + 2;
        aux = evals + kMaxSub;
        proj = aux + 4;
        BSIM_CUDA(cudaMemsetAsync(buf.p, 0, sizeof(double) * kAll, s));
        return BSIM_OK;
    }
    // the one read of an iteration: residual norm, breakdown flag, lowest Ritz value
    int read(double *rnorm, bool *breakdown, double *e0, cudaStream_t s) const
    {
        double v[3];
        BSIM_CUDA(cudaMemcpyAsync(v, sc, sizeof(double) * 3, cudaMemcpyDeviceToHost, s));
        BSIM_CUDA(cudaStreamSynchronize(s));
        *rnorm = v[0];
        *breakdown = v[1] != 0.0;
        *e0 = v[2];
        return BSIM_OK;
    }
    int set_scalar(int i, double v, cudaStream_t s)
    {
        BSIM_CUDA(cudaMemcpyAsync(sc + i, &v, sizeof(double), cudaMemcpyHostToDevice, s));
        BSIM_CUDA(cudaStreamSynchronize(s));   // v lives on the host stack
        return BSIM_OK;
    }
};
}  // namespace

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
    TRY(S.ensure(s));
    DavState D;
    TRY(D.init(s));
    std::vector<DevBuf> vb(maxspace), avb(maxspace), tb(ncv), tab(ncv), xb(2);
    DevBuf axb;
    std::vector<double *> V(maxspace), AV(maxspace), Vt(ncv), AVt(ncv), xk(2);
    for (int j = 0; j < maxspace; ++j) {
        TRY(alloc<double>(vb[j], n, s)); TRY(alloc<double>(avb[j], n, s));
        V[j] = (double *)vb[j].p; AV[j] = (double *)avb[j].p;
    }
    for (int j = 0; j < ncv; ++j) {
        TRY(alloc<double>(tb[j], n, s)); TRY(alloc<double>(tab[j], n, s));
        Vt[j] = (double *)tb[j].p; AVt[j] = (double *)tab[j].p;
    }
    for (int j = 0; j < 2; ++j) { TRY(alloc<double>(xb[j], n, s)); xk[j] = (double *)xb[j].p; }
    TRY(alloc<double>(axb, n, s));
    double *axt = (double *)axb.p;
    DavStats st{};

    BSIM_CUDA(cudaMemcpyAsync(V[0], v0, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    TRY(dav_normalize(S, n, V[0], D.aux + 2, s));
    TRY(sigma(B, N, V[0], nullptr, AV[0], false, s));
    st.sigma_fp64++;
    TRY(dav_multidot<double, double>(S, n, 1, V.data(), AV[0], D.h, s));
    int dim = 1;
    double e_prev = 0.0;
    for (int iter = 1; iter <= maxiter; ++iter) {
        TRY(dav_eigh_dev(dim, D.h, kMaxSub, D.evals, D.evecs, s));
        TRY(dav_ritz_residual_dev<double>(S, n, dim, D.evecs, D.evals, V.data(), AV.data(), axt, xk[iter & 1],
                                          D.sc, s));
        double norm_r, e;
        bool breakdown;
        TRY(D.read(&norm_r, &breakdown, &e, s));
        if (breakdown) {   // the last expansion lay in the subspace: the previous Ritz vector is the answer
            BSIM_CUDA(cudaMemcpyAsync(x_out, xk[(iter - 1) & 1], sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
            st.energy = e_prev;
            if (stats) *stats = st;
            BSIM_CUDA(cudaStreamSynchronize(s));
            return BSIM_OK;
        }
        if (verbose) printf("  Step %03d:  residual: %.4e,  e: %.14f\n", iter, norm_r, e);
        e_prev = e;
        st.iterations = iter;
        st.residual = norm_r;
        st.energy = e;
        if (norm_r < tol) {
            BSIM_CUDA(cudaMemcpyAsync(x_out, xk[iter & 1], sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
            st.converged = 1;
            if (stats) *stats = st;
            BSIM_CUDA(cudaStreamSynchronize(s));
            return BSIM_OK;
        }
        if (dim >= maxspace) {   // restart to the ncv lowest Ritz vectors, rebuild_heff (davidson.hpp:221-272)
            const int nsave = std::min(ncv, dim);
            for (int i = 0; i < nsave; ++i) {
                TRY(dav_combine_dev<double, double>(n, dim, D.evecs + (size_t)i * dim, V.data(), Vt[i], s));
                TRY(dav_combine_dev<double, double>(n, dim, D.evecs + (size_t)i * dim, AV.data(), AVt[i], s));
            }
            for (int i = 0; i < nsave; ++i) { std::swap(V[i], Vt[i]); std::swap(AV[i], AVt[i]); }
            dim = nsave;
            for (int j = 0; j < dim; ++j)
                TRY(dav_multidot<double, double>(S, n, dim, V.data(), AV[j], D.h + (size_t)j * kMaxSub, s));
            TRY(dav_sym_avg(dim, D.h, kMaxSub, s));
        }
        TRY(dav_precondition_dev<double>(S, n, axt, diags, D.evals, D.sc, D.aux, s));
        TRY(dav_cgs2_dev<double>(S, n, dim, V.data(), axt, D.aux, D.proj, s));
        TRY(dav_normalize_into<double>(n, axt, D.aux + 1, V[dim], D.sc + 1, s));
        TRY(sigma(B, N, V[dim], nullptr, AV[dim], false, s));
        st.sigma_fp64++;
        ++dim;
        TRY(dav_multidot<double, double>(S, n, dim, V.data(), AV[dim - 1], D.h + (size_t)(dim - 1) * kMaxSub, s));
        TRY(dav_mirror_col(dim, D.h, kMaxSub, s));
    }
    TRY(dav_eigh_dev(dim, D.h, kMaxSub, D.evals, D.evecs, s));
    TRY(dav_combine_dev<double, double>(n, dim, D.evecs, V.data(), x_out, s));
    double e;
    BSIM_CUDA(cudaMemcpyAsync(&e, D.evals, sizeof(double), cudaMemcpyDeviceToHost, s));
    BSIM_CUDA(cudaStreamSynchronize(s));
    st.energy = e;
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
    TRY(S.ensure(s));
    DavState D;
    TRY(D.init(s));
    std::vector<DevBuf> vb(maxspace), avb(maxspace);
    std::vector<float *> V(maxspace), AV(maxspace);
    for (int j = 0; j < maxspace; ++j) {
        TRY(alloc<float>(vb[j], n, s)); TRY(alloc<float>(avb[j], n, s));
        V[j] = (float *)vb[j].p; AV[j] = (float *)avb[j].p;
    }
    DevBuf xb, axb, rb, tb, ayb, xkb[2];
    TRY(alloc<double>(xb, n, s)); TRY(alloc<double>(axb, n, s)); TRY(alloc<double>(rb, n, s));
    TRY(alloc<double>(tb, n, s)); TRY(alloc<double>(ayb, n, s));
    TRY(alloc<double>(xkb[0], n, s)); TRY(alloc<double>(xkb[1], n, s));
    // x: current FP64 vector, ax = H x (FP64), r = ax - E x, t: expansion vector,
    // ay: FP32-bulk sigma of the newest subspace vector, xk: Ritz vectors of the
    // last two phase-A iterations
    double *x = (double *)xb.p, *ax = (double *)axb.p, *r = (double *)rb.p, *t = (double *)tb.p;
    double *ay = (double *)ayb.p, *xk[2] = {(double *)xkb[0].p, (double *)xkb[1].p};
    double *sc = S.res + kMaxSub;
    DavStats st{};
    const int grid = 1184;
    BSIM_CUDA(cudaMemcpyAsync(x, v0, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    TRY(dav_normalize(S, n, x, sc, s));
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
        TRY(dav_multidot<float, float>(S, n, 1, V.data(), AV[0], D.h, s));
        int dim = 1, last = 0;
        double best = 1e300;   // smallest residual so far and the iterations since it
        int since_best = 0;
        for (int iter = 1; iter <= maxiter; ++iter) {
            TRY(dav_eigh_dev(dim, D.h, kMaxSub, D.evals, D.evecs, s));
            TRY(dav_ritz_residual_dev<float>(S, n, dim, D.evecs, D.evals, V.data(), AV.data(), t, xk[iter & 1],
                                             D.sc, s));
            double norm_r, e;
            bool breakdown;
            TRY(D.read(&norm_r, &breakdown, &e, s));
            if (breakdown) { last = (iter - 1) & 1; break; }   // the previous Ritz vector
            last = iter & 1;
            if (verbose) printf("  fp32 step %03d: residual %.4e e %.14f\n", iter, norm_r, e);
            // leave at the tolerance, or when the FP32 residual has stopped improving
            // (its noise floor) for a whole subspace cycle
            if (norm_r < best) { best = norm_r; since_best = 0; }
            else ++since_best;
            if (norm_r < tol || since_best >= maxspace || total_inner >= maxiter) break;
            if (dim >= maxspace) {
                const int nsave = std::min(ncv, dim);
                for (int i = 0; i < nsave; ++i) {
                    TRY(dav_combine_dev<float, float>(n, dim, D.evecs + (size_t)i * dim, V.data(), Vt[i], s));
                    TRY(dav_combine_dev<float, float>(n, dim, D.evecs + (size_t)i * dim, AV.data(), AVt[i], s));
                }
                for (int i = 0; i < nsave; ++i) { std::swap(V[i], Vt[i]); std::swap(AV[i], AVt[i]); }
                dim = nsave;
                for (int j = 0; j < dim; ++j)
                    TRY(dav_multidot<float, float>(S, n, dim, V.data(), AV[j], D.h + (size_t)j * kMaxSub, s));
                TRY(dav_sym_avg(dim, D.h, kMaxSub, s));
            }
            TRY(dav_precondition_dev<double>(S, n, t, diags, D.evals, D.sc, D.aux, s));
            TRY(dav_cgs2_dev<float>(S, n, dim, V.data(), t, D.aux, D.proj, s));
            TRY(dav_normalize_into<float>(n, t, D.aux + 1, V[dim], D.sc + 1, s));
            TRY(sigma(B, N, nullptr, V[dim], ay, true, s));
            st.sigma_fp32++;
            ++total_inner;
            cvt_kernel_d2f<<<grid, 256, 0, s>>>(ay, AV[dim], n);
            ++dim;
            TRY(dav_multidot<float, float>(S, n, dim, V.data(), AV[dim - 1], D.h + (size_t)(dim - 1) * kMaxSub, s));
            TRY(dav_mirror_col(dim, D.h, kMaxSub, s));
        }
        BSIM_CUDA(cudaMemcpyAsync(x, xk[last], sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        TRY(dav_normalize(S, n, x, sc, s));
        // restarts swapped subspace slots with the temporaries freed at the end of
        // this scope (stream-ordered, after the copy above): point V/AV back at the
        // buffers that live through phase B
        for (int j = 0; j < maxspace; ++j) { V[j] = (float *)vb[j].p; AV[j] = (float *)avb[j].p; }
        TRY(D.set_scalar(1, 0.0, s));   // a phase-A breakdown flag does not carry into phase B
    }

    // ---- phase B: FP64 residual refinement ----
    for (int outer = 0; outer < maxiter; ++outer) {
        // ---- FP64 residual of the current vector ----
        TRY(sigma(B, N, x, nullptr, ax, false, s));
        st.sigma_fp64++;
        TRY(dav_dot(S, n, x, ax, sc, s));
        double E;
        BSIM_CUDA(cudaMemcpyAsync(&E, sc, sizeof(double), cudaMemcpyDeviceToHost, s));
        BSIM_CUDA(cudaStreamSynchronize(s));
        resid_kernel<<<grid, 256, 0, s>>>(n, x, ax, E, r);
        TRY(dav_dot(S, n, r, r, sc, s));
        double rr;
        BSIM_CUDA(cudaMemcpyAsync(&rr, sc, sizeof(double), cudaMemcpyDeviceToHost, s));
        BSIM_CUDA(cudaStreamSynchronize(s));
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
        {   // h[0][0] = E, the first Ritz value E and the residual norm on the device
            const double init[2] = {E, rnorm};
            BSIM_CUDA(cudaMemcpyAsync(D.h, &init[0], sizeof(double), cudaMemcpyHostToDevice, s));
            BSIM_CUDA(cudaMemcpyAsync(D.evals, &init[0], sizeof(double), cudaMemcpyHostToDevice, s));
            BSIM_CUDA(cudaMemcpyAsync(D.sc, &init[1], sizeof(double), cudaMemcpyHostToDevice, s));
            BSIM_CUDA(cudaStreamSynchronize(s));
        }
        BSIM_CUDA(cudaMemcpyAsync(t, r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        double rin = rnorm;
        bool have_eigh = false;   // evecs hold the eigenpairs of the current dim
        for (int it = 0; it < maxspace - 1; ++it) {
            TRY(dav_precondition_dev<double>(S, n, t, diags, D.evals, D.sc, D.aux, s));
            TRY(dav_cgs2_dev<float>(S, n, dim, V.data(), t, D.aux, D.proj, s));
            TRY(dav_normalize_into<float>(n, t, D.aux + 1, V[dim], D.sc + 1, s));
            // FP32-bulk sigma straight from the FP32 basis vector
            TRY(sigma(B, N, nullptr, V[dim], ay, true, s));
            st.sigma_fp32++;
            ++total_inner;
            cvt_kernel_d2f<<<grid, 256, 0, s>>>(ay, AV[dim], n);
            ++dim;
            double *hc = D.h + (size_t)(dim - 1) * kMaxSub;
            TRY(dav_multidot<float, float>(S, n, dim, V.data(), AV[dim - 1], hc, s));
            // the coupling to the current vector, <x|H|V_j> = <H x|V_j>, from the
            // FP64 sigma of x: near convergence it drives the correction, so it
            // must not carry the FP32-bulk sigma's rounding
            TRY(dav_multidot<float, double>(S, n, 1, V.data() + (dim - 1), ax, hc, s));
            TRY(dav_mirror_col(dim, D.h, kMaxSub, s));
            TRY(dav_eigh_dev(dim, D.h, kMaxSub, D.evals, D.evecs, s));
            const double rprev = rin;
            TRY(dav_ritz_residual_dev<float>(S, n, dim, D.evecs, D.evals, V.data(), AV.data(), t, nullptr, D.sc,
                                             s));
            double e_in;
            bool breakdown;
            TRY(D.read(&rin, &breakdown, &e_in, s));
            have_eigh = true;
            if (breakdown) {   // the last direction lay in the space: drop it
                --dim;
                TRY(D.set_scalar(1, 0.0, s));
                TRY(dav_eigh_dev(dim, D.h, kMaxSub, D.evals, D.evecs, s));
                break;
            }
            if (verbose) printf("    inner %02d: residual %.4e e %.14f\n", it, rin, e_in);
            // leave for an FP64 refinement once the inner residual dropped enough or
            // stalls at the FP32 noise floor
            if (rin < 0.05 * rnorm || rin < 0.5 * tol || (it >= 2 && rin > rprev) || total_inner >= maxiter)
                break;
        }
        // x <- y0 * x + sum_{j>=1} y_j V_j: the FP64 vector keeps its precision and
        // only the correction, small near convergence, carries FP32 rounding.
        if (have_eigh && dim > 1) {
            TRY(dav_combine_dev<float, double>(n, dim - 1, D.evecs + 1, V.data() + 1, t, s));
            TRY(dav_axpby_dev(n, D.evecs, x, t, s));
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
