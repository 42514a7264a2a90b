// VQE energy and adjoint (reverse-mode) gradient on device.
//
// Restates energy_objective (reference jl/vqe.jl:1-21): forward expm of every
// generator, one sigma, then the reverse sweep of fused backgrad steps that
// uncompute l and propagate r, grad = 2 * backgrad / |l|^2.  Differences from
// the reference's GPU workflow (jl/cuda/cunetwork.jl + cuda/backgrad.cuh):
//   * the whole sweep is one library call: no host round trip per generator
//     (the reference does cudaMalloc + D2H copy + cudaFree per backgrad);
//     every gradient term lands in a device array, read back once;
//   * checkpoints: the forward state is copied every `ckpt_every` parameters,
//     and the reverse sweep restores l from the copy when it reaches that
//     position, which stops uncompute drift (the Givens rotations are unitary
//     only to the precision of the SVD weights);
//   * spin-adapted generators are ordered products of spin-orbital components
//     sharing one parameter: param_idx maps each applied component to its
//     parameter and the gradient sums the component terms.
#include "vqe.h"
#include "dav.h"
#include "ops.h"

#include <algorithm>
#include <cmath>
#include <vector>

namespace bsim {

namespace {
struct Buf {
    void *p = nullptr;
    cudaStream_t s = 0;
    ~Buf() { if (p) cudaFreeAsync(p, s); }
    int get(size_t bytes, cudaStream_t st) {
        s = st;
        cudaError_t e = dmalloc_async(&p, std::max<size_t>(bytes, 8), st);
        if (e != cudaSuccess) { p = nullptr; return cuda_status(e, "vqe buffer"); }
        return BSIM_OK;
    }
};

__global__ void scatter_ref_kernel(double *__restrict__ v, const long long *__restrict__ idx,
                                   const double *__restrict__ val, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[idx[i]] = val[i];
}
}  // namespace

#define TRY(...) do { int st__ = (__VA_ARGS__); if (st__ != BSIM_OK) return st__; } while (0)

template <typename Ti>
int prepare_state(const DevBasis<Ti> *B, const DevNet<Ti> *P, i64 n_ops, const i64 *op_idx, const i64 *param_idx,
                  const double *thetas, const i64 *ref_idx, const double *ref_val, i64 n_ref, double *v,
                  cudaStream_t s)
{
    for (i64 i = 0; i < n_ref; ++i)
        if (ref_idx[i] < 0 || ref_idx[i] >= B->dim) { set_error("reference index out of range"); return BSIM_ERR_ARG; }
    BSIM_CUDA(cudaMemsetAsync(v, 0, sizeof(double) * B->dim, s));
    if (n_ref > 0) {
        Buf bi, bv;
        TRY(bi.get(sizeof(i64) * n_ref, s));
        TRY(bv.get(sizeof(double) * n_ref, s));
        BSIM_CUDA(cudaMemcpyAsync(bi.p, ref_idx, sizeof(i64) * n_ref, cudaMemcpyHostToDevice, s));
        BSIM_CUDA(cudaMemcpyAsync(bv.p, ref_val, sizeof(double) * n_ref, cudaMemcpyHostToDevice, s));
        scatter_ref_kernel<<<(unsigned)std::min<i64>(1024, (n_ref + 255) / 256), 256, 0, s>>>(
            v, (const long long *)bi.p, (const double *)bv.p, (int)n_ref);
        BSIM_CUDA(cudaGetLastError());
        BSIM_CUDA(cudaStreamSynchronize(s));   // host arrays of the copies must outlive them
    }
    for (i64 i = 0; i < n_ops; ++i) TRY(expm(B, P, op_idx[i], thetas[param_idx[i]], v, s));
    return BSIM_OK;
}

template <typename Ti>
int vqe_energy_grad(const DevBasis<Ti> *B, const DevNet<Ti> *H, const DevNet<Ti> *P, i64 n_ops, const i64 *op_idx,
                    const i64 *param_idx, i64 n_params, const double *thetas, const i64 *ref_idx,
                    const double *ref_val, i64 n_ref, i64 ckpt_every, double *lv, double *rv, double *energy,
                    double *variance, double *grad, cudaStream_t s)
{
    const i64 n = B->dim;
    for (i64 i = 0; i < n_ops; ++i) {
        if (op_idx[i] < 0 || op_idx[i] >= P->ngs) { set_error("op_idx[%lld] out of range", i); return BSIM_ERR_ARG; }
        if (param_idx[i] < 0 || param_idx[i] >= n_params) { set_error("param_idx[%lld] out of range", i); return BSIM_ERR_ARG; }
    }
    // checkpoint positions: the state before the first component of every
    // ckpt_every-th parameter
    std::vector<i64> ck_pos;
    if (ckpt_every > 0)
        for (i64 i = 0; i < n_ops; ++i)
            if ((i == 0 || param_idx[i] != param_idx[i - 1]) && param_idx[i] % ckpt_every == 0 && i > 0)
                ck_pos.push_back(i);
    // checkpoints, gradient terms, scalars and the reduction scratch live in the
    // basis workspace (grown on demand, kept between calls): no allocation per call
    const size_t n_ck = (size_t)n * ck_pos.size(), n_terms = (size_t)std::max<i64>(1, n_ops);
    void *wsp = nullptr;
    TRY(workspace_for(B).general(sizeof(double) * (n_ck + n_terms + 8 + kDavPartDoubles + kDavResDoubles), &wsp));
    double *ckp = static_cast<double *>(wsp), *tp = ckp + n_ck, *sc = tp + n_terms;
    DavScratch S;
    S.attach(sc + 8, sc + 8 + kDavPartDoubles);

    // forward: psi_0 = reference, psi_{i+1} = exp(theta G_i) psi_i
    TRY(prepare_state(B, P, 0, op_idx, param_idx, thetas, ref_idx, ref_val, n_ref, lv, s));
    size_t c = 0;
    for (i64 i = 0; i < n_ops; ++i) {
        if (c < ck_pos.size() && ck_pos[c] == i) {
            BSIM_CUDA(cudaMemcpyAsync(ckp + (size_t)c * n, lv, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
            ++c;
        }
        TRY(expm(B, P, op_idx[i], thetas[param_idx[i]], lv, s));
    }
    // energy: r = H l, E = <l|r>/<l|l>
    TRY(sigma(B, H, lv, nullptr, rv, false, s));
    TRY(dav_dot(S, n, lv, lv, sc + 0, s));
    TRY(dav_dot(S, n, lv, rv, sc + 1, s));
    TRY(dav_dot(S, n, rv, rv, sc + 2, s));
    // reverse sweep
    for (i64 i = n_ops - 1; i >= 0; --i) {
        TRY(backgrad(B, P, op_idx[i], thetas[param_idx[i]], lv, rv, tp + i, false, s));
        if (c > 0 && ck_pos[c - 1] == i) {
            --c;
            BSIM_CUDA(cudaMemcpyAsync(lv, ckp + (size_t)c * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        }
    }
    std::vector<double> h_terms(std::max<i64>(1, n_ops)), h_sc(3);
    BSIM_CUDA(cudaMemcpyAsync(h_terms.data(), tp, sizeof(double) * n_ops, cudaMemcpyDeviceToHost, s));
    BSIM_CUDA(cudaMemcpyAsync(h_sc.data(), sc, sizeof(double) * 3, cudaMemcpyDeviceToHost, s));
    BSIM_CUDA(cudaStreamSynchronize(s));
    const double ll = h_sc[0], lr = h_sc[1], rr = h_sc[2];
    const double E = lr / ll;
    if (energy) *energy = E;
    if (variance) *variance = std::max(0.0, rr / ll - E * E);
    if (grad) {
        for (i64 p = 0; p < n_params; ++p) grad[p] = 0.0;
        for (i64 i = 0; i < n_ops; ++i) grad[param_idx[i]] += 2.0 * h_terms[i] / ll;
    }
    return BSIM_OK;
}

template int prepare_state<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, i64, const i64 *,
                                     const i64 *, const double *, const i64 *, const double *, i64, double *,
                                     cudaStream_t);
template int vqe_energy_grad<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *,
                                       const DevNet<unsigned> *, i64, const i64 *, const i64 *, i64, const double *,
                                       const i64 *, const double *, i64, i64, double *, double *, double *, double *,
                                       double *, cudaStream_t);
template int prepare_state<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, i64, const i64 *,
                                     const i64 *, const double *, const i64 *, const double *, i64, double *,
                                     cudaStream_t);
template int vqe_energy_grad<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *,
                                       const DevNet<unsigned long long> *, i64, const i64 *, const i64 *, i64, const double *,
                                       const i64 *, const double *, i64, i64, double *, double *, double *, double *,
                                       double *, cudaStream_t);

}  // namespace bsim
