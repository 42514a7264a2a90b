// extern "C" entry points of libcuotf (declared in include/binsim_cuotf.h).
#include "../../include/binsim_cuotf.h"
#include "dav.h"
#include "mixed.cuh"
#include "vqe.h"

#include <cstdio>
#include <initializer_list>
#include <memory>
#include <mutex>

using bsim::DevBasis;
using bsim::DevNet;
using bsim::i64;

namespace {

using Basis = DevBasis<unsigned>;
using Net = DevNet<unsigned>;

int check(void *b, void *n)
{
    if (!bsim::valid(static_cast<Basis *>(b))) { bsim::set_error("invalid basis handle"); return BSIM_ERR_ARG; }
    if (n && !bsim::valid(static_cast<Net *>(n))) { bsim::set_error("invalid network handle"); return BSIM_ERR_ARG; }
    return BSIM_OK;
}

Basis *B(void *p) { return static_cast<Basis *>(p); }
Net *N(void *p) { return static_cast<Net *>(p); }

// f(basis) for a valid basis handle of either string type (no-op otherwise)
template <class F>
void with_handles_basis(void *basis, F &&f)
{
    if (bsim::is_u64_basis(basis)) f(static_cast<DevBasis<unsigned long long> *>(basis));
    else if (bsim::valid(B(basis))) f(B(basis));
    else bsim::set_error("invalid basis handle");
}

// Legacy entry points report like the reference (stderr) but do not exit.
void report(int st, const char *where)
{
    if (st != BSIM_OK) fprintf(stderr, "libcuotf %s: %s (status %d)\n", where, bsim::last_error(), st);
}

// A result slot for the synchronous legacy grad/backgrad: one device double per
// basis handle, allocated on first use.
double *result_slot(Basis *b)
{
    double *p = nullptr;
    const size_t ns = (size_t)bsim::pair_grid(b);
    // partials [ns] + ticket + result: reuse the workspace, keeping its layout
    if (b->ws.partials(ns + 2, &p) != BSIM_OK) return nullptr;
    return p + ns + 1;
}

std::mutex g_dav_mu;
bsim::DavScratch &dav_scratch()
{
    static bsim::DavScratch S;
    return S;
}

// Calls f(basis, net...) with handles of the basis' string type (UInt32 or UInt64,
// told by the handles' magic words); every network must match the basis' type.
template <class F>
int with_handles(void *basis, std::initializer_list<void *> nets, F &&f)
{
    if (bsim::is_u64_basis(basis)) {
        auto *b = static_cast<DevBasis<unsigned long long> *>(basis);
        for (void *n : nets)
            if (!bsim::valid(static_cast<DevNet<unsigned long long> *>(n))) {
                bsim::set_error("network handle is not a UInt64 network of this library");
                return BSIM_ERR_ARG;
            }
        return f(b);
    }
    if (!bsim::valid(B(basis))) { bsim::set_error("invalid basis handle"); return BSIM_ERR_ARG; }
    for (void *n : nets)
        if (!bsim::valid(N(n))) { bsim::set_error("invalid network handle (or string type differs from the basis)"); return BSIM_ERR_ARG; }
    return f(B(basis));
}
// handle validation first (bad handles report BSIM_ERR_ARG before argument checks)
int check_handles(void *basis, std::initializer_list<void *> nets)
{
    return with_handles(basis, nets, [](auto *) { return (int)BSIM_OK; });
}

template <typename Ti>
DevNet<Ti> *net_of(DevBasis<Ti> *, void *n) { return static_cast<DevNet<Ti> *>(n); }

}  // namespace

extern "C" {

// ============================== Part 1 ======================================
void sync_device_cuda(void) { cudaDeviceSynchronize(); }

void *build_basisdev_f64(void *host_basis)
{
    Basis *out = nullptr;
    int st = bsim::basis_from_ref_handle(host_basis, &out);
    report(st, "build_basisdev_f64");
    return out;
}

void destroy_basisdev_f64(void *basis)
{
    if (basis && bsim::valid(B(basis))) delete B(basis);
}

void *build_networkdev_f64(void *host_net)
{
    Net *out = nullptr;
    int st = bsim::network_from_ref_handle(host_net, &out);
    report(st, "build_networkdev_f64");
    return out;
}

void destroy_networkdev_f64(void *net)
{
    if (net && bsim::valid(N(net))) delete N(net);
}

void hvec_cuda(void *basis, void *net, const double *src, double *dst)
{
    report(bsim_hvec(basis, net, src, dst, nullptr), "hvec_cuda");
}

void get_diags_elements_cuda(void *basis, void *net, double *diags)
{
    report(bsim_diag(basis, net, diags, nullptr), "get_diags_elements_cuda");
}

void expm_cuda(void *basis, void *net, int64_t idx, double theta, double *vec)
{
    report(bsim_expm(basis, net, idx, theta, vec, nullptr), "expm_cuda");
}

static double legacy_scalar(void *basis, void *net, int64_t idx, double theta, double *l, double *r, bool back,
                            const char *name)
{
    int st = check(basis, net);
    double h = 0.0;
    if (st == BSIM_OK) {
        double *slot = result_slot(B(basis));
        if (!slot) st = BSIM_ERR_ALLOC;
        else {
            st = back ? bsim::backgrad(B(basis), N(net), idx, theta, l, r, slot, false, nullptr)
                      : bsim::grad(B(basis), N(net), idx, theta, l, r, slot, false, nullptr);
            if (st == BSIM_OK) {
                cudaError_t e = cudaMemcpy(&h, slot, sizeof(double), cudaMemcpyDeviceToHost);
                if (e != cudaSuccess) st = bsim::cuda_status(e, name);
            }
        }
    }
    report(st, name);
    return h;
}

double grad_cuda(void *basis, void *net, int64_t idx, double theta, const double *l, const double *r)
{
    return legacy_scalar(basis, net, idx, theta, const_cast<double *>(l), const_cast<double *>(r), false, "grad_cuda");
}

double backgrad_cuda(void *basis, void *net, int64_t idx, double theta, double *l, double *r)
{
    return legacy_scalar(basis, net, idx, theta, l, r, true, "backgrad_cuda");
}

void batchgrad_cuda(void *basis, void *net, const double *thetas, const double *l, const double *r, double *grads)
{
    report(bsim_batchgrad(basis, net, thetas, l, r, grads, nullptr), "batchgrad_cuda");
}

void tvec_cuda(void *basis, void *net, int64_t idx, const double *src, double *dst)
{
    report(bsim_tvec(basis, net, idx, src, dst, nullptr), "tvec_cuda");
}

void backtran_cuda(void *basis, void *net, int64_t idx, double theta, double *l, double *r, double *b)
{
    report(bsim_backtran(basis, net, idx, theta, l, r, b, nullptr), "backtran_cuda");
}

void batchexpm_cuda(void *basis, void *net, int64_t idx, double theta, double *matrix, int ld, int num_vecs)
{
    report(bsim_batchexpm(basis, net, idx, theta, matrix, ld, num_vecs, nullptr), "batchexpm_cuda");
}

void batchtran_cuda(void *basis, void *net, const double *l, const double *r, double *trans)
{
    report(bsim_batchtran(basis, net, l, r, trans, nullptr), "batchtran_cuda");
}

void expm_cuda_2d(void *basis, void *net, int64_t idx, double theta, double *vec)
{
    expm_cuda(basis, net, idx, theta, vec);
}

double grad_cuda_2d(void *basis, void *net, int64_t idx, double theta, const double *l, const double *r)
{
    return grad_cuda(basis, net, idx, theta, l, r);
}

double backgrad_cuda_2d(void *basis, void *net, int64_t idx, double theta, double *l, double *r)
{
    return backgrad_cuda(basis, net, idx, theta, l, r);
}

// ============================== Part 2 ======================================
const char *bsim_last_error(void) { return bsim::last_error(); }
const char *bsim_version(void) { return "libcuotf sm_100a 0.1"; }
int64_t bsim_device_alloc_count(void) { return (int64_t)bsim::device_alloc_count(); }
int bsim_release_cached_memory(void)
{
    const cudaError_t e = bsim::trim_library_pool();
    return e == cudaSuccess ? bsim::BSIM_OK : bsim::cuda_status(e, "release cached memory");
}

int bsim_tensor_core_timeouts(int32_t *count, int32_t reset)
{
    if (!count) { bsim::set_error("null count"); return bsim::BSIM_ERR_NULL; }
    int c = 0;
    const int st = bsim::mixed_tc_timeouts(&c, reset != 0);
    *count = c;
    return st;
}

int bsim_basis_create_u32(int64_t norb, int64_t na, int64_t nb, int64_t total_sym, const int64_t *orbsym,
                          int64_t num_irreps, void **out)
{
    if (!out) { bsim::set_error("null out"); return BSIM_ERR_NULL; }
    Basis *b = nullptr;
    int st = bsim::make_basis<unsigned>(norb, na, nb, total_sym, (const i64 *)orbsym, num_irreps, &b);
    *out = b;
    return st;
}

int bsim_basis_from_host(void *host_basis, void **out)
{
    if (!out) { bsim::set_error("null out"); return BSIM_ERR_NULL; }
    Basis *b = nullptr;
    int st = bsim::basis_from_ref_handle(host_basis, &b);
    *out = b;
    return st;
}

int bsim_basis_create_u64(int64_t norb, int64_t na, int64_t nb, int64_t total_sym, const int64_t *orbsym,
                          int64_t num_irreps, void **out)
{
    if (!out) { bsim::set_error("null out"); return BSIM_ERR_NULL; }
    DevBasis<unsigned long long> *b = nullptr;
    int st = bsim::make_basis<unsigned long long>(norb, na, nb, total_sym, (const i64 *)orbsym, num_irreps, &b);
    *out = b;
    return st;
}

int bsim_basis_destroy(void *basis)
{
    if (bsim::is_u64_basis(basis)) {
        delete static_cast<DevBasis<unsigned long long> *>(basis);
        return BSIM_OK;
    }
    int st = check(basis, nullptr);
    if (st == BSIM_OK) delete B(basis);
    return st;
}

int64_t bsim_basis_dim(void *basis)
{
    int64_t d = -1;
    with_handles_basis(basis, [&](auto *b) { d = b->dim; });
    return d;
}

int64_t bsim_basis_find_det(void *basis, uint64_t astr, uint64_t bstr)
{
    int64_t i = -1;
    with_handles_basis(basis, [&](auto *b) { i = b->find_det(astr, bstr); });
    return i;
}

int bsim_network_create_u32(const int64_t *orbsym, int64_t norb, int64_t ngs, const uint32_t *axs,
                            const uint32_t *bxs, const int64_t *ranks, const int64_t *num_zas,
                            const int64_t *num_zbs, const uint32_t *flat_zas, const uint32_t *flat_zbs,
                            const double *flat_wa, const double *flat_wb, void **out)
{
    if (!out) { bsim::set_error("null out"); return BSIM_ERR_NULL; }
    Net *n = nullptr;
    int st = bsim::make_network<unsigned>((const i64 *)orbsym, norb, ngs, axs, bxs, (const i64 *)ranks,
                                          (const i64 *)num_zas, (const i64 *)num_zbs, flat_zas, flat_zbs, flat_wa,
                                          flat_wb, &n);
    *out = n;
    return st;
}

int bsim_network_from_host(void *host_net, void **out)
{
    if (!out) { bsim::set_error("null out"); return BSIM_ERR_NULL; }
    Net *n = nullptr;
    int st = bsim::network_from_ref_handle(host_net, &n);
    *out = n;
    return st;
}

int bsim_network_create_u64(const int64_t *orbsym, int64_t norb, int64_t ngs, const uint64_t *axs,
                            const uint64_t *bxs, const int64_t *ranks, const int64_t *num_zas,
                            const int64_t *num_zbs, const uint64_t *flat_zas, const uint64_t *flat_zbs,
                            const double *flat_wa, const double *flat_wb, void **out)
{
    if (!out) { bsim::set_error("null out"); return BSIM_ERR_NULL; }
    DevNet<unsigned long long> *n = nullptr;
    using U = unsigned long long;
    int st = bsim::make_network<U>((const i64 *)orbsym, norb, ngs, (const U *)axs, (const U *)bxs,
                                   (const i64 *)ranks, (const i64 *)num_zas, (const i64 *)num_zbs,
                                   (const U *)flat_zas, (const U *)flat_zbs, flat_wa, flat_wb, &n);
    *out = n;
    return st;
}

int bsim_network_destroy(void *net)
{
    if (bsim::is_c64_net(net)) {
        if (*static_cast<const unsigned *>(net) == bsim::HandleMagic<unsigned long long>::net_c64)
            delete static_cast<DevNet<unsigned long long> *>(net);
        else
            delete static_cast<DevNet<unsigned> *>(net);
        return BSIM_OK;
    }
    if (bsim::is_u64_net(net)) {
        delete static_cast<DevNet<unsigned long long> *>(net);
        return BSIM_OK;
    }
    if (!bsim::valid(N(net))) { bsim::set_error("invalid network handle"); return BSIM_ERR_ARG; }
    delete N(net);
    return BSIM_OK;
}

int64_t bsim_network_ngs(void *net)
{
    if (bsim::is_c64_net(net)) {
        if (*static_cast<const unsigned *>(net) == bsim::HandleMagic<unsigned long long>::net_c64)
            return static_cast<DevNet<unsigned long long> *>(net)->ngs;
        return static_cast<DevNet<unsigned> *>(net)->ngs;
    }
    if (bsim::is_u64_net(net)) return static_cast<DevNet<unsigned long long> *>(net)->ngs;
    return bsim::valid(N(net)) ? N(net)->ngs : -1;
}

#define NEED(p) do { if (!(p)) { bsim::set_error("null pointer argument: %s", #p); return BSIM_ERR_NULL; } } while (0)

int bsim_hvec(void *basis, void *net, const double *src, double *dst, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(src); NEED(dst);
    return with_handles(basis, {net}, [&](auto *b) { return bsim::sigma(b, net_of(b, net), src, nullptr, dst, false, stream); });
}

namespace {

// Device side of bsim_hvec_host: two input and two output vectors, a copy
// stream per direction and the events that order them.
struct HostPipe {
    double *in[2] = {nullptr, nullptr}, *out[2] = {nullptr, nullptr};
    cudaStream_t cin = nullptr, cout = nullptr;
    cudaEvent_t in_ready[2] = {}, done[2] = {}, out_read[2] = {};
    ~HostPipe()
    {
        for (int i = 0; i < 2; ++i) {
            if (in[i]) cudaFree(in[i]);
            if (out[i]) cudaFree(out[i]);
            for (cudaEvent_t e : {in_ready[i], done[i], out_read[i]})
                if (e) cudaEventDestroy(e);
        }
        if (cin) cudaStreamDestroy(cin);
        if (cout) cudaStreamDestroy(cout);
    }
    int init(int64_t dim)
    {
        for (int i = 0; i < 2; ++i) {
            BSIM_CUDA(bsim::dmalloc(&in[i], sizeof(double) * std::max<int64_t>(dim, 1)));
            BSIM_CUDA(bsim::dmalloc(&out[i], sizeof(double) * std::max<int64_t>(dim, 1)));
            BSIM_CUDA(cudaEventCreateWithFlags(&in_ready[i], cudaEventDisableTiming));
            BSIM_CUDA(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming));
            BSIM_CUDA(cudaEventCreateWithFlags(&out_read[i], cudaEventDisableTiming));
        }
        BSIM_CUDA(cudaStreamCreateWithFlags(&cin, cudaStreamNonBlocking));
        BSIM_CUDA(cudaStreamCreateWithFlags(&cout, cudaStreamNonBlocking));
        return BSIM_OK;
    }
};

}  // namespace

int bsim_hvec_host(void *basis, void *net, int64_t nvec, const double *const *src_host, double *const *dst_host,
                   int mixed, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    if (nvec < 0) { bsim::set_error("nvec = %lld", (long long)nvec); return BSIM_ERR_ARG; }
    if (nvec == 0) return BSIM_OK;
    NEED(src_host); NEED(dst_host);
    for (int64_t k = 0; k < nvec; ++k) { NEED(src_host[k]); NEED(dst_host[k]); }
    return with_handles(basis, {net}, [&](auto *b) -> int {
        const int64_t dim = b->dim;
        const size_t bytes = sizeof(double) * (size_t)dim;
        // one pipe per process, kept between calls and regrown for a larger basis
        static std::mutex mu;
        static std::unique_ptr<HostPipe> pipe;
        static int64_t pipe_dim = -1;
        std::lock_guard<std::mutex> lk(mu);
        int st = BSIM_OK;
        if (!pipe || pipe_dim < dim) {
            pipe.reset();
            pipe_dim = -1;
            auto np = std::make_unique<HostPipe>();
            if ((st = np->init(dim)) != BSIM_OK) return st;
            pipe = std::move(np);
            pipe_dim = dim;
        }
        HostPipe &P = *pipe;
        // step k: H2D on cin into in[k%2] (after sigma k-2 read it), sigma on the
        // caller's stream into out[k%2] (after the D2H of step k-2 read it), D2H
        // on cout; the copies of neighbouring steps overlap the sigma between them
        for (int64_t k = 0; k < nvec; ++k) {
            const int sl = (int)(k & 1);
            if (k >= 2) BSIM_CUDA(cudaStreamWaitEvent(P.cin, P.done[sl], 0));
            BSIM_CUDA(cudaMemcpyAsync(P.in[sl], src_host[k], bytes, cudaMemcpyHostToDevice, P.cin));
            BSIM_CUDA(cudaEventRecord(P.in_ready[sl], P.cin));
            BSIM_CUDA(cudaStreamWaitEvent(stream, P.in_ready[sl], 0));
            if (k >= 2) BSIM_CUDA(cudaStreamWaitEvent(stream, P.out_read[sl], 0));
            st = bsim::sigma(b, net_of(b, net), P.in[sl], nullptr, P.out[sl], mixed != 0, stream);
            if (st != BSIM_OK) break;
            BSIM_CUDA(cudaEventRecord(P.done[sl], stream));
            BSIM_CUDA(cudaStreamWaitEvent(P.cout, P.done[sl], 0));
            BSIM_CUDA(cudaMemcpyAsync(dst_host[k], P.out[sl], bytes, cudaMemcpyDeviceToHost, P.cout));
            BSIM_CUDA(cudaEventRecord(P.out_read[sl], P.cout));
        }
        cudaError_t e1 = cudaStreamSynchronize(P.cout), e2 = cudaStreamSynchronize(stream);
        // keep the pipeline's four vectors between calls only while they are small
        // (8 GB in all); larger ones are released with the call
        if (4.0 * (double)bytes > 8e9) {
            pipe.reset();
            pipe_dim = -1;
        }
        if (st != BSIM_OK) return st;
        if (e1 != cudaSuccess) return bsim::cuda_status(e1, "hvec_host");
        if (e2 != cudaSuccess) return bsim::cuda_status(e2, "hvec_host");
        return (int)BSIM_OK;
    });
}

int bsim_hvec_mixed(void *basis, void *net, const double *src, double *dst, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(src); NEED(dst);
    return with_handles(basis, {net}, [&](auto *b) { return bsim::sigma(b, net_of(b, net), src, nullptr, dst, true, stream); });
}

int bsim_hvec_f32in(void *basis, void *net, const float *src, double *dst, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(src); NEED(dst);
    return with_handles(basis, {net}, [&](auto *b) { return bsim::sigma(b, net_of(b, net), nullptr, src, dst, true, stream); });
}

int bsim_hvec_path(void *basis, void *net, char *why, int why_len, int *residual_groups)
{
    return with_handles(basis, {net}, [&](auto *b) -> int {
        std::string w;
        int nres = 0;
        const int r = bsim::fast_sigma_info(b, net_of(b, net), &w, &nres);
        if (r < 0) return r;
        if (why && why_len > 0) snprintf(why, why_len, "%s", w.c_str());
        if (residual_groups) *residual_groups = nres;
        return r;
    });
}

int bsim_hvec_cols(void *basis, void *net, const double *src, double *dst, int64_t col_lo, int64_t col_hi,
                   int mixed, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(src); NEED(dst);
    return with_handles(basis, {net}, [&](auto *b) {
        return bsim::sigma_fast_cols(b, net_of(b, net), src, dst, mixed != 0, col_lo, col_hi, stream);
    });
}

int bsim_hvec_stage_times(void *basis, void *net, const double *src, double *dst, int mixed, double *ms_out,
                          int *launches_out, int nstages, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(src); NEED(dst); NEED(ms_out); NEED(launches_out);
    return with_handles(basis, {net}, [&](auto *b) {
        return bsim::sigma_fast_stages(b, net_of(b, net), src, dst, mixed != 0, stream, ms_out, launches_out, nstages);
    });
}

int bsim_fma_peak(int fp64, double *tflops_out, bsim_stream_t stream)
{
    NEED(tflops_out);
    return bsim::fma_peak(fp64 == 2 ? 2 : (fp64 != 0 ? 1 : 0), tflops_out, stream);
}

int64_t bsim_hvec_num_tiles(void *basis)
{
    int64_t n = -1;
    with_handles(basis, {}, [&](auto *b) { n = bsim::num_tiles(b); return BSIM_OK; });
    return n;
}

int bsim_hvec_tiles(void *basis, void *net, const double *src, double *dst, int64_t tile_lo, int64_t tile_hi,
                    int mixed, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(src); NEED(dst);
    return with_handles(basis, {net}, [&](auto *b) {
        return bsim::sigma_tiles(b, net_of(b, net), src, nullptr, dst, mixed != 0, tile_lo, tile_hi, stream);
    });
}

int bsim_diag(void *basis, void *net, double *diags, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(diags);
    return with_handles(basis, {net}, [&](auto *b) { return bsim::diag_elements(b, net_of(b, net), diags, stream); });
}

int bsim_expm(void *basis, void *net, int64_t idx, double theta, double *vec, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(vec);
    return with_handles(basis, {net}, [&](auto *b) { return bsim::expm(b, net_of(b, net), idx, theta, vec, stream); });
}

int bsim_expm_seq(void *basis, void *net, int64_t n, const int64_t *idx, const double *theta, double *vec,
                  bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(vec);
    if (n > 0) { NEED(idx); NEED(theta); }
    return with_handles(basis, {net}, [&](auto *b) {
        for (int64_t i = 0; i < n; ++i) {
            int st = bsim::expm(b, net_of(b, net), idx[i], theta[i], vec, stream);
            if (st != BSIM_OK) return st;
        }
        return (int)BSIM_OK;
    });
}

int bsim_grad(void *basis, void *net, int64_t idx, double theta, const double *l, const double *r,
              double *out_dev, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(l); NEED(r); NEED(out_dev);
    return with_handles(basis, {net}, [&](auto *b) {
        return bsim::grad(b, net_of(b, net), idx, theta, l, r, out_dev, false, stream);
    });
}

int bsim_backgrad(void *basis, void *net, int64_t idx, double theta, double *l, double *r, double *out_dev,
                  bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(l); NEED(r); NEED(out_dev);
    return with_handles(basis, {net}, [&](auto *b) {
        return bsim::backgrad(b, net_of(b, net), idx, theta, l, r, out_dev, false, stream);
    });
}

int bsim_batchgrad(void *basis, void *net, const double *thetas, const double *l, const double *r, double *grads,
                   bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(thetas); NEED(l); NEED(r); NEED(grads);
    return with_handles(basis, {net}, [&](auto *b) {
        return bsim::batchgrad(b, net_of(b, net), thetas, l, r, grads, stream);
    });
}

int bsim_tvec(void *basis, void *net, int64_t idx, const double *src, double *dst, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(src); NEED(dst);
    return with_handles(basis, {net}, [&](auto *b) { return bsim::tvec(b, net_of(b, net), idx, src, dst, stream); });
}

int bsim_backtran(void *basis, void *net, int64_t idx, double theta, double *l, double *r, double *bvec,
                  bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(l); NEED(r); NEED(bvec);
    return with_handles(basis, {net}, [&](auto *b) {
        return bsim::backtran(b, net_of(b, net), idx, theta, l, r, bvec, stream);
    });
}

int bsim_batchexpm(void *basis, void *net, int64_t idx, double theta, double *matrix, int ld, int num_vecs,
                   bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(matrix);
    return with_handles(basis, {net}, [&](auto *b) {
        return bsim::batchexpm(b, net_of(b, net), idx, theta, matrix, ld, num_vecs, stream);
    });
}

int bsim_batchtran(void *basis, void *net, const double *l, const double *r, double *trans, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(l); NEED(r); NEED(trans);
    return with_handles(basis, {net}, [&](auto *b) { return bsim::batchtran(b, net_of(b, net), l, r, trans, stream); });
}

int bsim_prepare_state(void *basis, void *pool, int64_t n_ops, const int64_t *op_idx, const int64_t *param_idx,
                       const double *thetas, const int64_t *ref_idx, const double *ref_val, int64_t n_ref,
                       double *vec, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {pool})) return st0;
    NEED(vec);
    if (n_ops > 0) { NEED(op_idx); NEED(param_idx); NEED(thetas); }
    if (n_ref > 0) { NEED(ref_idx); NEED(ref_val); }
    return with_handles(basis, {pool}, [&](auto *b) -> int {
        auto *P = net_of(b, pool);
        for (int64_t i = 0; i < n_ops; ++i)
            if (op_idx[i] < 0 || op_idx[i] >= P->ngs || param_idx[i] < 0) {
                bsim::set_error("op_idx/param_idx[%lld] out of range", (long long)i);
                return BSIM_ERR_ARG;
            }
        return bsim::prepare_state(b, P, n_ops, (const i64 *)op_idx, (const i64 *)param_idx, thetas,
                                   (const i64 *)ref_idx, ref_val, n_ref, vec, stream);
    });
}

int bsim_vqe_energy_grad(void *basis, void *ham, void *pool, int64_t n_ops, const int64_t *op_idx,
                         const int64_t *param_idx, int64_t n_params, const double *thetas, const int64_t *ref_idx,
                         const double *ref_val, int64_t n_ref, int64_t ckpt_every, double *lv, double *rv,
                         double *energy, double *variance, double *grad, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {ham, pool})) return st0;
    NEED(lv); NEED(rv);
    if (n_ops > 0) { NEED(op_idx); NEED(param_idx); NEED(thetas); }
    if (n_ref > 0) { NEED(ref_idx); NEED(ref_val); }
    return with_handles(basis, {ham, pool}, [&](auto *b) {
        return bsim::vqe_energy_grad(b, net_of(b, ham), net_of(b, pool), n_ops, (const i64 *)op_idx,
                                     (const i64 *)param_idx, n_params, thetas, (const i64 *)ref_idx, ref_val, n_ref,
                                     ckpt_every, lv, rv, energy, variance, grad, stream);
    });
}

int bsim_davidson(void *basis, void *net, double *v0, const double *diags, double tol, int maxiter, int ncv,
                  int maxspace, int mixed, double *x_out, double *energy, double *residual, int *iterations,
                  int *sigma_fp64, int *sigma_fp32, int verbose, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(v0); NEED(diags); NEED(x_out);
    bsim::DavStats st{};
    int rc = with_handles(basis, {net}, [&](auto *b) {
        return mixed ? bsim::davidson_mixed(b, net_of(b, net), v0, diags, tol, maxiter, maxspace, x_out, &st, verbose,
                                            stream)
                     : bsim::davidson_fp64(b, net_of(b, net), v0, diags, tol, maxiter, ncv, maxspace, x_out, &st,
                                           verbose, stream);
    });
    if (rc == BSIM_OK) {
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) rc = bsim::cuda_status(e, "davidson");
    }
    if (energy) *energy = st.energy;
    if (residual) *residual = st.residual;
    if (iterations) *iterations = st.iterations;
    if (sigma_fp64) *sigma_fp64 = st.sigma_fp64;
    if (sigma_fp32) *sigma_fp32 = st.sigma_fp32;
    return rc;
}

int bsim_davidson_block(void *basis, void *net, int nroots, double *X, const void *diags, int diag_fp32, double tol,
                        int maxiter, int ncv, int maxspace, int mixed, double *energies, double *residuals,
                        int *iterations, int *sigma_fp64, int *sigma_fp32, int verbose, bsim_stream_t stream)
{
    if (int st0 = check_handles(basis, {net})) return st0;
    NEED(X); NEED(diags);
    bsim::DavBlockStats st{};
    int rc = with_handles(basis, {net}, [&](auto *b) {
        return bsim::davidson_block(b, net_of(b, net), nroots, X, diags, diag_fp32 != 0, tol, maxiter, ncv, maxspace,
                                    mixed != 0, &st, verbose, stream);
    });
    if (rc == BSIM_OK) {
        cudaError_t e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) rc = bsim::cuda_status(e, "davidson_block");
    }
    for (int i = 0; i < nroots && i < bsim::kMaxRoots; ++i) {
        if (energies) energies[i] = st.energy[i];
        if (residuals) residuals[i] = st.residual[i];
    }
    if (iterations) *iterations = st.iterations;
    if (sigma_fp64) *sigma_fp64 = st.sigma_fp64;
    if (sigma_fp32) *sigma_fp32 = st.sigma_fp32;
    return rc;
}

// ============================== Part 3 ======================================
static double fetch1(const double *dev)
{
    double h = 0.0;
    cudaError_t e = cudaMemcpy(&h, dev, sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) report(bsim::cuda_status(e, "davidson helper"), "davidson helper");
    return h;
}

double build_ritz_and_residual_cuda(int64_t N, int dim, const double *coeffs, double min_e, const double **V,
                                    const double **AV, double *axt)
{
    std::lock_guard<std::mutex> g(g_dav_mu);
    auto &S = dav_scratch();
    int st = S.ensure();
    if (st == BSIM_OK) st = bsim::dav_ritz_residual<double>(S, N, dim, coeffs, min_e, V, AV, axt, S.res, nullptr);
    report(st, "build_ritz_and_residual_cuda");
    return st == BSIM_OK ? fetch1(S.res) : 0.0;
}

void build_ritz_vector_cuda(int64_t N, int dim, const double *coeffs, const double **V, double *xt)
{
    int st = bsim::dav_combine<double, double>(N, dim, coeffs, V, xt, nullptr);
    if (st == BSIM_OK) cudaDeviceSynchronize();
    report(st, "build_ritz_vector_cuda");
}

void apply_preconditioner_inplace_cuda(int64_t N, double *axt, const double *diags, double min_e, double shift)
{
    std::lock_guard<std::mutex> g(g_dav_mu);
    auto &S = dav_scratch();
    int st = bsim::dav_precondition(S, N, axt, diags, min_e, shift, nullptr, nullptr);
    if (st == BSIM_OK) cudaDeviceSynchronize();
    report(st, "apply_preconditioner_inplace_cuda");
}

double mgs_orthogonalize_cuda(int64_t N, int dim, const double **V, double *vt)
{
    std::lock_guard<std::mutex> g(g_dav_mu);
    auto &S = dav_scratch();
    int st = S.ensure();
    if (st == BSIM_OK) st = bsim::dav_mgs<double>(S, N, dim, V, vt, S.res + bsim::kMaxSub, nullptr);
    report(st, "mgs_orthogonalize_cuda");
    return st == BSIM_OK ? fetch1(S.res + bsim::kMaxSub) : 0.0;
}

double inplace_normalize_cuda(int64_t N, double *vec)
{
    std::lock_guard<std::mutex> g(g_dav_mu);
    auto &S = dav_scratch();
    int st = S.ensure();
    if (st == BSIM_OK) st = bsim::dav_normalize(S, N, vec, S.res, nullptr);
    report(st, "inplace_normalize_cuda");
    return st == BSIM_OK ? fetch1(S.res) : 0.0;
}

double fast_dot_cuda(int64_t N, const double *v1, const double *v2)
{
    std::lock_guard<std::mutex> g(g_dav_mu);
    auto &S = dav_scratch();
    int st = S.ensure();
    if (st == BSIM_OK) st = bsim::dav_dot(S, N, v1, v2, S.res, nullptr);
    report(st, "fast_dot_cuda");
    return st == BSIM_OK ? fetch1(S.res) : 0.0;
}

void compute_heff_col_cuda(int64_t N, int dim, const double **V, const double *AV_dim, double *out_col)
{
    std::lock_guard<std::mutex> g(g_dav_mu);
    auto &S = dav_scratch();
    int st = S.ensure();
    if (st == BSIM_OK) st = bsim::dav_multidot<double, double>(S, N, dim, V, AV_dim, S.res, nullptr);
    if (st == BSIM_OK) {
        cudaError_t e = cudaMemcpy(out_col, S.res, sizeof(double) * dim, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) st = bsim::cuda_status(e, "compute_heff_col_cuda");
    }
    report(st, "compute_heff_col_cuda");
}

void rebuild_heff_cuda(int64_t N, int dim, const double **V, const double **AV, double *heff, int ldh)
{
    std::lock_guard<std::mutex> g(g_dav_mu);
    auto &S = dav_scratch();
    int st = S.ensure();
    double col[bsim::kMaxSub];
    for (int j = 0; j < dim && st == BSIM_OK; ++j) {
        st = bsim::dav_multidot<double, double>(S, N, dim, V, AV[j], S.res, nullptr);
        if (st == BSIM_OK) {
            cudaError_t e = cudaMemcpy(col, S.res, sizeof(double) * dim, cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) st = bsim::cuda_status(e, "rebuild_heff_cuda");
        }
        for (int i = 0; i < dim && st == BSIM_OK; ++i) heff[i + (int64_t)j * ldh] = col[i];
    }
    report(st, "rebuild_heff_cuda");
}

}  // extern "C"
