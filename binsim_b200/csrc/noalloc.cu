// grad without any device allocation: bsim_grad_noalloc.
//
// Some hosts cannot call cudaMalloc once they are running: a host whose
// memory pool (for example a Julia or Python framework's caching allocator)
// has reserved the whole device, or a latency-critical loop where an
// allocation's implicit device synchronisation is not acceptable.  The regular
// bsim_grad allocates its reduction scratch in the basis workspace on first
// use; this variant takes its scratch from a fixed array compiled into the
// library instead, so no call ever allocates.
//
// The scratch is one file-scope __device__ array of kNoAllocSlots doubles
// (512 KiB plus a ticket word).  Every GPU that loads the library holds it
// until the process exits.  All calls share it and it keeps the previous
// call's contents, so calls whose kernels overlap on the GPU (different
// streams, or different host threads) race; issue them on one stream.
#include "../../include/binsim_cuotf.h"
#include "ops.h"

#include <mutex>

namespace bsim {

// one partial sum per CTA of the row-pair kernel, plus one ticket word
constexpr size_t kNoAllocSlots = 65536;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocSlots + 1];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device.  In host code the
// symbol's name is only a host-side stand-in, never a device address, so the
// address is looked up once per device (with that device current) and cached.
int scratch_address(double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) { set_error("device ordinal %d out of range", dev); return BSIM_ERR_ARG; }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_addr[dev] = static_cast<double *>(p);
    }
    *out = g_addr[dev];
    return BSIM_OK;
}
}  // namespace

template <typename Ti>
int grad_noalloc(const DevBasis<Ti> *B, const DevNet<Ti> *N, i64 gidx, double theta, const double *l,
                 const double *r, double *out_dev, cudaStream_t s)
{
    const size_t nslots = (size_t)pair_grid(B);
    if (nslots > kNoAllocSlots) {
        set_error("grad_noalloc: %zu partial sums needed (alpha strings x blocks) but the fixed scratch holds %zu",
                  nslots, kNoAllocSlots);
        return BSIM_ERR_TOO_LARGE;
    }
    double *scratch = nullptr;
    int st = scratch_address(&scratch);
    if (st != BSIM_OK) return st;
    // the ticket that elects the last CTA must start at zero
    cudaError_t e = cudaMemsetAsync(scratch + nslots, 0, sizeof(double), s);
    if (e != cudaSuccess) return cuda_status(e, "grad_noalloc ticket reset");
    return grad(B, N, gidx, theta, l, r, out_dev, false, s, scratch, nslots + 1);
}

template int grad_noalloc<unsigned>(const DevBasis<unsigned> *, const DevNet<unsigned> *, i64, double,
                                    const double *, const double *, double *, cudaStream_t);
template int grad_noalloc<unsigned long long>(const DevBasis<unsigned long long> *, const DevNet<unsigned long long> *, i64, double,
                                    const double *, const double *, double *, cudaStream_t);

}  // namespace bsim

extern "C" int bsim_grad_noalloc(void *basis, void *net, int64_t idx, double theta, const double *l, const double *r,
                                 double *out_dev, bsim_stream_t stream)
{
    if (!l || !r || !out_dev) { bsim::set_error("null vector or output pointer"); return bsim::BSIM_ERR_NULL; }
    if (bsim::is_u64_basis(basis)) {   // UInt64 strings
        auto *b = static_cast<bsim::DevBasis<unsigned long long> *>(basis);
        auto *n = static_cast<bsim::DevNet<unsigned long long> *>(net);
        if (!bsim::valid(b)) { bsim::set_error("invalid basis handle"); return bsim::BSIM_ERR_ARG; }
        if (!bsim::valid(n)) { bsim::set_error("invalid network handle"); return bsim::BSIM_ERR_ARG; }
        return bsim::grad_noalloc(b, n, idx, theta, l, r, out_dev, stream);
    }
    auto *b = static_cast<bsim::DevBasis<unsigned> *>(basis);
    auto *n = static_cast<bsim::DevNet<unsigned> *>(net);
    if (!bsim::valid(b)) { bsim::set_error("invalid basis handle"); return bsim::BSIM_ERR_ARG; }
    if (!bsim::valid(n)) { bsim::set_error("invalid network handle"); return bsim::BSIM_ERR_ARG; }
    return bsim::grad_noalloc(b, n, idx, theta, l, r, out_dev, stream);
}
