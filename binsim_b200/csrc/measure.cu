// Measurement helpers: the CUDA-core FMA peak that the sigma kernels' compute
// roofline is quoted against (the driver-measured peaks cover HBM and bf16
// tensor throughput only).
#include "ops.h"

#include <algorithm>

namespace bsim {

namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_chain_kernel(T *__restrict__ out, int iters, T a, T b)
{
    T x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = (T)(threadIdx.x + k) * (T)1e-3;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == (T)-12345.0) out[blockIdx.x] = s;   // keeps the chains live; never true for these inputs
}

}  // namespace

int fma_peak(bool fp64, double *tflops, cudaStream_t s)
{
    int dev = 0, sms = 0;
    BSIM_CUDA(cudaGetDevice(&dev));
    BSIM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8, threads = 256, iters = 8192;
    void *out = nullptr;
    BSIM_CUDA(cudaMallocAsync(&out, sizeof(double) * blocks, s));
    cudaEvent_t e0, e1;
    BSIM_CUDA(cudaEventCreate(&e0));
    BSIM_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        BSIM_CUDA(cudaEventRecord(e0, s));
        if (fp64) fma_chain_kernel<double><<<blocks, threads, 0, s>>>((double *)out, iters, 0.9999999, 1e-7);
        else fma_chain_kernel<float><<<blocks, threads, 0, s>>>((float *)out, iters, 0.9999999f, 1e-7f);
        BSIM_CUDA(cudaEventRecord(e1, s));
        BSIM_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        BSIM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0) best = std::min(best, ms);   // the first launch is a warm-up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BSIM_CUDA(cudaFreeAsync(out, s));
    const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return BSIM_OK;
}

}  // namespace bsim
