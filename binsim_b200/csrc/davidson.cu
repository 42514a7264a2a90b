// Davidson vector operations on device vectors and a device-resident Davidson
// driver (reference diag/davidson.hpp:31-272 and jl/davidson.jl:1-185).
//
// All reductions are deterministic: a fixed grid writes per-CTA partials and a
// single CTA sums them in index order.  The streaming kernels read each vector
// once per call, so they run at HBM bandwidth: a k-vector Ritz/residual step
// moves (2k + 1) * dim * 8 bytes.
#include "dav.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace bsim {

constexpr int kRedCtas = 148 * 8;
constexpr int kRedThreads = 256;

template <typename T>
struct Ptrs { const T *p[kMaxSub]; };

// ---- final reduction: out[j] = sum_b part[b * nout + j] ---------------------------
__global__ void finish_kernel(const double *__restrict__ part, int nblk, int nout, double *__restrict__ out,
                              int sqrt_out)
{
    __shared__ double red[32];
    for (int j = 0; j < nout; ++j) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += part[(i64)b * nout + j];
        s = warp_sum(s);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
            out[j] = sqrt_out ? sqrt(t) : t;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void cta_partial(double v, double *red, double *dst)
{
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        *dst = t;
    }
    __syncthreads();
}

// axt = sum_j c_j AV_j - e sum_j c_j V_j ; partial |axt|^2   (davidson.hpp:31-69)
template <typename TV>
__global__ void ritz_residual_kernel(i64 n, int k, Coeffs c, double e, Ptrs<TV> V, Ptrs<TV> AV,
                                     double *__restrict__ axt, double *__restrict__ part)
{
    __shared__ double red[32];
    double s = 0.0;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        double x = 0.0, ax = 0.0;
        for (int j = 0; j < k; ++j) {
            x += c.v[j] * (double)V.p[j][i];
            ax += c.v[j] * (double)AV.p[j][i];
        }
        const double rr = ax - e * x;
        axt[i] = rr;
        s += rr * rr;
    }
    cta_partial(s, red, part + blockIdx.x);
}

// x = sum_j c_j V_j  (davidson.hpp:71-95); TX may be float or double
template <typename TV, typename TX>
__global__ void combine_kernel(i64 n, int k, Coeffs c, Ptrs<TV> V, TX *__restrict__ x)
{
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < k; ++j) s += c.v[j] * (double)V.p[j][i];
        x[i] = (TX)s;
    }
}

// r_i /= (d_i - e), denominator clamped to +-|shift|  (davidson.hpp:97-117); the
// diagonal may be stored in FP32 (the preconditioner only needs it approximately)
template <typename TD>
__global__ void precondition_kernel(i64 n, double *__restrict__ r, const TD *__restrict__ d, double e,
                                    double shift, double *__restrict__ part)
{
    __shared__ double red[32];
    const double as = fabs(shift);
    double s = 0.0;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        double diff = (double)d[i] - e;
        if (fabs(diff) < as) diff = (diff >= 0) ? as : -as;
        const double v = r[i] / diff;
        r[i] = v;
        s += v * v;
    }
    if (part) cta_partial(s, red, part + blockIdx.x);
}

// One modified Gram-Schmidt step, fused with the next projection:
// v -= p_prev * Vprev (p_prev read from device), partial <Vnext, v>.
template <typename TV>
__global__ void mgs_step_kernel(i64 n, double *__restrict__ v, const TV *__restrict__ vprev,
                                const double *__restrict__ pprev, const TV *__restrict__ vnext,
                                double *__restrict__ part)
{
    __shared__ double red[32];
    const double p = vprev ? *pprev : 0.0;
    double s = 0.0;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        double x = v[i];
        if (vprev) { x -= p * (double)vprev[i]; v[i] = x; }
        s += vnext ? (double)vnext[i] * x : x * x;
    }
    cta_partial(s, red, part + blockIdx.x);
}

__global__ void scale_kernel(i64 n, double *__restrict__ v, const double *__restrict__ nrm)
{
    const double inv = 1.0 / *nrm;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) v[i] *= inv;
}

// out_j partials = <V_j, w> for j < k <= kDotChunk (davidson.hpp:186-219); the
// sums stay in registers (a fixed-size, fully unrolled array), the host splits
// larger subspaces into chunks
constexpr int kDotChunk = 8;
template <typename TV, typename TW>
__global__ void multidot_kernel(i64 n, int k, Ptrs<TV> V, const TW *__restrict__ w, double *__restrict__ part)
{
    __shared__ double red[32];
    double s[kDotChunk];
#pragma unroll
    for (int j = 0; j < kDotChunk; ++j) s[j] = 0.0;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        const double x = (double)w[i];
#pragma unroll
        for (int j = 0; j < kDotChunk; ++j)
            if (j < k) s[j] += (double)V.p[j][i] * x;
    }
#pragma unroll
    for (int j = 0; j < kDotChunk; ++j)
        if (j < k) cta_partial(s[j], red, part + (i64)blockIdx.x * k + j);
}

__global__ void dot_kernel(i64 n, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ part)
{
    __shared__ double red[32];
    double s = 0.0;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) s += a[i] * b[i];
    cta_partial(s, red, part + blockIdx.x);
}

// ---- host wrappers -----------------------------------------------------------------
static_assert(kDavPartDoubles == kRedCtas * kMaxSub, "partial-sum scratch of the reductions");

DavScratch::~DavScratch()
{
    if (!owned) return;
    if (part) cudaFreeAsync(part, stream);
    if (res) cudaFreeAsync(res, stream);
}

int DavScratch::ensure(cudaStream_t s)
{
    if (part) return BSIM_OK;
    owned = true;
    stream = s;
    cudaError_t e = dmalloc_async(&part, sizeof(double) * kDavPartDoubles, s);
    if (e != cudaSuccess) { part = nullptr; return cuda_status(e, "davidson scratch"); }
    e = dmalloc_async(&res, sizeof(double) * kDavResDoubles, s);
    if (e != cudaSuccess) { res = nullptr; return cuda_status(e, "davidson scratch"); }
    return BSIM_OK;
}

static int grid_for(i64 n) { return (int)std::max<i64>(1, std::min<i64>(kRedCtas, (n + kRedThreads - 1) / kRedThreads)); }

template <typename TV>
static Ptrs<TV> pack(const TV *const *v, int k)
{
    Ptrs<TV> p{};
    for (int j = 0; j < k; ++j) p.p[j] = v[j];
    return p;
}

template <typename TV>
int dav_ritz_residual(DavScratch &S, i64 n, int k, const double *coeffs, double e, const TV *const *V,
                      const TV *const *AV, double *axt, double *norm_dev, cudaStream_t s)
{
    if (k < 1 || k > kMaxSub) { set_error("subspace size %d out of range", k); return BSIM_ERR_ARG; }
    int st = S.ensure();
    if (st) return st;
    Coeffs c{};
    for (int j = 0; j < k; ++j) c.v[j] = coeffs[j];
    const int g = grid_for(n);
    ritz_residual_kernel<TV><<<g, kRedThreads, 0, s>>>(n, k, c, e, pack(V, k), pack(AV, k), axt, S.part);
    finish_kernel<<<1, 1024, 0, s>>>(S.part, g, 1, norm_dev, 1);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename TV, typename TX>
int dav_combine(i64 n, int k, const double *coeffs, const TV *const *V, TX *x, cudaStream_t s)
{
    if (k < 1 || k > kMaxSub) { set_error("subspace size %d out of range", k); return BSIM_ERR_ARG; }
    Coeffs c{};
    for (int j = 0; j < k; ++j) c.v[j] = coeffs[j];
    combine_kernel<TV, TX><<<grid_for(n), kRedThreads, 0, s>>>(n, k, c, pack(V, k), x);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename TD>
static int precondition_impl(DavScratch &S, i64 n, double *r, const TD *d, double e, double shift,
                             double *norm_dev, cudaStream_t s)
{
    int st = S.ensure();
    if (st) return st;
    const int g = grid_for(n);
    precondition_kernel<TD><<<g, kRedThreads, 0, s>>>(n, r, d, e, shift, norm_dev ? S.part : nullptr);
    if (norm_dev) finish_kernel<<<1, 1024, 0, s>>>(S.part, g, 1, norm_dev, 1);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

int dav_precondition(DavScratch &S, i64 n, double *r, const double *d, double e, double shift, double *norm_dev,
                     cudaStream_t s)
{
    return precondition_impl(S, n, r, d, e, shift, norm_dev, s);
}

int dav_precondition(DavScratch &S, i64 n, double *r, const float *d, double e, double shift, double *norm_dev,
                     cudaStream_t s)
{
    return precondition_impl(S, n, r, d, e, shift, norm_dev, s);
}

template <typename TV>
int dav_mgs(DavScratch &S, i64 n, int k, const TV *const *V, double *v, double *norm_dev, cudaStream_t s)
{
    int st = S.ensure();
    if (st) return st;
    if (k < 0 || k > kMaxSub) { set_error("subspace size %d out of range", k); return BSIM_ERR_ARG; }
    const int g = grid_for(n);
    // projections p_j land in S.res[j]; the final pass computes |v|^2
    for (int j = 0; j <= k; ++j) {
        const TV *prev = j > 0 ? V[j - 1] : nullptr;
        const TV *next = j < k ? V[j] : nullptr;
        mgs_step_kernel<TV><<<g, kRedThreads, 0, s>>>(n, v, prev, j > 0 ? S.res + (j - 1) : nullptr, next, S.part);
        if (j < k) finish_kernel<<<1, 1024, 0, s>>>(S.part, g, 1, S.res + j, 0);
        else finish_kernel<<<1, 1024, 0, s>>>(S.part, g, 1, norm_dev, 1);
    }
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

int dav_normalize(DavScratch &S, i64 n, double *v, double *norm_dev, cudaStream_t s)
{
    int st = S.ensure();
    if (st) return st;
    const int g = grid_for(n);
    mgs_step_kernel<double><<<g, kRedThreads, 0, s>>>(n, v, nullptr, nullptr, nullptr, S.part);
    finish_kernel<<<1, 1024, 0, s>>>(S.part, g, 1, norm_dev, 1);
    scale_kernel<<<g, kRedThreads, 0, s>>>(n, v, norm_dev);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

int dav_dot(DavScratch &S, i64 n, const double *a, const double *b, double *out_dev, cudaStream_t s)
{
    int st = S.ensure();
    if (st) return st;
    const int g = grid_for(n);
    dot_kernel<<<g, kRedThreads, 0, s>>>(n, a, b, S.part);
    finish_kernel<<<1, 1024, 0, s>>>(S.part, g, 1, out_dev, 0);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename TV, typename TW>
int dav_multidot(DavScratch &S, i64 n, int k, const TV *const *V, const TW *w, double *out_dev, cudaStream_t s)
{
    if (k < 1 || k > kMaxSub) { set_error("subspace size %d out of range", k); return BSIM_ERR_ARG; }
    int st = S.ensure();
    if (st) return st;
    const int g = grid_for(n);
    for (int j0 = 0; j0 < k; j0 += kDotChunk) {
        const int kc = std::min(kDotChunk, k - j0);
        multidot_kernel<TV, TW><<<g, kRedThreads, 0, s>>>(n, kc, pack(V + j0, kc), w, S.part);
        finish_kernel<<<1, 1024, 0, s>>>(S.part, g, kc, out_dev + j0, 0);
    }
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template int dav_ritz_residual<double>(DavScratch &, i64, int, const double *, double, const double *const *,
                                       const double *const *, double *, double *, cudaStream_t);
template int dav_ritz_residual<float>(DavScratch &, i64, int, const double *, double, const float *const *,
                                      const float *const *, double *, double *, cudaStream_t);
template int dav_combine<double, double>(i64, int, const double *, const double *const *, double *, cudaStream_t);
template int dav_combine<float, double>(i64, int, const double *, const float *const *, double *, cudaStream_t);
template int dav_combine<float, float>(i64, int, const double *, const float *const *, float *, cudaStream_t);
template int dav_combine<double, float>(i64, int, const double *, const double *const *, float *, cudaStream_t);
template int dav_mgs<double>(DavScratch &, i64, int, const double *const *, double *, double *, cudaStream_t);
template int dav_mgs<float>(DavScratch &, i64, int, const float *const *, double *, double *, cudaStream_t);
template int dav_multidot<double, double>(DavScratch &, i64, int, const double *const *, const double *, double *,
                                          cudaStream_t);
template int dav_multidot<float, float>(DavScratch &, i64, int, const float *const *, const float *, double *,
                                        cudaStream_t);
template int dav_multidot<float, double>(DavScratch &, i64, int, const float *const *, const double *, double *,
                                         cudaStream_t);

// ---- small symmetric eigensolver (cyclic Jacobi, FP64, k <= 64) --------------------
// ---- device-scalar helpers of the device-resident drivers ---------------------------
// Every scalar the host drivers used to read back (Ritz coefficients, energy,
// norms, the re-orthogonalisation test) stays on the device; the drivers read
// one residual norm per iteration.

// Jacobi eigensolver of the leading k x k block of the symmetric h (column-
// major, ld ldh) by one warp, A and the eigenvectors V in shared memory: the
// rotation formulas and stopping rule of jacobi_eigh, with the disjoint pairs of
// a round-robin round (k / 2 of them, k rounded up to even) rotated together
// (parallel ordering: each round's rotations are computed from the same A,
// then applied to the columns, to the rows and to V).  evals ascending,
// evecs[i + j k] = component i of eigenvector j.
__global__ void eigh_kernel(int k, const double *__restrict__ h, int ldh, double *__restrict__ evals,
                            double *__restrict__ evecs)
{
    extern __shared__ double A[];   // A[k * k], then V[k * k]
    __shared__ double rc[32], rs[32];
    __shared__ int rp[32], rq[32];
    double *work = A + k * k;
    const int lane = threadIdx.x;
    for (int i = lane; i < k * k; i += 32) {
        const int r = i % k, c = i / k;
        A[i] = h[r + (i64)c * ldh];
        work[i] = r == c ? 1.0 : 0.0;
    }
    __syncwarp();
    const int ke = (k + 1) & ~1, npair = ke / 2;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int i = lane; i < k * k; i += 32) {
            const double v = A[i] * A[i];
            tot += v;
            if (i % k != i / k) off += v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
        }
        if (off <= 1e-30 * fmax(tot, 1e-300)) break;
        for (int round = 0; round < ke - 1; ++round) {
            // pair i of the round: positions i and ke - 1 - i of the sequence
            // 0, 1 + (round + 0) % (ke - 1), 1 + (round + 1) % (ke - 1), ...
            for (int pi = lane; pi < npair; pi += 32) {
                auto pos = [&](int j) { return j == 0 ? 0 : 1 + (j - 1 + round) % (ke - 1); };
                int p = pos(pi), q = pos(ke - 1 - pi);
                if (p > q) { const int t = p; p = q; q = t; }
                double c = 1.0, sn = 0.0;
                if (q < k) {
                    const double apq = A[p + q * k];
                    if (fabs(apq) >= 1e-300) {
                        const double app = A[p + p * k], aqq = A[q + q * k];
                        const double tau = (aqq - app) / (2.0 * apq);
                        const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                        c = 1.0 / sqrt(1.0 + t * t);
                        sn = t * c;
                    }
                }
                rp[pi] = p; rq[pi] = q < k ? q : p; rc[pi] = c; rs[pi] = sn;
            }
            __syncwarp();
            for (int w = lane; w < npair * k; w += 32) {   // A = A J: columns p, q of every pair
                const int pi = w / k, r = w % k, p = rp[pi], q = rq[pi];
                if (p == q) continue;
                const double c = rc[pi], sn = rs[pi], arp = A[r + p * k], arq = A[r + q * k];
                A[r + p * k] = c * arp - sn * arq;
                A[r + q * k] = sn * arp + c * arq;
            }
            __syncwarp();
            for (int w = lane; w < npair * k; w += 32) {   // A = J^T A: rows p, q; V = V J
                const int pi = w / k, r = w % k, p = rp[pi], q = rq[pi];
                if (p == q) continue;
                const double c = rc[pi], sn = rs[pi], apr = A[p + r * k], aqr = A[q + r * k];
                A[p + r * k] = c * apr - sn * aqr;
                A[q + r * k] = sn * apr + c * aqr;
                const double vrp = work[r + p * k], vrq = work[r + q * k];
                work[r + p * k] = c * vrp - sn * vrq;
                work[r + q * k] = sn * vrp + c * vrq;
            }
            __syncwarp();
        }
    }
    // ascending order (ties by index): each lane places its eigenpairs
    for (int j = lane; j < k; j += 32) {
        const double d = A[j + j * k];
        int rank = 0;
        for (int i = 0; i < k; ++i) {
            const double di = A[i + i * k];
            rank += (di < d) || (di == d && i < j);
        }
        evals[rank] = d;
        for (int i = 0; i < k; ++i) evecs[i + rank * k] = work[i + j * k];
    }
}

// r = sum_j c_j AV_j - e sum_j c_j V_j, x = sum_j c_j V_j (if x), partial |r|^2;
// c = eigenvector 0 and e = evals[0], both read from the device
template <typename TV>
__global__ void ritz_dev_kernel(i64 n, int k, const double *__restrict__ cdev, const double *__restrict__ edev,
                                Ptrs<TV> V, Ptrs<TV> AV, double *__restrict__ r, double *__restrict__ x,
                                double *__restrict__ part)
{
    __shared__ double red[32], c[kMaxSub];
    for (int j = threadIdx.x; j < k; j += blockDim.x) c[j] = cdev[j];
    __syncthreads();
    const double e = *edev;
    double s = 0.0;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        double xv = 0.0, ax = 0.0;
        for (int j = 0; j < k; ++j) {
            xv += c[j] * (double)V.p[j][i];
            ax += c[j] * (double)AV.p[j][i];
        }
        const double rr = ax - e * xv;
        r[i] = rr;
        if (x) x[i] = xv;
        s += rr * rr;
    }
    cta_partial(s, red, part + blockIdx.x);
}

// x = sum_j c_j V_j with the coefficients on the device
template <typename TV, typename TX>
__global__ void combine_dev_kernel(i64 n, int k, const double *__restrict__ cdev, Ptrs<TV> V, TX *__restrict__ x)
{
    __shared__ double c[kMaxSub];
    for (int j = threadIdx.x; j < k; j += blockDim.x) c[j] = cdev[j];
    __syncthreads();
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < k; ++j) s += c[j] * (double)V.p[j][i];
        x[i] = (TX)s;
    }
}

// the preconditioner of precondition_kernel with e = evals[0] and the reference's
// shift max(1e-2 |r|, 1e-4) (jl/davidson.jl:116) from the residual norm on the device
template <typename TD>
__global__ void precondition_dev_kernel(i64 n, double *__restrict__ r, const TD *__restrict__ d,
                                        const double *__restrict__ edev, const double *__restrict__ rnorm,
                                        double *__restrict__ part)
{
    __shared__ double red[32];
    const double e = *edev, as = fmax(*rnorm * 1e-2, 1e-4);
    double s = 0.0;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        double diff = (double)d[i] - e;
        if (fabs(diff) < as) diff = (diff >= 0) ? as : -as;
        const double v = r[i] / diff;
        r[i] = v;
        s += v * v;
    }
    cta_partial(s, red, part + blockIdx.x);
}

// Gate of the second Gram-Schmidt pass (jl/davidson.jl:124-133): run when the
// norm after the first pass (g[1]) fell below 0.717 of the norm before it (g[0]).
__device__ __forceinline__ bool cgs_skip(const double *g) { return g && !(g[1] < 0.717 * g[0]); }

// classical Gram-Schmidt projections p_j = <V_j, v>, j < k (<= kDotChunk per launch)
template <typename TV>
__global__ void cgs_proj_kernel(i64 n, int k, Ptrs<TV> V, const double *__restrict__ v, double *__restrict__ part,
                                const double *__restrict__ gate)
{
    if (cgs_skip(gate)) return;
    __shared__ double red[32];
    double s[kDotChunk];
#pragma unroll
    for (int j = 0; j < kDotChunk; ++j) s[j] = 0.0;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        const double x = v[i];
#pragma unroll
        for (int j = 0; j < kDotChunk; ++j)
            if (j < k) s[j] += (double)V.p[j][i] * x;
    }
#pragma unroll
    for (int j = 0; j < kDotChunk; ++j)
        if (j < k) cta_partial(s[j], red, part + (i64)blockIdx.x * k + j);
}

// v -= sum_j p_j V_j, partial |v|^2
template <typename TV>
__global__ void cgs_update_kernel(i64 n, int k, Ptrs<TV> V, const double *__restrict__ p, double *__restrict__ v,
                                  double *__restrict__ part, const double *__restrict__ gate)
{
    if (cgs_skip(gate)) return;
    __shared__ double red[32], c[kMaxSub];
    for (int j = threadIdx.x; j < k; j += blockDim.x) c[j] = p[j];
    __syncthreads();
    double s = 0.0;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        double x = v[i];
        for (int j = 0; j < k; ++j) x -= c[j] * (double)V.p[j][i];
        v[i] = x;
        s += x * x;
    }
    cta_partial(s, red, part + blockIdx.x);
}

__global__ void finish_gated_kernel(const double *__restrict__ part, int nblk, int nout, double *__restrict__ out,
                                    int sqrt_out, const double *__restrict__ gate)
{
    if (cgs_skip(gate)) return;
    __shared__ double red[32];
    for (int j = 0; j < nout; ++j) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += part[(i64)b * nout + j];
        s = warp_sum(s);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
            out[j] = sqrt_out ? sqrt(t) : t;
        }
        __syncthreads();
    }
}

// out = v / |v| (|v| on the device, in the precision of out); when |v| < 1e-12
// (the new direction lies in the subspace) the breakdown flag is set and out = v
template <typename TO>
__global__ void normalize_into_kernel(i64 n, const double *__restrict__ v, const double *__restrict__ nrm,
                                      TO *__restrict__ out, double *__restrict__ breakdown)
{
    const double m = *nrm;
    const bool bad = !(m >= 1e-12);
    if (bad && blockIdx.x == 0 && threadIdx.x == 0) *breakdown = 1.0;
    const double inv = bad ? 1.0 : 1.0 / m;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        out[i] = (TO)(v[i] * inv);
}

// h[dim-1 + i ld] = h[i + (dim-1) ld]: the new column mirrored into its row
__global__ void mirror_col_kernel(int dim, double *__restrict__ h, int ld)
{
    const int i = threadIdx.x;
    if (i < dim) h[(dim - 1) + (i64)i * ld] = h[i + (i64)(dim - 1) * ld];
}

// h <- (h + h^T) / 2 on the leading dim x dim block (rebuild_heff's symmetrisation)
__global__ void sym_avg_kernel(int dim, double *__restrict__ h, int ld)
{
    for (int t = threadIdx.x; t < dim * dim; t += blockDim.x) {
        const int i = t % dim, j = t / dim;
        if (i < j) {
            const double a = 0.5 * (h[i + (i64)j * ld] + h[j + (i64)i * ld]);
            h[i + (i64)j * ld] = a;
            h[j + (i64)i * ld] = a;
        }
    }
}

// x = a[0] * x + t with a on the device
__global__ void axpby_dev_kernel(i64 n, const double *__restrict__ a, double *__restrict__ x,
                                 const double *__restrict__ t)
{
    const double s = *a;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        x[i] = s * x[i] + t[i];
}

int dav_eigh_dev(int k, const double *h, int ldh, double *evals, double *evecs, cudaStream_t s)
{
    if (k < 1 || k > kMaxSub) { set_error("subspace size %d out of range", k); return BSIM_ERR_ARG; }
    const int smem = (int)(sizeof(double) * 2 * k * k);   // <= 64 KB (k <= 64)
    if (smem > 48 * 1024)
        BSIM_CUDA(cudaFuncSetAttribute(eigh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    eigh_kernel<<<1, 32, smem, s>>>(k, h, ldh, evals, evecs);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename TV>
int dav_ritz_residual_dev(DavScratch &S, i64 n, int k, const double *coeffs_dev, const double *e_dev,
                          const TV *const *V, const TV *const *AV, double *r, double *x, double *norm_dev,
                          cudaStream_t s)
{
    if (k < 1 || k > kMaxSub) { set_error("subspace size %d out of range", k); return BSIM_ERR_ARG; }
    const int g = grid_for(n);
    ritz_dev_kernel<TV><<<g, kRedThreads, 0, s>>>(n, k, coeffs_dev, e_dev, pack(V, k), pack(AV, k), r, x, S.part);
    finish_kernel<<<1, 1024, 0, s>>>(S.part, g, 1, norm_dev, 1);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename TV, typename TX>
int dav_combine_dev(i64 n, int k, const double *coeffs_dev, const TV *const *V, TX *x, cudaStream_t s)
{
    if (k < 1 || k > kMaxSub) { set_error("subspace size %d out of range", k); return BSIM_ERR_ARG; }
    combine_dev_kernel<TV, TX><<<grid_for(n), kRedThreads, 0, s>>>(n, k, coeffs_dev, pack(V, k), x);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename TD>
int dav_precondition_dev(DavScratch &S, i64 n, double *r, const TD *d, const double *e_dev,
                         const double *rnorm_dev, double *norm_dev, cudaStream_t s)
{
    const int g = grid_for(n);
    precondition_dev_kernel<TD><<<g, kRedThreads, 0, s>>>(n, r, d, e_dev, rnorm_dev, S.part);
    finish_kernel<<<1, 1024, 0, s>>>(S.part, g, 1, norm_dev, 1);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

// Orthogonalise v against V[0..k) by classical Gram-Schmidt; nrm[0] holds |v|
// before the call, nrm[1] receives |v| after it.  A second pass runs (decided on
// the device) when nrm[1] < 0.717 nrm[0], the reference's test for repeating
// the orthogonalisation (jl/davidson.jl:124-133).  proj: kMaxSub device doubles.
template <typename TV>
int dav_cgs2_dev(DavScratch &S, i64 n, int k, const TV *const *V, double *v, double *nrm, double *proj,
                 cudaStream_t s)
{
    if (k < 0 || k > kMaxSub) { set_error("subspace size %d out of range", k); return BSIM_ERR_ARG; }
    const int g = grid_for(n);
    for (int pass = 0; pass < 2; ++pass) {
        const double *gate = pass ? nrm : nullptr;
        for (int j0 = 0; j0 < k; j0 += kDotChunk) {
            const int kc = std::min(kDotChunk, k - j0);
            cgs_proj_kernel<TV><<<g, kRedThreads, 0, s>>>(n, kc, pack(V + j0, kc), v, S.part, gate);
            finish_gated_kernel<<<1, 1024, 0, s>>>(S.part, g, kc, proj + j0, 0, gate);
        }
        cgs_update_kernel<TV><<<g, kRedThreads, 0, s>>>(n, k, pack(V, k), proj, v, S.part, gate);
        finish_gated_kernel<<<1, 1024, 0, s>>>(S.part, g, 1, nrm + 1, 1, gate);
    }
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template <typename TO>
int dav_normalize_into(i64 n, const double *v, const double *nrm_dev, TO *out, double *breakdown_dev,
                       cudaStream_t s)
{
    normalize_into_kernel<TO><<<grid_for(n), kRedThreads, 0, s>>>(n, v, nrm_dev, out, breakdown_dev);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

int dav_mirror_col(int dim, double *h, int ld, cudaStream_t s)
{
    mirror_col_kernel<<<1, kMaxSub, 0, s>>>(dim, h, ld);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

int dav_sym_avg(int dim, double *h, int ld, cudaStream_t s)
{
    sym_avg_kernel<<<1, 256, 0, s>>>(dim, h, ld);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

int dav_axpby_dev(i64 n, const double *a_dev, double *x, const double *t, cudaStream_t s)
{
    axpby_dev_kernel<<<grid_for(n), kRedThreads, 0, s>>>(n, a_dev, x, t);
    BSIM_CUDA(cudaGetLastError());
    return BSIM_OK;
}

template int dav_ritz_residual_dev<double>(DavScratch &, i64, int, const double *, const double *,
                                           const double *const *, const double *const *, double *, double *,
                                           double *, cudaStream_t);
template int dav_ritz_residual_dev<float>(DavScratch &, i64, int, const double *, const double *,
                                          const float *const *, const float *const *, double *, double *,
                                          double *, cudaStream_t);
template int dav_combine_dev<double, double>(i64, int, const double *, const double *const *, double *,
                                             cudaStream_t);
template int dav_combine_dev<float, double>(i64, int, const double *, const float *const *, double *,
                                            cudaStream_t);
template int dav_combine_dev<float, float>(i64, int, const double *, const float *const *, float *, cudaStream_t);
template int dav_precondition_dev<double>(DavScratch &, i64, double *, const double *, const double *,
                                          const double *, double *, cudaStream_t);
template int dav_precondition_dev<float>(DavScratch &, i64, double *, const float *, const double *,
                                         const double *, double *, cudaStream_t);
template int dav_cgs2_dev<double>(DavScratch &, i64, int, const double *const *, double *, double *, double *,
                                  cudaStream_t);
template int dav_cgs2_dev<float>(DavScratch &, i64, int, const float *const *, double *, double *, double *,
                                 cudaStream_t);
template int dav_normalize_into<double>(i64, const double *, const double *, double *, double *, cudaStream_t);
template int dav_normalize_into<float>(i64, const double *, const double *, float *, double *, cudaStream_t);

void jacobi_eigh(int k, const double *A_in, int lda, double *evals, double *evecs /* k x k col-major */)
{
    std::vector<double> A((size_t)k * k);
    for (int j = 0; j < k; ++j)
        for (int i = 0; i < k; ++i) A[i + (size_t)j * k] = A_in[i + (size_t)j * lda];
    for (int i = 0; i < k * k; ++i) evecs[i] = 0.0;
    for (int i = 0; i < k; ++i) evecs[i + i * k] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int j = 0; j < k; ++j)
            for (int i = 0; i < k; ++i) {
                const double v = A[i + (size_t)j * k] * A[i + (size_t)j * k];
                tot += v;
                if (i != j) off += v;
            }
        if (off <= 1e-30 * std::max(tot, 1e-300)) break;
        for (int p = 0; p < k - 1; ++p)
            for (int q = p + 1; q < k; ++q) {
                const double apq = A[p + (size_t)q * k];
                if (fabs(apq) < 1e-300) continue;
                const double app = A[p + (size_t)p * k], aqq = A[q + (size_t)q * k];
                const double tau = (aqq - app) / (2.0 * apq);
                const double t = (tau >= 0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
                for (int r = 0; r < k; ++r) {   // A = J^T A J
                    const double arp = A[r + (size_t)p * k], arq = A[r + (size_t)q * k];
                    A[r + (size_t)p * k] = c * arp - s * arq;
                    A[r + (size_t)q * k] = s * arp + c * arq;
                }
                for (int r = 0; r < k; ++r) {
                    const double apr = A[p + (size_t)r * k], aqr = A[q + (size_t)r * k];
                    A[p + (size_t)r * k] = c * apr - s * aqr;
                    A[q + (size_t)r * k] = s * apr + c * aqr;
                }
                for (int r = 0; r < k; ++r) {
                    const double vrp = evecs[r + p * k], vrq = evecs[r + q * k];
                    evecs[r + p * k] = c * vrp - s * vrq;
                    evecs[r + q * k] = s * vrp + c * vrq;
                }
            }
    }
    // sort ascending
    std::vector<int> idx(k);
    for (int i = 0; i < k; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return A[a + (size_t)a * k] < A[b + (size_t)b * k]; });
    std::vector<double> V(evecs, evecs + (size_t)k * k);
    for (int j = 0; j < k; ++j) {
        evals[j] = A[idx[j] + (size_t)idx[j] * k];
        for (int i = 0; i < k; ++i) evecs[i + (size_t)j * k] = V[i + (size_t)idx[j] * k];
    }
}

}  // namespace bsim
