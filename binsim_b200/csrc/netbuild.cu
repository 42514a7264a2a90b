// Native OTF network construction (host): the grouping and SVD compression of
// jl/network.jl:158-246 (compress_by_svd) for a list of aabb Pauli terms
// (ax, az, bx, bz, c), in C++ instead of the host scripting language.
//
// Terms with equal (ax, bx) form a group (groups in order of first appearance);
// the group's coefficient matrix M[za, zb] (distinct za and zb sorted
// ascending) is factorised by a one-sided Jacobi SVD; singular values above
// tol are kept (rank), wa = U sqrt(S), wb = V sqrt(S), entries below 1e-12 are
// zeroed, and the weights are stored column-major [num_z x rank] as the
// reference's build_network_otf expects (otf.hpp:84-85).  Groups are
// independent and compressed on all host threads, or (bsim_netbuild_compress_device)
// with the Jacobi sweeps of every group on the GPU, one CTA per group.  The
// result feeds bsim_network_create_u32 / _u64.
#include "../../include/binsim_cuotf.h"
#include "common.cuh"

#include <algorithm>
#include <cmath>
#include <thread>
#include <unordered_map>
#include <vector>

namespace bsim {

namespace {

struct BuiltGroup {
    u64 ax, bx;
    std::vector<u64> za, zb;
    int rank = 0;
    std::vector<double> wa, wb;   // column-major [nza x rank], [nzb x rank]
};

struct NetBuild {
    unsigned magic = 0xB5B1B11Du;
    std::vector<BuiltGroup> g;
};

// One-sided Jacobi SVD of A (m x n, column-major, m >= n): on return A's
// columns are U * S, V (n x n, column-major) the right singular vectors, in
// the order of the columns (unsorted).
void jacobi_svd(int m, int n, std::vector<double> &A, std::vector<double> &V)
{
    V.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < n - 1; ++p)
            for (int q = p + 1; q < n; ++q) {
                double *ap = &A[(size_t)p * m], *aq = &A[(size_t)q * m];
                double alpha = 0.0, beta = 0.0, gamma = 0.0;
                for (int i = 0; i < m; ++i) {
                    alpha += ap[i] * ap[i];
                    beta += aq[i] * aq[i];
                    gamma += ap[i] * aq[i];
                }
                if (std::fabs(gamma) <= 1e-300) continue;
                const double scale = std::sqrt(alpha * beta);
                if (scale <= 0.0) continue;
                off = std::max(off, std::fabs(gamma) / scale);
                if (std::fabs(gamma) <= 1e-15 * scale) continue;
                const double zeta = (beta - alpha) / (2.0 * gamma);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
                for (int i = 0; i < m; ++i) {
                    const double x = ap[i], y = aq[i];
                    ap[i] = c * x - s * y;
                    aq[i] = s * x + c * y;
                }
                double *vp = &V[(size_t)p * n], *vq = &V[(size_t)q * n];
                for (int i = 0; i < n; ++i) {
                    const double x = vp[i], y = vq[i];
                    vp[i] = c * x - s * y;
                    vq[i] = s * x + c * y;
                }
            }
        if (off <= 1e-15) break;
    }
}

// The factored matrix: A = M (m x n, column-major) when m >= n, else A = M^T, so
// that A is at least as tall as it is wide (one-sided Jacobi rotates columns).
void factored(int m, int n, const std::vector<double> &M, bool tr, double *A)
{
    const int mm = tr ? n : m;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            const double v = M[(size_t)j * m + i];
            if (tr) A[(size_t)i * mm + j] = v;   // A = M^T
            else A[(size_t)j * mm + i] = v;
        }
}

// After the Jacobi sweeps (A's columns = U S, V the right vectors): the rank
// above tol and the weights wa, wb of the original orientation.
void finish_factors(int mm, int nn, bool tr, const double *A, const double *V, double tol, BuiltGroup &G);

// M (m x n, column-major) -> rank, wa (m x rank), wb (n x rank), column-major
void compress(int m, int n, const std::vector<double> &M, double tol, BuiltGroup &G)
{
    const bool tr = m < n;   // factor the transpose when it is the taller one
    const int mm = tr ? n : m, nn = tr ? m : n;
    std::vector<double> A((size_t)mm * nn), V;
    factored(m, n, M, tr, A.data());
    jacobi_svd(mm, nn, A, V);
    finish_factors(mm, nn, tr, A.data(), V.data(), tol, G);
}

void finish_factors(int mm, int nn, bool tr, const double *A, const double *V, double tol, BuiltGroup &G)
{
    std::vector<double> sv(nn);
    for (int k = 0; k < nn; ++k) {
        double s = 0.0;
        for (int i = 0; i < mm; ++i) s += A[(size_t)k * mm + i] * A[(size_t)k * mm + i];
        sv[k] = std::sqrt(s);
    }
    std::vector<int> order(nn);
    for (int k = 0; k < nn; ++k) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return sv[a] > sv[b]; });
    std::vector<int> keep;
    for (int k : order)
        if (sv[k] > tol) keep.push_back(k);
    const int r = (int)keep.size();
    // A's column k is sv_k u_k (left vectors of the factored matrix), V's column k is v_k
    std::vector<double> L((size_t)mm * r), R((size_t)nn * r);
    for (int t = 0; t < r; ++t) {
        const int k = keep[t];
        const double sq = std::sqrt(sv[k]);
        for (int i = 0; i < mm; ++i) L[(size_t)t * mm + i] = A[(size_t)k * mm + i] / sv[k] * sq;
        for (int i = 0; i < nn; ++i) R[(size_t)t * nn + i] = V[(size_t)k * nn + i] * sq;
    }
    // M = L R^T when not transposed; M^T = L R^T (so M = R L^T) when transposed
    G.rank = r;
    G.wa = tr ? R : L;
    G.wb = tr ? L : R;
    for (double &x : G.wa)
        if (std::fabs(x) < 1e-12) x = 0.0;
    for (double &x : G.wb)
        if (std::fabs(x) < 1e-12) x = 0.0;
}

// ---- device SVD: one CTA per group -----------------------------------------------
struct SvdJob {
    i64 a_off, v_off;   // A (m x n, column-major, m >= n) and V (n x n) in the packed buffers
    int m, n;
};

// The one-sided Jacobi SVD of jacobi_svd on the device: each sweep visits every
// column pair once in n' - 1 rounds of the round-robin (circle) schedule, n' = n
// rounded up to even; the pairs of a round are disjoint and go to the warps of
// the CTA, each warp reducing the pair's dot products over the rows with its
// lanes.  Same rotation, skip and convergence rules as the host code.
__global__ void __launch_bounds__(512) jacobi_svd_kernel(const SvdJob *__restrict__ jobs, double *__restrict__ A,
                                                         double *__restrict__ V, int max_sweeps)
{
    const SvdJob J = jobs[blockIdx.x];
    const int m = J.m, n = J.n;
    double *a = A + J.a_off, *v = V + J.v_off;
    for (i64 i = threadIdx.x; i < (i64)n * n; i += blockDim.x) v[i] = (i % (n + 1) == 0) ? 1.0 : 0.0;
    if (n < 2) return;
    __syncthreads();
    const int np = n + (n & 1);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __shared__ unsigned long long offbits;   // max |gamma| / scale of the sweep (non-negative: bits order like values)
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
        if (threadIdx.x == 0) offbits = 0ull;
        __syncthreads();
        double off = 0.0;
        for (int r = 0; r < np - 1; ++r) {
            for (int k = w; k < np / 2; k += nw) {
                int p = k == 0 ? np - 1 : (r + k) % (np - 1);
                int q = k == 0 ? r : (r - k + np - 1) % (np - 1);
                if (p > q) { const int t = p; p = q; q = t; }
                if (q >= n) continue;   // paired with the bye
                double *ap = a + (i64)p * m, *aq = a + (i64)q * m;
                double al = 0.0, be = 0.0, ga = 0.0;
                for (int i = lane; i < m; i += 32) {
                    const double x = ap[i], y = aq[i];
                    al += x * x;
                    be += y * y;
                    ga += x * y;
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    al += __shfl_xor_sync(0xffffffffu, al, o);
                    be += __shfl_xor_sync(0xffffffffu, be, o);
                    ga += __shfl_xor_sync(0xffffffffu, ga, o);
                }
                if (fabs(ga) <= 1e-300) continue;
                const double scale = sqrt(al * be);
                if (scale <= 0.0) continue;
                off = fmax(off, fabs(ga) / scale);
                if (fabs(ga) <= 1e-15 * scale) continue;
                const double zeta = (be - al) / (2.0 * ga);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
                for (int i = lane; i < m; i += 32) {
                    const double x = ap[i], y = aq[i];
                    ap[i] = c * x - s * y;
                    aq[i] = s * x + c * y;
                }
                double *vp = v + (i64)p * n, *vq = v + (i64)q * n;
                for (int i = lane; i < n; i += 32) {
                    const double x = vp[i], y = vq[i];
                    vp[i] = c * x - s * y;
                    vq[i] = s * x + c * y;
                }
            }
            __syncthreads();   // the next round's pairs reuse these columns
        }
        if (lane == 0) atomicMax(&offbits, (unsigned long long)__double_as_longlong(off));
        __syncthreads();
        const double o = __longlong_as_double((long long)offbits);
        __syncthreads();   // every thread has read offbits before it is reset
        if (o <= 1e-15) break;
    }
}

// Jacobi SVDs of the packed factored matrices on the current device, small
// jobs (n <= 8) with 64 threads per CTA and the rest with 512.
int device_svds(const std::vector<SvdJob> &jobs, std::vector<double> &A, std::vector<double> &V, cudaStream_t s)
{
    if (jobs.empty()) return BSIM_OK;
    std::vector<SvdJob> small, large;
    for (const SvdJob &j : jobs) (j.n <= 8 ? small : large).push_back(j);
    SvdJob *dj = nullptr;
    double *dA = nullptr, *dV = nullptr;
    int st = BSIM_OK;
    cudaError_t e = dmalloc(&dj, sizeof(SvdJob) * jobs.size());
    if (e == cudaSuccess) e = dmalloc(&dA, sizeof(double) * std::max<size_t>(A.size(), 1));
    if (e == cudaSuccess) e = dmalloc(&dV, sizeof(double) * std::max<size_t>(V.size(), 1));
    if (e == cudaSuccess) e = cudaMemcpyAsync(dA, A.data(), sizeof(double) * A.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !small.empty())
        e = cudaMemcpyAsync(dj, small.data(), sizeof(SvdJob) * small.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !large.empty())
        e = cudaMemcpyAsync(dj + small.size(), large.data(), sizeof(SvdJob) * large.size(), cudaMemcpyHostToDevice, s);
    // grid x is limited to 2^31 - 1 CTAs; one launch per kind of job
    if (e == cudaSuccess && !small.empty()) {
        jacobi_svd_kernel<<<(unsigned)small.size(), 64, 0, s>>>(dj, dA, dV, 60);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && !large.empty()) {
        jacobi_svd_kernel<<<(unsigned)large.size(), 512, 0, s>>>(dj + small.size(), dA, dV, 60);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(A.data(), dA, sizeof(double) * A.size(), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(V.data(), dV, sizeof(double) * V.size(), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = cuda_status(e, "device network SVD");
    cudaFree(dj);
    cudaFree(dA);
    cudaFree(dV);
    return st;
}

NetBuild *nb_of(void *h)
{
    auto *p = static_cast<NetBuild *>(h);
    return (p && p->magic == 0xB5B1B11Du) ? p : nullptr;
}

}  // namespace
}  // namespace bsim

static int netbuild(int64_t nterms, const uint64_t *ax, const uint64_t *az, const uint64_t *bx, const uint64_t *bz,
                    const double *coef, double tol, int64_t nruns, const int64_t *run_sizes, void **out,
                    bool device = false, cudaStream_t stream = nullptr)
{
    using bsim::u64;
    if (!out) { bsim::set_error("null out"); return BSIM_ERR_NULL; }
    *out = nullptr;
    if (nterms < 0) { bsim::set_error("nterms = %lld", (long long)nterms); return BSIM_ERR_ARG; }
    if (nterms > 0 && (!ax || !az || !bx || !bz || !coef)) { bsim::set_error("null term array"); return BSIM_ERR_NULL; }
    std::vector<std::vector<int64_t>> members;
    std::vector<std::pair<u64, u64>> keys;
    if (run_sizes) {
        // one group per run of consecutive terms (one X group per generator, network.jl:248-301)
        int64_t t0 = 0;
        for (int64_t r = 0; r < nruns; ++r) {
            const int64_t n = run_sizes[r];
            if (n <= 0 || t0 + n > nterms) { bsim::set_error("run %lld of size %lld exceeds the terms", (long long)r, (long long)n); return BSIM_ERR_ARG; }
            members.emplace_back();
            keys.emplace_back((u64)ax[t0], (u64)bx[t0]);
            for (int64_t t = t0; t < t0 + n; ++t) {
                if ((u64)ax[t] != keys.back().first || (u64)bx[t] != keys.back().second) {
                    bsim::set_error("run %lld mixes X masks", (long long)r);
                    return BSIM_ERR_ARG;
                }
                members.back().push_back(t);
            }
            t0 += n;
        }
        if (t0 != nterms) { bsim::set_error("runs cover %lld of %lld terms", (long long)t0, (long long)nterms); return BSIM_ERR_ARG; }
    } else {
        // groups in order of first appearance of (ax, bx)
        struct KeyHash {
            size_t operator()(const std::pair<u64, u64> &k) const { return std::hash<u64>()(k.first * 0x9E3779B97F4A7C15ull ^ k.second); }
        };
        std::unordered_map<std::pair<u64, u64>, int, KeyHash> gid;
        for (int64_t t = 0; t < nterms; ++t) {
            const auto key = std::make_pair((u64)ax[t], (u64)bx[t]);
            auto it = gid.find(key);
            int g;
            if (it == gid.end()) {
                g = (int)members.size();
                gid.emplace(key, g);
                members.emplace_back();
                keys.push_back(key);
            } else g = it->second;
            members[g].push_back(t);
        }
    }
    auto *B = new bsim::NetBuild();
    B->g.resize(members.size());
    for (size_t g = 0; g < members.size(); ++g) { B->g[g].ax = keys[g].first; B->g[g].bx = keys[g].second; }
    const int ng = (int)members.size();
    const int nth = std::max(1, std::min(32, (int)std::thread::hardware_concurrency()));
    auto run = [&](auto &&fn) {
        std::vector<std::thread> th;
        for (int w = 1; w < nth; ++w) th.emplace_back(fn, w);
        fn(0);
        for (auto &x : th) x.join();
    };
    // the group's Z lists and coefficient matrix M[za, zb] (column-major)
    auto matrix = [&](int g, std::vector<double> &M) {
        bsim::BuiltGroup &G = B->g[g];
        for (int64_t t : members[g]) { G.za.push_back((u64)az[t]); G.zb.push_back((u64)bz[t]); }
        std::sort(G.za.begin(), G.za.end());
        G.za.erase(std::unique(G.za.begin(), G.za.end()), G.za.end());
        std::sort(G.zb.begin(), G.zb.end());
        G.zb.erase(std::unique(G.zb.begin(), G.zb.end()), G.zb.end());
        const int m = (int)G.za.size(), n = (int)G.zb.size();
        M.assign((size_t)m * n, 0.0);
        for (int64_t t : members[g]) {
            const int i = (int)(std::lower_bound(G.za.begin(), G.za.end(), (u64)az[t]) - G.za.begin());
            const int j = (int)(std::lower_bound(G.zb.begin(), G.zb.end(), (u64)bz[t]) - G.zb.begin());
            M[(size_t)j * m + i] += coef[t];
        }
    };
    if (!device) {
        run([&](int w) {
            std::vector<double> M;
            for (int g = w; g < ng; g += nth) {
                matrix(g, M);
                bsim::compress((int)B->g[g].za.size(), (int)B->g[g].zb.size(), M, tol, B->g[g]);
            }
        });
        *out = B;
        return BSIM_OK;
    }
    // device SVDs: the host groups the terms and packs every group's factored
    // matrix; the Jacobi sweeps run on the GPU, one CTA per group; the host then
    // keeps the singular values above tol and scales the factors
    std::vector<bsim::SvdJob> jobs(ng);
    std::vector<std::vector<double>> Ms(ng);
    run([&](int w) {
        for (int g = w; g < ng; g += nth) matrix(g, Ms[g]);
    });
    int64_t na_tot = 0, nv_tot = 0;
    for (int g = 0; g < ng; ++g) {
        const int m = (int)B->g[g].za.size(), n = (int)B->g[g].zb.size();
        const int mm = std::max(m, n), nn = std::min(m, n);
        jobs[g] = bsim::SvdJob{na_tot, nv_tot, mm, nn};
        na_tot += (int64_t)mm * nn;
        nv_tot += (int64_t)nn * nn;
    }
    std::vector<double> A((size_t)na_tot), V((size_t)nv_tot);
    run([&](int w) {
        for (int g = w; g < ng; g += nth) {
            const int m = (int)B->g[g].za.size(), n = (int)B->g[g].zb.size();
            bsim::factored(m, n, Ms[g], m < n, A.data() + jobs[g].a_off);
            std::vector<double>().swap(Ms[g]);
        }
    });
    int st = bsim::device_svds(jobs, A, V, stream);
    if (st != BSIM_OK) { delete B; return st; }
    run([&](int w) {
        for (int g = w; g < ng; g += nth) {
            const int m = (int)B->g[g].za.size(), n = (int)B->g[g].zb.size();
            bsim::finish_factors(jobs[g].m, jobs[g].n, m < n, A.data() + jobs[g].a_off, V.data() + jobs[g].v_off,
                                 tol, B->g[g]);
        }
    });
    *out = B;
    return BSIM_OK;
}

extern "C" {

int bsim_netbuild_compress(int64_t nterms, const uint64_t *ax, const uint64_t *az, const uint64_t *bx,
                           const uint64_t *bz, const double *coef, double tol, void **out)
{
    return netbuild(nterms, ax, az, bx, bz, coef, tol, 0, nullptr, out);
}

int bsim_netbuild_compress_runs(int64_t nterms, const uint64_t *ax, const uint64_t *az, const uint64_t *bx,
                                const uint64_t *bz, const double *coef, double tol, int64_t nruns,
                                const int64_t *run_sizes, void **out)
{
    if (nruns > 0 && !run_sizes) { bsim::set_error("null run_sizes"); return BSIM_ERR_NULL; }
    if (nruns < 0) { bsim::set_error("nruns = %lld", (long long)nruns); return BSIM_ERR_ARG; }
    static const int64_t none = 0;
    return netbuild(nterms, ax, az, bx, bz, coef, tol, nruns, nruns > 0 ? run_sizes : &none, out);
}

int bsim_netbuild_compress_device(int64_t nterms, const uint64_t *ax, const uint64_t *az, const uint64_t *bx,
                                  const uint64_t *bz, const double *coef, double tol, int64_t nruns,
                                  const int64_t *run_sizes, bsim_stream_t stream, void **out)
{
    if (nruns > 0 && !run_sizes) { bsim::set_error("null run_sizes"); return BSIM_ERR_NULL; }
    if (nruns < 0) { bsim::set_error("nruns = %lld", (long long)nruns); return BSIM_ERR_ARG; }
    return netbuild(nterms, ax, az, bx, bz, coef, tol, nruns, nruns > 0 ? run_sizes : nullptr, out, true,
                    static_cast<cudaStream_t>(stream));
}

int bsim_netbuild_sizes(void *h, int64_t *ngs, int64_t *nza_total, int64_t *nzb_total, int64_t *nwa_total,
                        int64_t *nwb_total)
{
    bsim::NetBuild *B = bsim::nb_of(h);
    if (!B) { bsim::set_error("invalid network builder handle"); return BSIM_ERR_ARG; }
    int64_t a = 0, b = 0, wa = 0, wb = 0;
    for (auto &G : B->g) {
        a += (int64_t)G.za.size();
        b += (int64_t)G.zb.size();
        wa += (int64_t)G.wa.size();
        wb += (int64_t)G.wb.size();
    }
    if (ngs) *ngs = (int64_t)B->g.size();
    if (nza_total) *nza_total = a;
    if (nzb_total) *nzb_total = b;
    if (nwa_total) *nwa_total = wa;
    if (nwb_total) *nwb_total = wb;
    return BSIM_OK;
}

int bsim_netbuild_export(void *h, uint64_t *axs, uint64_t *bxs, int64_t *ranks, int64_t *num_zas, int64_t *num_zbs,
                         uint64_t *flat_zas, uint64_t *flat_zbs, double *flat_wa, double *flat_wb)
{
    bsim::NetBuild *B = bsim::nb_of(h);
    if (!B) { bsim::set_error("invalid network builder handle"); return BSIM_ERR_ARG; }
    if (!B->g.empty() && (!axs || !bxs || !ranks || !num_zas || !num_zbs)) {
        bsim::set_error("null output array");
        return BSIM_ERR_NULL;
    }
    int64_t oa = 0, ob = 0, owa = 0, owb = 0;
    for (size_t i = 0; i < B->g.size(); ++i) {
        const auto &G = B->g[i];
        axs[i] = G.ax;
        bxs[i] = G.bx;
        ranks[i] = G.rank;
        num_zas[i] = (int64_t)G.za.size();
        num_zbs[i] = (int64_t)G.zb.size();
        if (flat_zas) std::copy(G.za.begin(), G.za.end(), flat_zas + oa);
        if (flat_zbs) std::copy(G.zb.begin(), G.zb.end(), flat_zbs + ob);
        if (flat_wa) std::copy(G.wa.begin(), G.wa.end(), flat_wa + owa);
        if (flat_wb) std::copy(G.wb.begin(), G.wb.end(), flat_wb + owb);
        oa += (int64_t)G.za.size();
        ob += (int64_t)G.zb.size();
        owa += (int64_t)G.wa.size();
        owb += (int64_t)G.wb.size();
    }
    return BSIM_OK;
}

int bsim_netbuild_destroy(void *h)
{
    bsim::NetBuild *B = bsim::nb_of(h);
    if (!B) { bsim::set_error("invalid network builder handle"); return BSIM_ERR_ARG; }
    B->magic = 0;
    delete B;
    return BSIM_OK;
}

}  // extern "C"
