/*
 * binsim_cuotf.h -- C-ABI of libcuotf, the B200 (sm_100a) implementation of
 * BinSim's on-the-fly (OTF) operator path.
 *
 * Part 1 keeps the reference GPU library's entry points with identical names,
 * argument lists and semantics, so Julia's ccall sites bind unchanged.  Part 2
 * adds status-returning, stream-taking entry points.  Part 3 puts libdiag's
 * Davidson vector helpers on device pointers.
 *
 * Conventions (all parts):
 *   - vectors are device pointers to FP64 arrays of length bsim_basis_dim(),
 *     ordered block offset + alpha index * n_beta + beta index
 *     (reference src/include/basis/basis.hpp:327);
 *   - group / generator indices are 0-based original network indices (the
 *     Julia layer passes idx-1, reference jl/cuda/cunetwork.jl:124);
 *   - strings are UInt32 bit strings (orbital p = bit p), norb <= 26.
 *
 * Thread safety: a basis handle owns reusable device scratch, so calls that
 * share one basis handle must be issued from one host thread / one stream at
 * a time.
 */
#ifndef BINSIM_CUOTF_H
#define BINSIM_CUOTF_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *bsim_stream_t; /* a cudaStream_t; NULL = legacy default stream */

/* ========================================================================
 * Part 1: reference-compatible entry points (src/extern/cuotf.cu:7-162).
 * They run on the legacy default stream.  hvec/expm/batchgrad/diag return
 * before the GPU finishes; grad/backgrad return the scalar, so they wait.
 * On failure they print to stderr and leave bsim_last_error() set; they never
 * exit the process (the reference calls exit(1), common.cuh:42-49).
 * ====================================================================== */

/* cuotf.cu:9-12 */
void sync_device_cuda(void);
/* cuotf.cu:26-31: host_basis is a BasisManager<uint32>* returned by libbasis
 * create_basis_manager (basis/declare.hpp:24-33); its tables are copied. */
void *build_basisdev_f64(void *host_basis);
/* cuotf.cu:14-24 */
void destroy_basisdev_f64(void *basis);
/* cuotf.cu:43-48: host_net is a Network_OTF<uint32,double>* returned by
 * libotf_native build_network_otf_f64 (op/declare.hpp:25-35). */
void *build_networkdev_f64(void *host_net);
/* cuotf.cu:33-41 */
void destroy_networkdev_f64(void *net);
/* cuotf.cu:50-60: dst = H src (dst overwritten). */
void hvec_cuda(void *basis, void *net, const double *src, double *dst);
/* cuotf.cu:62-71: diags += diagonal of H (caller zeroes, as jl/fci.jl:3-4). */
void get_diags_elements_cuda(void *basis, void *net, double *diags);
/* cuotf.cu:73-83: vec <- exp(theta G_idx) vec. */
void expm_cuda(void *basis, void *net, int64_t idx, double theta, double *vec);
/* cuotf.cu:85-96: <l| G e^{theta G} |r> in the reference's orientation. */
double grad_cuda(void *basis, void *net, int64_t idx, double theta, const double *l, const double *r);
/* cuotf.cu:98-109: l <- e^{-theta G} l; returns the gradient term; r <- e^{-theta G} r. */
double backgrad_cuda(void *basis, void *net, int64_t idx, double theta, double *l, double *r);
/* cuotf.cu:111-123: grads[g] for every group g at thetas[g] (device arrays,
 * indexed by original group index); grads is overwritten. */
void batchgrad_cuda(void *basis, void *net, const double *thetas, const double *l, const double *r, double *grads);
/* cuotf.cu:125-161: same semantics as the entries above. */
void expm_cuda_2d(void *basis, void *net, int64_t idx, double theta, double *vec);
double grad_cuda_2d(void *basis, void *net, int64_t idx, double theta, const double *l, const double *r);
double backgrad_cuda_2d(void *basis, void *net, int64_t idx, double theta, double *l, double *r);
/* GPU counterparts of the reference CPU library's tvec_contract_otf,
 * backtran_contract_otf, batch_expm_contract_otf and batch_tran_contract_otf
 * (op/declare.hpp:76-123), which jl/cuda/cunetwork.jl:78-84 leaves as no-ops
 * (f_tvec, f_backtran, f_batchexpm, f_batchtran); same arguments on device
 * pointers, idx 0-based.  tvec: dst = T_idx src (dst overwritten).  backtran:
 * l, r <- e^{theta T} l, r and b = T l of the rotated l (b overwritten).
 * batchexpm: e^{theta T} on the first num_vecs columns of the row-major
 * dim x ld matrix.  batchtran: trans[g] = <l|T_g|r> for every group
 * (original order, overwritten). */
void tvec_cuda(void *basis, void *net, int64_t idx, const double *src, double *dst);
void backtran_cuda(void *basis, void *net, int64_t idx, double theta, double *l, double *r, double *b);
void batchexpm_cuda(void *basis, void *net, int64_t idx, double theta, double *matrix, int ld, int num_vecs);
void batchtran_cuda(void *basis, void *net, const double *l, const double *r, double *trans);

/* ========================================================================
 * Part 2: status-returning API.  Every function returns 0 on success or a
 * negative BSIM_ERR_* code; bsim_last_error() describes the last failure of
 * the calling thread.  Work is enqueued on `stream`.
 * ====================================================================== */
enum {
    BSIM_OK = 0,
    BSIM_ERR_NULL = -1,
    BSIM_ERR_ARG = -2,
    BSIM_ERR_UNSUPPORTED = -3,
    BSIM_ERR_ALLOC = -4,
    BSIM_ERR_TIMEOUT = -5,
    BSIM_ERR_CUDA = -6,
    BSIM_ERR_TOO_LARGE = -7
};

const char *bsim_last_error(void);
const char *bsim_version(void);
/* No counterpart in the reference.  Number of device allocations (cudaMalloc /
 * cudaMallocAsync) the library has made in this process, on any device: a
 * caller compares two readings to check that the calls between them allocated
 * nothing. */
int64_t bsim_device_alloc_count(void);
/* No counterpart in the reference.  The solvers' stream-ordered buffers come from
 * a memory pool of the library that keeps freed memory for the next call (a
 * Davidson or VQE call then does not map its vectors anew each time).  This call
 * hands the current device's unused pool memory back (it synchronises the
 * device); the library also does so by itself when a cudaMalloc of its own runs
 * out of memory. */
int bsim_release_cached_memory(void);
/* No counterpart in the reference.  Waits inside the library's tensor-core
 * (tcgen05) kernels are bounded; a wait that gives up makes its CTA skip the
 * rest of its work (the result is then wrong) and is counted.  *count = the
 * count on the current device since the last reset (0 in normal operation);
 * reset != 0 clears it.  Synchronous (reads device memory). */
int bsim_tensor_core_timeouts(int32_t *count, int32_t reset);

/* Basis: create_basis_manager's arguments (basis/declare.hpp:24-33). */
int bsim_basis_create_u32(int64_t norb, int64_t na, int64_t nb, int64_t total_sym, const int64_t *orbsym,
                          int64_t num_irreps, void **out);
/* UInt64 strings (up to 63 spatial orbitals), the string type of the reference's
 * _ui64_f64 operator exports (src/extern/otf_native.cpp:5; jl/network.jl binds
 * build_network_otf_ui64_f64).  Above 26 orbitals a string is addressed by its
 * colex rank instead of a dense 2^norb table (basis.hpp:271 overflows there).
 * Every entry point taking a basis handle accepts either string type; its
 * networks must have the same type. */
int bsim_basis_create_u64(int64_t norb, int64_t na, int64_t nb, int64_t total_sym, const int64_t *orbsym,
                          int64_t num_irreps, void **out);
/* Basis from the reference's host BasisManager<uint32>* (as build_basisdev_f64). */
int bsim_basis_from_host(void *host_basis, void **out);
int bsim_basis_destroy(void *basis);
int64_t bsim_basis_dim(void *basis);
/* Determinant index of (alpha string, beta string) or -1 (set_det_coeff
 * semantics, basis/basis.hpp:298-330). */
int64_t bsim_basis_find_det(void *basis, uint64_t astr, uint64_t bstr);

/* Network: build_network_otf_f64's arguments (op/declare.hpp:25-35); flat_wa /
 * flat_wb hold each group's weights column-major [num_z x rank]. */
int bsim_network_create_u32(const int64_t *orbsym, int64_t norb, int64_t ngs, const uint32_t *axs,
                            const uint32_t *bxs, const int64_t *ranks, const int64_t *num_zas,
                            const int64_t *num_zbs, const uint32_t *flat_zas, const uint32_t *flat_zbs,
                            const double *flat_wa, const double *flat_wb, void **out);
/* build_network_otf_ui64_f64's arguments (otf_native.cpp:5, op/declare.hpp:25-35). */
int bsim_network_create_u64(const int64_t *orbsym, int64_t norb, int64_t ngs, const uint64_t *axs,
                            const uint64_t *bxs, const int64_t *ranks, const int64_t *num_zas,
                            const int64_t *num_zbs, const uint64_t *flat_zas, const uint64_t *flat_zbs,
                            const double *flat_wa, const double *flat_wb, void **out);
/* Network from the reference's host Network_OTF<uint32,double>*. */
int bsim_network_from_host(void *host_net, void **out);
int bsim_network_destroy(void *net);
int64_t bsim_network_ngs(void *net);

/* dst = H src, FP64. */
int bsim_hvec(void *basis, void *net, const double *src, double *dst, bsim_stream_t stream);
/* sigma of nvec HOST vectors: dst_host[k] = H src_host[k] (dim doubles each;
 * the same host buffer may appear in several slots).  The library holds two
 * device input and two output vectors and orders, per step, the host-to-device
 * copy (its own copy stream), sigma (on `stream`) and the device-to-host copy
 * (a second copy stream), so the copies of neighbouring steps overlap the sigma
 * between them; returns when the last result is on the host.  Page-locked host
 * buffers let the copies run asynchronously.  mixed selects the FP32-bulk sigma.
 * The four device vectors stay allocated for the next call while they total at
 * most 8 GB, and are released at the end of the call otherwise. */
int bsim_hvec_host(void *basis, void *net, int64_t nvec, const double *const *src_host, double *const *dst_host,
                   int mixed, bsim_stream_t stream);
/* dst = H src with FP32 bulk (FP32 phases, weights and gathered source,
 * products summed in FP32 per chunk of <= 64 group-ranks) and FP64
 * accumulation across chunks. */
int bsim_hvec_mixed(void *basis, void *net, const double *src, double *dst, bsim_stream_t stream);
/* As bsim_hvec_mixed with an FP32 input vector. */
int bsim_hvec_f32in(void *basis, void *net, const float *src, double *dst, bsim_stream_t stream);
/* Which sigma kernel bsim_hvec uses for this (basis, network) pair: 1 the
 * structured path with the mixed GEMM's source row in shared memory, 2 the
 * structured path with the FP64 source row read from global memory (beta rows
 * longer than shared memory, e.g. 18 orbitals 8 electrons), 0 the generic tile
 * kernel; negative on error.  why receives the reason, and
 * residual_groups the number of groups the structured path leaves to the
 * generic kernel.  Builds (and caches) the plan on first use. */
int bsim_hvec_path(void *basis, void *net, char *why, int why_len, int *residual_groups);
/* Beta-column band of sigma: dst[a, b] = (H src)[a, b] for every alpha row a and
 * col_lo <= b < col_hi (within the single symmetry block; col_lo a multiple of
 * 128), every other element of dst untouched.  src must hold the whole vector.
 * Ranks that split [0, num_b) into such bands compute disjoint parts of one
 * sigma.  Needs the structured path (bsim_hvec_path == 1) with no residual
 * groups, else BSIM_ERR_UNSUPPORTED.  mixed selects FP32 bulk. */
int bsim_hvec_cols(void *basis, void *net, const double *src, double *dst, int64_t col_lo, int64_t col_hi,
                   int mixed, bsim_stream_t stream);
/* Measurement: one structured sigma (dst = H src, FP64 or FP32 bulk) with CUDA
 * events around every launch.  ms_out[i] / launches_out[i] receive the device
 * milliseconds and launch count of stage i for i < nstages: 0 frame+transpose,
 * 1 pure-alpha rows (+ diagonal), 2 pure-beta rows, 3 mixed GEMM, 4 mixed
 * gather, 5 final combine, 6 groups left to the generic kernel, 7 same-spin
 * doubles' intermediate-string GEMM, 8 their gather.  Fails with
 * BSIM_ERR_UNSUPPORTED when the structured path is off. */
int bsim_hvec_stage_times(void *basis, void *net, const double *src, double *dst, int mixed, double *ms_out,
                          int *launches_out, int nstages, bsim_stream_t stream);
/* Measurement: throughput of this GPU in TFLOP/s from chains of dependent
 * operations on every SM: fp64 = 0 FP32 FMA, 1 FP64 FMA, 2 FP64 tensor-core
 * MMA (m8n8k4, the DMMA path the FP64 sigma GEMMs use). */
int bsim_fma_peak(int fp64, double *tflops_out, bsim_stream_t stream);
/* Number of 32 x 32 destination tiles of sigma (block-major, then row-major). */
int64_t bsim_hvec_num_tiles(void *basis);
/* sigma restricted to destination tiles [tile_lo, tile_hi): the rows of those
 * tiles get (H src) there, every other element of dst is left untouched.  A
 * contiguous tile range is a contiguous range of 32-row bands, so ranks that
 * split [0, num_tiles) share sigma by destination rows.  mixed selects FP32 bulk. */
int bsim_hvec_tiles(void *basis, void *net, const double *src, double *dst, int64_t tile_lo, int64_t tile_hi,
                    int mixed, bsim_stream_t stream);
/* diags += diagonal of H. */
int bsim_diag(void *basis, void *net, double *diags, bsim_stream_t stream);
/* vec <- exp(theta G_idx) vec. */
int bsim_expm(void *basis, void *net, int64_t idx, double theta, double *vec, bsim_stream_t stream);
/* vec <- exp(theta[n-1] G_idx[n-1]) ... exp(theta[0] G_idx[0]) vec; idx/theta are host arrays. */
int bsim_expm_seq(void *basis, void *net, int64_t n, const int64_t *idx, const double *theta, double *vec,
                  bsim_stream_t stream);
/* *out_dev (a device double) = grad term; nothing is read back. */
int bsim_grad(void *basis, void *net, int64_t idx, double theta, const double *l, const double *r,
              double *out_dev, bsim_stream_t stream);
/* No counterpart in the reference.  The same result as bsim_grad, for callers
 * that must not allocate device memory once running (a host whose memory pool
 * already owns the device, or a loop that cannot afford cudaMalloc's implicit
 * synchronisation): its reduction scratch is a fixed array inside the library
 * (65536 partial sums, 512 KiB per GPU, held until the process exits), so no
 * call allocates.  Limit: (alpha strings of the largest block) x (symmetry
 * blocks) <= 65536, else BSIM_ERR_TOO_LARGE and nothing runs.  The first call
 * on a device looks up the array's device address; make that first call
 * before any stream capture.  All calls share the array: calls that overlap
 * on the GPU (other streams or host threads) race, so issue them on one stream. */
int bsim_grad_noalloc(void *basis, void *net, int64_t idx, double theta, const double *l, const double *r,
                      double *out_dev, bsim_stream_t stream);
/* Fused adjoint step; *out_dev (device) = gradient term. */
int bsim_backgrad(void *basis, void *net, int64_t idx, double theta, double *l, double *r, double *out_dev,
                  bsim_stream_t stream);
/* Pool gradient (thetas, grads: device, original group order). */
int bsim_batchgrad(void *basis, void *net, const double *thetas, const double *l, const double *r,
                   double *grads, bsim_stream_t stream);
/* ------------------------------------------------------------------------
 * Native network construction (host code, no device work): the grouping and
 * SVD compression of jl/network.jl:158-246 for nterms aabb Pauli terms
 * (per-spin X / Z masks and real coefficients).  Terms with equal (ax, bx)
 * form a group (groups in order of first appearance); each group's matrix
 * M[za, zb] (distinct za, zb ascending) is factorised by a one-sided Jacobi
 * SVD, singular values above tol kept, wa = U sqrt(S), wb = V sqrt(S) with
 * entries below 1e-12 zeroed.  bsim_netbuild_sizes gives the array lengths of
 * bsim_netbuild_export, whose outputs are the bsim_network_create_* arguments
 * (flat_* may be NULL to skip them).
 * ------------------------------------------------------------------------ */
int bsim_netbuild_compress(int64_t nterms, const uint64_t *ax, const uint64_t *az, const uint64_t *bx,
                           const uint64_t *bz, const double *coef, double tol, void **out);
/* As bsim_netbuild_compress with one group per run of run_sizes[r] consecutive
 * terms (the pool form, one X group per generator: jl/network.jl:248-301); every
 * term of a run must share its (ax, bx). */
int bsim_netbuild_compress_runs(int64_t nterms, const uint64_t *ax, const uint64_t *az, const uint64_t *bx,
                                const uint64_t *bz, const double *coef, double tol, int64_t nruns,
                                const int64_t *run_sizes, void **out);
/* The same compression with every group's SVD on the GPU: groups (by key, or
 * one per run when nruns > 0) formed on the host, then all groups' one-sided
 * Jacobi SVDs in one batched launch on the stream (one CTA per group, the
 * disjoint column pairs of each round-robin round rotated in parallel, the host
 * builder's rotation, skip and convergence rules); the result handle is read
 * with bsim_netbuild_sizes / bsim_netbuild_export.  No reference counterpart
 * (the reference compresses on the host: jl/network.jl:158-301). */
int bsim_netbuild_compress_device(int64_t nterms, const uint64_t *ax, const uint64_t *az, const uint64_t *bx,
                                  const uint64_t *bz, const double *coef, double tol, int64_t nruns,
                                  const int64_t *run_sizes, bsim_stream_t stream, void **out);
int bsim_netbuild_sizes(void *h, int64_t *ngs, int64_t *nza_total, int64_t *nzb_total, int64_t *nwa_total,
                        int64_t *nwb_total);
int bsim_netbuild_export(void *h, uint64_t *axs, uint64_t *bxs, int64_t *ranks, int64_t *num_zas, int64_t *num_zbs,
                         uint64_t *flat_zas, uint64_t *flat_zbs, double *flat_wa, double *flat_wb);
int bsim_netbuild_destroy(void *h);

/* ------------------------------------------------------------------------
 * Pool-gradient plan (host code, no device work).  Recognises each group of a
 * generator network (the bsim_network_create_* arrays) as
 * lam * (t - t^dagger), t a spin-orbital excitation with at most two creators
 * and two annihilators (the pool components of jl/adapt.jl, one group per
 * component as jl/network.jl:248-301 builds them).  For such groups the pool
 * gradient at theta = 0 (batch_grad_contract_otf, op/batchgrad.hpp:529-540)
 * is grad_g = coef[g] * (X[dagger(i)] - X[i]), i = idx[4g..4g+3] and X one of
 * the transition densities of l~ = eps l, r~ = eps r (eps(a, b) =
 * (-1)^popc(b & K(a)), K(a) = XOR over alpha electrons i of (1 << i) - 1)
 * chosen by kind[g]:
 *   BSIM_POOL_D1A  X[p][q]       = <l~| a+_p a_q |r~> (alpha),  dagger(p,q) = (q,p)
 *   BSIM_POOL_D1B  the same for beta
 *   BSIM_POOL_TAB  X[p][q][r][s] = <l~| a+_p a_q (alpha) a+_r a_s (beta) |r~>,
 *                  dagger(p,q,r,s) = (q,p,s,r)
 *   BSIM_POOL_GAA  X[p][q][r][s] = <l~| a+_p a+_q a_r a_s |r~> (alpha),
 *                  dagger(p,q,r,s) = (s,r,q,p)
 *   BSIM_POOL_GBB  the same for beta
 * BSIM_POOL_ZERO marks groups whose gradient is zero for real vectors
 * (diagonal or empty groups); BSIM_POOL_GENERAL groups match no excitation and
 * keep the pair-list gradient.  norb <= 64.
 * ------------------------------------------------------------------------ */
enum {
    BSIM_POOL_GENERAL = -1,
    BSIM_POOL_ZERO = 0,
    BSIM_POOL_D1A = 1,
    BSIM_POOL_D1B = 2,
    BSIM_POOL_TAB = 3,
    BSIM_POOL_GAA = 4,
    BSIM_POOL_GBB = 5
};
int bsim_poolplan_classify(int64_t norb, int64_t ngs, const uint64_t *axs, const uint64_t *bxs,
                           const int64_t *ranks, const int64_t *num_zas, const int64_t *num_zbs,
                           const uint64_t *flat_zas, const uint64_t *flat_zbs, const double *flat_wa,
                           const double *flat_wb, int32_t *kind, int32_t *idx, double *coef);
/* The transition densities of the pool plan on the GPU (bases with at least one
 * electron of each spin; a symmetry-blocked basis is computed in the dense array
 * over all alpha and beta strings, without a saving from its symmetry).
 * bsim_pooldensity_create takes a basis handle and the host arrays of
 * bsim_poolplan_classify (idx as 4 int32 per group) and allocates the hole tables
 * and the table scratch (2 x alpha strings x beta strings + (norb^2)^2 doubles and
 * more); the basis handle must outlive the plan.  bsim_pooldensity_grad writes
 * grads[g] = coef[g] (X[dagger(i)] - X[i]) for every group on device vectors l, r
 * (0 for BSIM_POOL_ZERO, NaN for BSIM_POOL_GENERAL groups, whose gradient the
 * pair-list call gives).  bsim_pooldensity_hole_table (host) lists the hole
 * strings of a string list in increasing order and, per hole string h and created
 * orbital (holes = 1: p; holes = 2: the pair x > y at x (x - 1) / 2 + y, created as
 * a+_x a+_y |h>), the entry (index of the created string << 1) | creation sign,
 * or -1; table may be NULL to get *nh only. */
int bsim_pooldensity_hole_table(int64_t norb, int64_t holes, int64_t nstr, const uint64_t *strs, int64_t *nh,
                                int32_t *table);
int bsim_pooldensity_create(void *basis, int64_t ngs, const int32_t *kind, const int32_t *idx, const double *coef,
                            void **out);
int bsim_pooldensity_grad(void *plan, const double *l, const double *r, double *grads, bsim_stream_t stream);
int bsim_pooldensity_destroy(void *plan);

/* ------------------------------------------------------------------------
 * Complex (c64) networks and operators: the reference CPU library's _c64
 * exports (src/extern/otf_native.cpp:4,6; Tv = complex<double>) on device
 * vectors of interleaved (re, im) doubles, dim complex entries each.  The
 * reference has no GPU counterpart.  flat_wa / flat_wb hold interleaved complex
 * weights (2 doubles per weight, the layout of ComplexF64 arrays); the other
 * arguments are those of bsim_network_create_u32 / _u64.  A c64 network works
 * only with the _c64 calls (and bsim_network_destroy), and any basis handle.
 * Semantics per call as the real ones, with the complex rules of
 * core/math.hpp:7-252 (diagonal groups: exp(i theta Im vt) factors):
 *   hvec: dst = H src (overwritten); diag: diag += diagonal (accumulates);
 *   expm: vec <- e^{theta G} vec; grad / backgrad: *out_dev (2 doubles, device)
 *   = the complex gradient term; tvec: dst = T src (overwritten); backtran:
 *   l, r <- e^{theta T} l, r and b = T l (overwritten); batchexpm on num_vecs
 *   entries of ld per determinant; batchgrad: grads[g] at thetas_host[g] (host
 *   angles, device complex grads); batchtran: trans[g] = <l|T_g|r>.
 * ------------------------------------------------------------------------ */
int bsim_network_create_c64(const int64_t *orbsym, int64_t norb, int64_t ngs, const uint32_t *axs,
                            const uint32_t *bxs, const int64_t *ranks, const int64_t *num_zas,
                            const int64_t *num_zbs, const uint32_t *flat_zas, const uint32_t *flat_zbs,
                            const double *flat_wa, const double *flat_wb, void **out);
int bsim_network_create_c64_u64(const int64_t *orbsym, int64_t norb, int64_t ngs, const uint64_t *axs,
                                const uint64_t *bxs, const int64_t *ranks, const int64_t *num_zas,
                                const int64_t *num_zbs, const uint64_t *flat_zas, const uint64_t *flat_zbs,
                                const double *flat_wa, const double *flat_wb, void **out);
int bsim_hvec_c64(void *basis, void *net, const double *src, double *dst, bsim_stream_t stream);
int bsim_diag_c64(void *basis, void *net, double *diag, bsim_stream_t stream);
int bsim_expm_c64(void *basis, void *net, int64_t idx, double theta, double *vec, bsim_stream_t stream);
int bsim_grad_c64(void *basis, void *net, int64_t idx, double theta, const double *l, const double *r,
                  double *out_dev, bsim_stream_t stream);
int bsim_backgrad_c64(void *basis, void *net, int64_t idx, double theta, double *l, double *r, double *out_dev,
                      bsim_stream_t stream);
int bsim_tvec_c64(void *basis, void *net, int64_t idx, const double *src, double *dst, bsim_stream_t stream);
int bsim_backtran_c64(void *basis, void *net, int64_t idx, double theta, double *l, double *r, double *b,
                      bsim_stream_t stream);
int bsim_batchexpm_c64(void *basis, void *net, int64_t idx, double theta, double *matrix, int ld, int num_vecs,
                       bsim_stream_t stream);
int bsim_batchgrad_c64(void *basis, void *net, const double *thetas_host, const double *l, const double *r,
                       double *grads, bsim_stream_t stream);
int bsim_batchtran_c64(void *basis, void *net, const double *l, const double *r, double *trans, bsim_stream_t stream);

/* Status-returning forms of tvec_cuda, backtran_cuda, batchexpm_cuda and
 * batchtran_cuda (same semantics; every group type and symmetry-block layout;
 * batchexpm needs 0 <= num_vecs <= ld). */
int bsim_tvec(void *basis, void *net, int64_t idx, const double *src, double *dst, bsim_stream_t stream);
int bsim_backtran(void *basis, void *net, int64_t idx, double theta, double *l, double *r, double *b,
                  bsim_stream_t stream);
int bsim_batchexpm(void *basis, void *net, int64_t idx, double theta, double *matrix, int ld, int num_vecs,
                   bsim_stream_t stream);
int bsim_batchtran(void *basis, void *net, const double *l, const double *r, double *trans, bsim_stream_t stream);
/* vec <- prod_i exp(thetas[param_idx[i]] G_{op_idx[i]}) |ref>, |ref> = sum_j ref_val[j] e_{ref_idx[j]};
 * all index/angle arrays are host arrays. */
int bsim_prepare_state(void *basis, void *pool, int64_t n_ops, const int64_t *op_idx, const int64_t *param_idx,
                       const double *thetas, const int64_t *ref_idx, const double *ref_val, int64_t n_ref,
                       double *vec, bsim_stream_t stream);
/* VQE energy E = <psi|H|psi>/<psi|psi>, variance <H^2> - E^2 and the adjoint
 * gradient dE/dtheta_p (jl/vqe.jl:1-21) for psi = prepare_state(...).
 * Components sharing a parameter (spin-adapted generators) sum their terms.
 * ckpt_every > 0 stores the forward state every ckpt_every parameters and
 * restores it during the reverse sweep.  lv, rv: device work vectors (dim).
 * energy, variance, grad[n_params]: host outputs. */
int bsim_vqe_energy_grad(void *basis, void *ham, void *pool, int64_t n_ops, const int64_t *op_idx,
                         const int64_t *param_idx, int64_t n_params, const double *thetas, const int64_t *ref_idx,
                         const double *ref_val, int64_t n_ref, int64_t ckpt_every, double *lv, double *rv,
                         double *energy, double *variance, double *grad, bsim_stream_t stream);
/* Lowest eigenpair by Davidson on device (jl/davidson.jl:1-185).  mixed = 0:
 * FP64 throughout (ncv, maxspace as the reference); mixed = 1: FP32 subspace
 * and FP32-bulk sigma inside FP64 residual refinement (ncv unused).  v0 is
 * normalised in place; x_out receives the eigenvector.  Outputs may be NULL. */
int bsim_davidson(void *basis, void *net, double *v0, const double *diags, double tol, int maxiter, int ncv,
                  int maxspace, int mixed, double *x_out, double *energy, double *residual, int *iterations,
                  int *sigma_fp64, int *sigma_fp32, int verbose, bsim_stream_t stream);
/* Lowest nroots (1..8) eigenpairs by block Davidson on device: the steps of
 * jl/davidson.jl:1-185 (Ritz residual, clamped preconditioner, MGS, restart to
 * ncv Ritz vectors) applied to every unconverged root of the block; the
 * reference driver follows one root only.  X (device, nroots x dim, FP64,
 * root-major): start vectors on entry (orthonormalised in place), Ritz vectors
 * on exit.  diags: the Hamiltonian diagonal, FP64 (diag_fp32 = 0) or FP32 (1).
 * nroots <= ncv <= 8, ncv + nroots <= maxspace <= 64.  mixed = 0: FP64
 * subspace (the first nroots subspace vectors are X itself) and FP64 sigma.
 * mixed = 1: FP32 subspace storage and FP32-bulk sigma until the FP32
 * residuals reach tol or stall, then FP64 refinement of the block (FP64 sigma
 * and Rayleigh-Ritz among the roots, FP32 corrections coupled through the FP64
 * sigmas) until every FP64 residual norm is below tol.  energies, residuals
 * (host, nroots): Ritz values and FP64 residual norms at exit; convergence is
 * residuals[i] < tol for all i.  Outputs may be NULL. */
int bsim_davidson_block(void *basis, void *net, int nroots, double *X, const void *diags, int diag_fp32, double tol,
                        int maxiter, int ncv, int maxspace, int mixed, double *energies, double *residuals,
                        int *iterations, int *sigma_fp64, int *sigma_fp32, int verbose, bsim_stream_t stream);

/* ========================================================================
 * Part 3: libdiag's Davidson helpers (diag/declare.hpp:4-75) on device
 * vectors.  N, dim, coeffs and the returned scalars are host values; V / AV
 * are host arrays of device pointers.  Each call completes before returning.
 * ====================================================================== */
/* diag/declare.hpp:7-16 */
double build_ritz_and_residual_cuda(int64_t N, int dim, const double *coeffs, double min_e, const double **V,
                                    const double **AV, double *axt);
/* diag/declare.hpp:18-25 */
void build_ritz_vector_cuda(int64_t N, int dim, const double *coeffs, const double **V, double *xt);
/* diag/declare.hpp:27-34 */
void apply_preconditioner_inplace_cuda(int64_t N, double *axt, const double *diags, double min_e, double shift);
/* diag/declare.hpp:36-42 */
double mgs_orthogonalize_cuda(int64_t N, int dim, const double **V, double *vt);
/* diag/declare.hpp:44-49 */
double inplace_normalize_cuda(int64_t N, double *vec);
/* diag/declare.hpp:51-57 */
double fast_dot_cuda(int64_t N, const double *v1, const double *v2);
/* diag/declare.hpp:59-66: out_col is a host array of dim entries. */
void compute_heff_col_cuda(int64_t N, int dim, const double **V, const double *AV_dim, double *out_col);
/* diag/declare.hpp:68-75: heff is a host array (column-major, leading dim ldh). */
void rebuild_heff_cuda(int64_t N, int dim, const double **V, const double **AV, double *heff, int ldh);

#ifdef __cplusplus
}
#endif

#endif /* BINSIM_CUOTF_H */
