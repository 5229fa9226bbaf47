/*
 * taco_b200.h -- C-ABI of the B200 TCL4 engine (libtaco_b200.so).
 *
 * Plain pointers and sizes only.  Complex numbers are interleaved (re, im) pairs,
 * layout-compatible with std::complex<double> / cuDoubleComplex (taco_c128) and
 * std::complex<float> (taco_c64).  Matrices are column-major, as Eigen's defaults in
 * the reference.  Every entry point returns a taco_status; on failure the message is
 * available from taco_last_error() (thread-local).  The status codes correspond to the
 * exception types the reference throws:
 *   TACO_ERR_INVALID_ARGUMENT  std::invalid_argument
 *   TACO_ERR_OUT_OF_RANGE      std::out_of_range   (time index >= Nt)
 *   TACO_ERR_RUNTIME           std::runtime_error  (pair_to_freq contains -1, ...)
 *   TACO_ERR_OVERFLOW          std::overflow_error (sizes)
 *   TACO_ERR_CUDA              std::runtime_error raised by cuda_check
 *
 * Calls are synchronous (they return after the results are in the output buffers),
 * use one CUDA stream per host thread and device unless a stream is passed, and keep
 * a grow-only device workspace per host thread and device, like the reference's
 * thread-local fused workspace (cpp/src/backend/cuda/tcl4_fused_cuda.cu:676-685).
 */
#ifndef TACO_B200_H
#define TACO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TACO_B200_VERSION "0.1.0"

typedef struct { double re, im; } taco_c128;
typedef struct { float re, im; } taco_c64;

typedef enum {
    TACO_OK = 0,
    TACO_ERR_INVALID_ARGUMENT = 1,
    TACO_ERR_OUT_OF_RANGE = 2,
    TACO_ERR_RUNTIME = 3,
    TACO_ERR_OVERFLOW = 4,
    TACO_ERR_CUDA = 5,
    TACO_ERR_TIMEOUT = 6,
    TACO_ERR_NO_DEVICE = 7
} taco_status;

/* FCRMethod (cpp/include/taco/tcl4_kernels.hpp:11-14).  The device path implements
 * Convolution only, like the reference's fused CUDA path
 * (cpp/src/backend/cuda/tcl4_fused_cuda.cu:1107-1109). */
enum { TACO_FCR_CONVOLUTION = 0, TACO_FCR_DIRECT = 1 };

/* TACO_PREC_FP64: the plain FP64 path (complex128 results).
 * TACO_PREC_FP32: FFT convolutions and the L4 contraction in FP32 (complex64 L4),
 *                 FP64 phases, FP64 prefix-integral carries. */
enum { TACO_PREC_FP64 = 0, TACO_PREC_FP32 = 1 };

/* flags */
enum {
    TACO_IN_DEVICE = 1,          /* gamma (and RK4 inputs) are device pointers */
    TACO_OUT_DEVICE = 2,         /* outputs are device pointers */
    TACO_CAUSAL_TRUNCATION = 4,  /* (default) FFT length from max(tidx)+1: F/C/R(t) depend on gamma[0..t] only */
    TACO_FULL_LENGTH_FFT = 8     /* FFT length from Nt, as the reference (same results, more work) */
};

/* What the device path reads from taco::sys::System (cpp/include/taco/system.hpp:201-226)
 * and the Tcl4Map (cpp/include/taco/tcl4.hpp:13-26). */
typedef struct {
    int N;                       /* system dimension (eig.dim) */
    int nf;                      /* number of Bohr-frequency buckets */
    int num_ops;                 /* number of coupling operators */
    const double* omegas;        /* [nf] bucket frequencies, ascending */
    const int* mirror;           /* [nf] bucket of -omega (NULL: computed as build_map does) */
    const int* pair_to_freq;     /* [N*N] column-major bucket index of pair (a, b) */
    const taco_c128* ops;        /* [num_ops][N*N] column-major coupling operators, eigenbasis */
    double tol;                  /* bucket tolerance used for the mirror search (<= 0: 1e-9) */
} taco_system_view;

/* One instance of the batched build. */
typedef struct {
    taco_system_view sys;
    const taco_c128* gamma;      /* [Nt x nf] column-major: gamma[t + Nt*b] */
    size_t Nt;
    double dt;
    const uint32_t* tidx;        /* host array of requested time indices (NULL/T=0: all Nt) */
    size_t T;
    void* L4_out;                /* [T][N^2 x N^2]: taco_c128 (FP64) or taco_c64 (FP32) */
} taco_tcl4_instance;

const char* taco_version(void);
const char* taco_last_error(void);
int taco_device_count(int* count);
int taco_set_device(int gpu_id);

/* set_fcr_fft_pad_factor / get_fcr_fft_pad_factor (cpp/include/taco/tcl4_kernels.hpp:16-19):
 * Nfft = next_pow2(max(2n-1, factor*n)); 0 keeps the default. */
void taco_set_fcr_fft_pad_factor(size_t factor);
size_t taco_get_fcr_fft_pad_factor(void);

/* compute_triple_kernels(system, gamma_series, dt, nmax, method, exec{Cuda})
 * (cpp/include/taco/tcl4.hpp:37-42, backend cpp/src/backend/cuda/tcl4_kernels_cuda.cu:41-291).
 * F, C, R: [nf^3][Nt] complex128, series of triple (i,j,k) at index (i*nf + j)*nf + k
 * (TripleKernelSeries F[i][j][k](t), cpp/include/taco/tcl4.hpp:30-34). */
int taco_compute_triple_kernels(const taco_system_view* sys, const taco_c128* gamma, size_t Nt, double dt,
                                int method, taco_c128* F, taco_c128* C, taco_c128* R, int flags,
                                void* stream);

/* Batching form of compute_triple_kernels (no counterpart in the reference, which computes
 * one system per call): the F, C, R series of n instances in as few launches as the work
 * budget allows.  Device buffers only (gamma [nf][Nt], F/C/R [nf^3][Nt] complex128);
 * instances with equal Nt share build groups. */
typedef struct {
    taco_system_view sys;
    const taco_c128* gamma;
    size_t Nt;
    double dt;
    taco_c128* F;
    taco_c128* C;
    taco_c128* R;
} taco_fcr_request;
int taco_compute_triple_kernels_batch(const taco_fcr_request* reqs, size_t n, int method, void* stream);

/* build_TCL4_generator_cuda_fused_batch(system, gamma_series, dt, time_indices, method, exec,
 * cuda_fcr_ms) (cpp/include/taco/backend/cuda/tcl4_fused_cuda.hpp:25-41).  tidx == NULL or
 * T == 0 means all time indices [0, Nt).  L4_out: [T][N^2 x N^2] column-major, complex128
 * for TACO_PREC_FP64 and complex64 for TACO_PREC_FP32.  fcr_ms (nullable) receives the
 * device time of the F/C/R stage. */
int taco_tcl4_build_batch(const taco_system_view* sys, const taco_c128* gamma, size_t Nt, double dt,
                          const uint32_t* tidx, size_t T, int method, int precision, void* L4_out,
                          int flags, void* stream, double* fcr_ms);

/* build_TCL4_generator_cuda_fused(system, gamma_series, dt, time_index, method, exec)
 * (cpp/include/taco/backend/cuda/tcl4_fused_cuda.hpp:16-21). */
int taco_tcl4_build(const taco_system_view* sys, const taco_c128* gamma, size_t Nt, double dt,
                    size_t time_index, int method, taco_c128* L4_out, int flags, void* stream);

/* build_correction_series_cuda_fused (cpp/include/taco/backend/cuda/tcl4_fused_cuda.hpp:44-48):
 * L4 at every t in [0, Nt). */
int taco_tcl4_correction_series(const taco_system_view* sys, const taco_c128* gamma, size_t Nt,
                                double dt, int method, taco_c128* L4_out, int flags, void* stream);

/* Batching form (no counterpart in the reference): many instances of possibly different
 * (N, nf, Nt, T) in one call; instances sharing an FFT length share every launch. */
int taco_tcl4_build_instances(const taco_tcl4_instance* inst, size_t count, int method, int precision,
                              int flags, void* stream);

/* Plans (no counterpart in the reference, whose fused path caches one CUDA graph per
 * shape, cpp/src/backend/cuda/tcl4_fused_cuda.cu:164-191): validate and prepare a batched
 * build once -- metadata and job tables resident on the device, the whole launch sequence
 * captured in a CUDA graph -- and replay it.  Inputs and outputs must be device pointers
 * (TACO_IN_DEVICE | TACO_OUT_DEVICE); they are bound at creation.  taco_tcl4_plan_execute
 * is asynchronous on exactly `stream` (NULL is the legacy default stream, not the library's
 * per-thread stream), so the caller orders it with its own work and synchronises. */
typedef struct taco_tcl4_plan taco_tcl4_plan;
int taco_tcl4_plan_create(const taco_tcl4_instance* inst, size_t count, int method, int precision, int flags,
                          taco_tcl4_plan** plan);
int taco_tcl4_plan_execute(taco_tcl4_plan* plan, void* stream);
int taco_tcl4_plan_destroy(taco_tcl4_plan* plan);

/* No counterpart in the reference.  The L4 build of one instance (the job of
 * taco_tcl4_build_batch with TACO_IN_DEVICE | TACO_OUT_DEVICE) for callers that cannot
 * allocate device memory while they run: code inside a framework whose caching allocator
 * already holds the GPU's memory, latency-critical loops where cudaMalloc/cudaFree would
 * synchronise the device, plugin hosts that forbid allocation after start-up.  It calls no
 * cudaMalloc, cudaFree or other allocating routine: all scratch comes from one fixed device
 * array of TACO_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until the
 * process exits.  gamma ([Nt x nf] column-major) and L4_out ([T][N^2 x N^2]: complex128 for
 * TACO_PREC_FP64, complex64 for TACO_PREC_FP32) must be device (or managed) memory of the
 * current device, aligned for their complex type; anything else fails with
 * TACO_ERR_INVALID_ARGUMENT before any launch.  tidx is a host array (NULL/T = 0: all Nt).
 * The FFT length is a power of two following max(tidx)+1.  A request whose scratch would
 * exceed the fixed size fails with TACO_ERR_OVERFLOW and a message stating the need.  The
 * first call on a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current.  All calls share the array, so calls that overlap on the GPU (other
 * threads or streams) race.  The call copies its metadata from pageable host memory and
 * synchronises `stream` (NULL: the legacy default stream) before returning; on a stream
 * that is being captured it fails with TACO_ERR_INVALID_ARGUMENT before any work. */
#define TACO_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)
int taco_tcl4_build_batch_noalloc(const taco_system_view* sys, const taco_c128* gamma, size_t Nt, double dt,
                                  const uint32_t* tidx, size_t T, int precision, void* L4_out, void* stream);

/* propagate_rk4_dense_serial/_omp(L_series[, L_half_series], r, t0, dt, on_sample, sample_every)
 * (cpp/include/taco/rk4_dense.hpp:85-100, 114-129) on the device.
 * L_series: [steps+1][D x D]; L_half: [steps][D x D] or NULL (midpoints by averaging);
 * L_add: [steps+1][D x D] or NULL, added to L_series (e.g. L2 + L4);
 * l_is_fp32: the three series are complex64 instead of complex128;
 * r: [D] complex128 in/out; samples (nullable): r every sample_every steps plus the final
 * state, [n][D]; obs (nullable, [D]) and obs_out ([n]): <O> = sum_l obs_l r_l at each sample.
 * n = ceil(steps / sample_every) + 1.  All pointers follow TACO_IN_DEVICE. */
int taco_rk4_propagate(const void* L_series, const void* L_half, const void* L_add, int l_is_fp32,
                       size_t steps, int D, double dt, taco_c128* r, size_t sample_every,
                       taco_c128* samples, const taco_c128* obs, taco_c128* obs_out, int flags,
                       void* stream);

/* The TCL2 generator L2(t) = -i[diag(eps) + H_LS(t), .] + D2(t) at the requested times
 * (build_tcl2_components(...).total(), cpp/src/tcl/generator.cpp:164-177, with the
 * spin-boson example's kernel fill, examples/TCL4_spin_boson_example.cpp:303-315).
 * eps: [N] eigenvalues (host).  L2_out: [T][N^2 x N^2] complex128. */
int taco_tcl2_generator_series(const taco_system_view* sys, const double* eps, const taco_c128* gamma, size_t Nt,
                               const uint32_t* tidx, size_t T, taco_c128* L2_out, int flags, void* stream);

/* gamma::compute_trapz_prefix_multi_matrix (cpp/include/taco/gamma.hpp:166-213) on the
 * device: G [M][N] (the reference's column-major N x M) from C [N]; omegas: host [M]. */
int taco_gamma_trapz(const taco_c128* C, size_t N, double dt, const double* omegas, size_t M, taco_c128* G,
                     int flags, void* stream);

/* The example's propagation (examples/TCL4_spin_boson_example.cpp:317-394) on the device:
 * L(t_k) = L0 (order 0), L2(t_k) (order 2) or L2(t_k) + L4(t_k) (order 4) for k = 0..steps,
 * RK4 with midpoints by averaging, rho(0) = rho0 ([N^2] vec, eigenbasis), FP64 state.
 * obs (nullable, [N^2]) gives <O>(t) = sum_l obs_l r_l every sample_every steps plus the
 * final step (obs_out: ceil(steps/sample_every)+1 values); rho_out (nullable): final state.
 * precision applies to the L4 build (FP32: complex64 L4 added to the FP64 L2). */
int taco_propagate_tcl(const taco_system_view* sys, const double* eps, const taco_c128* gamma, size_t Nt, double dt,
                       size_t steps, int order, int precision, const taco_c128* rho0, const taco_c128* obs,
                       size_t sample_every, taco_c128* obs_out, taco_c128* rho_out, int flags, void* stream);

/* The unfused stages, batched over T times (leading dimension), for callers of the
 * reference's stage-by-stage API.  All array arguments follow TACO_IN_DEVICE / TACO_OUT_DEVICE.
 * build_mikx_cuda / build_mikx_cuda_batch (cpp/include/taco/backend/cuda/tcl4_mikx_cuda.hpp:56-79):
 *   F, C, R: [T][nf^3] at (i*nf + j)*nf + k; pair_to_freq [N*N] column-major;
 *   M, I, K: [T][N^2 x N^2] column-major (row (j,k) = j + N k); X: [T][N^6] flat6 order. */
int taco_build_mikx(const taco_c128* F, const taco_c128* C, const taco_c128* R, const int* pair_to_freq, int N,
                    int nf, size_t T, taco_c128* M, taco_c128* I, taco_c128* K, taco_c128* X, int flags, void* stream);
/* assemble_liouvillian_cuda (cpp/include/taco/backend/cuda/tcl4_assemble_cuda.hpp:18-44): GW [T][N^2 x N^2]
 * (row (n,i), col (m,j)); symmetrize = 0 gives the raw T (assemble_liouvillian_cuda_device_raw). */
int taco_assemble_liouvillian(const taco_c128* M, const taco_c128* I, const taco_c128* K, const taco_c128* X,
                              const taco_c128* ops, int N, int num_ops, size_t T, int symmetrize, taco_c128* GW,
                              int flags, void* stream);
/* gw_to_liouvillian (cpp/include/taco/tcl4_assemble.hpp:18-21): L4(n + N m, i + N j) = GW(n + N i, m + N j). */
int taco_gw_to_liouvillian(const taco_c128* GW, int N, size_t T, taco_c128* L4, int flags, void* stream);

/* The time-independent linear map L4_e(t) = sum_k coef_k * v_{src_k}(t) (v conjugated when
 * bit 31 of src_k is set) of the MIKX -> GW -> L4 chain (cpp/src/tcl/tcl4_mikx.cpp:87-177,
 * cpp/src/tcl/tcl4_assemble.cpp:53-230).  Sources: F (s < nf^3), C, R of triple s mod nf^3.
 * rowptr: [N^4 + 1]; src/coef: capacity `cap`; nnz receives the number of terms (when it
 * exceeds cap only nnz is written). */
int taco_l4_coefficients(const taco_system_view* sys, int32_t* rowptr, uint32_t* src, taco_c128* coef,
                         size_t cap, size_t* nnz);

/* Transient device memory one group of a build may use (0, the default: 45% of the free
 * memory at the call, at most 64 GiB).  Instances that need more are built in slices of
 * their frequency triples (same results, more passes over the output). */
int taco_set_work_budget(size_t bytes);
/* No counterpart in the reference.  Precision guard of the FP32 form (TACO_PREC_FP32 builds
 * and plans): after the FP32 build, a head of each instance's leading times [0, H) is built
 * in FP64 (t_count = max(tidx)+1; H = t_count/4 for plans, t_count/16 for direct calls, at
 * least 512) and compared with the FP32 result row by row; the FP32 rows up to the last
 * dyadic window [2^k, 2^(k+1)) that misses `tol` (relative Frobenius) are replaced by FP64
 * rows, the head growing fourfold while the misses reach its end, up to a full FP64 build of
 * the instance.  The FP64 rows below 2048 and 256 come from builds of those times alone
 * (short FFTs, whose round-off at the first, tiny L4 values is far below the full-length
 * transform's) wherever those builds change the head's rows by more than tol/8.  Plans
 * choose their heads once, at creation, and replay them beside the FP32 graph; direct calls
 * remember, per gamma buffer and a fingerprint of its contents, the heads a call needed,
 * prepare them once as FP64 plans and replay them beside the next calls' FP32 passes.
 * tol = 0 turns the guard off; the default is 5e-7.  taco_get_fp32_guard returns the
 * current value. */
/* No counterpart in the reference.  The fused F/C/R path: for FFT lengths whose working
 * array fits one CTA's shared memory (FP32 up to 24576 points, FP64 up to 12288), one CTA per
 * (triple, half) runs the forward transform, the spectral product, the inverse transform, the
 * prefix integrals and the assembly in shared memory.  on = 0 (the default) selects the
 * four-step passes and the scan kernels for every length; results agree to rounding.  On
 * B200 the fused path is the slower one at the lengths it fits (one CTA per SM, latency
 * bound), so it stays off unless selected.  taco_get_fused_conv returns the setting. */
int taco_set_fused_conv(int on);
int taco_get_fused_conv(int* on);
/* No counterpart in the reference (whose thread_local workspace is freed at thread exit,
 * cpp/src/backend/cuda/tcl4_fused_cuda.cu:676-685).  Frees the calling thread's grow-only
 * device and pinned transient buffers on the current device after its streams finish, with
 * the precision guard's buffers and the FP64 heads it prepared for repeated direct calls;
 * the next call allocates them again.  Plans keep their own buffers. */
int taco_release_workspace(void);
int taco_set_fp32_guard(double tol);
int taco_get_fp32_guard(double* tol);
/* What the guard did in the calling thread's last FP32 build or plan creation, six counts:
 * instances of the call, instances with an FP64 head, requested times rebuilt in FP64,
 * requested times of those instances, instances rebuilt in FP64 entirely, growth rounds. */
int taco_fp32_guard_stats(uint64_t* counts6);
/* No counterpart in the reference.  Bytes of FP64 head rows the precision guard builds and
 * patches at a time (0: the default, 1 GiB): heads beyond it are built in further chunks
 * (plans then replay their heads after the FP32 graph instead of beside it; direct calls
 * check them instead of replaying remembered ones).  For memory-tight batches and tests. */
int taco_set_guard_chunk_bytes(size_t bytes);
/* FFT length the build uses for n_in consumed samples (flags: TACO_FULL_LENGTH_FFT selects
 * the reference's power-of-two rule), and its schedule key for taco_set_tuning: log2 of a
 * power of two, + 64 for 3 * 2^k, + 128 for 5 * 2^k. */
int taco_fft_length(size_t n_in, int precision, int flags, size_t* nfft, int* key);
/* Launch schedule of the F/C/R passes for the FFT length with schedule key `log2_nfft`
 * (taco_fft_length) and a precision, as chosen by the autotuner (taco_b200/autotune.py):
 * column / row tile sizes in elements (powers of two in [8, 8192]), bytes of Z/W scratch per
 * chunk of triples, and the largest number of output rows for which the inverse column pass
 * is a pruned direct DFT.  Unset lengths use the defaults (4096, 2048, 48 MiB, 0). */
int taco_set_tuning(int log2_nfft, int precision, int col_tile, int row_tile, size_t chunk_bytes, int inv_dft_rows);
/* No counterpart in the reference.  Whether the causal rule may pick the mixed length of
 * schedule key `key` (64 + k: 3 * 2^k, 128 + k: 5 * 2^k) for `precision`; the autotuner turns
 * off a mixed length that it measured slower than the next longer one (default: enabled). */
int taco_set_fft_length_enabled(int key, int precision, int enabled);
int taco_get_tuning(int log2_nfft, int precision, int* col_tile, int* row_tile, size_t* chunk_bytes,
                    int* inv_dft_rows);
/* Points per CTA of the thread-block-cluster convolution path for FFT length 2^log2_nfft:
 * -1 automatic (2^13 FP32 / 2^12 FP64 points per CTA, at most 8 CTAs per cluster), 0 the
 * multi-pass four-step path, 3..13 a fixed 2^log2_points (clamped to the precision's maximum). */
int taco_set_cluster_points(int log2_nfft, int precision, int log2_points);
int taco_clear_tuning(void);

/* Kernel accounting (tracing).  taco_kernel_launches: kernels this library launched since
 * the process started.  With profiling on, every launch is bracketed by CUDA events and its
 * device time is summed per kernel name (CUDA-event stage timing, as the reference's
 * TACO_CUDA_FCR_PROFILE / TACO_CUDA_GW_PROFILE switches).  taco_profile_get returns entry
 * `index` (name valid until the next reset) and writes the number of entries to *count. */
int taco_kernel_launches(uint64_t* launches);
int taco_profile_enable(int on);
int taco_profile_reset(void);
int taco_profile_get(size_t index, const char** name, uint64_t* launches, double* total_ms, size_t* count);

/* Batched trapezoid Gamma on device arrays: C [N], G [M][N] per request (omegas on the host). */
typedef struct {
    const taco_c128* C;
    size_t N;
    double dt;
    const double* omegas;
    size_t M;
    taco_c128* G;
} taco_gamma_request;
int taco_gamma_trapz_batch(const taco_gamma_request* reqs, size_t n, void* stream);

/* ---------------------------------------------------------------------------------------
 * Bath correlation function on the device: bcf_fft_fun (cpp/include/taco/correlation_fft.hpp:153-214)
 * for J(w) = alpha w e^{-w/omega_c} (+ 2 lambda gamma w / (w^2 + gamma^2) when model = 1), and
 * its derivatives in alpha, omega_c, beta (which = 1, 2, 3; the Drude-Lorentz terms are held
 * fixed).  out[k] = C(k dt) (or its derivative) for k < n_out <= N + 1; host arrays unless
 * TACO_OUT_DEVICE.  Requests are batched into one pair of launches per FFT length. */
typedef struct {
    int model;
    int which;
    double alpha, omega_c, lambda, gamma, beta;
    size_t N;
    double dt;
    taco_c128* out;
    size_t n_out;
} taco_bcf_request;
int taco_bcf_fft(const taco_bcf_request* reqs, size_t n, int flags, void* stream);

/* ---------------------------------------------------------------------------------------
 * Differentiation.  Real losses; every gradient G(z) = dloss/dRe z + i dloss/dIm z.
 * All arrays are device pointers except where marked host.  No reference counterpart: the
 * reference has no derivatives.
 *
 * RK4 with checkpoints (the endpoint overload of propagate_rk4_dense, rk4_dense.hpp:85-129,
 * Lh = (L_i + L_{i+1}) / 2): taco_rk4_forward_checkpointed writes <O> samples, the final state
 * and the state every checkpoint_every steps; taco_rk4_adjoint recomputes each segment from its
 * checkpoint and returns G(L) for every endpoint, G(rho0) and G(obs).  D = N^2 <= 16. */
typedef struct {
    const taco_c128* L;            /* [steps+1][D x D] column-major */
    const taco_c128* L_add;        /* nullable, added to L (its gradient is L_bar) */
    size_t steps;
    int D;
    double dt;
    const taco_c128* r0;           /* [D] */
    const taco_c128* obs;          /* [D]: <O> = sum_l obs_l r_l (nullable without samples) */
    size_t sample_every;           /* samples at steps 0, s, 2s, ... < steps, and after the last */
    taco_c128* ckpt;               /* [ceil(steps / checkpoint_every)][D] */
    taco_c128* obs_out;            /* forward: samples of <O> (nullable) */
    taco_c128* r_out;              /* forward: final state (nullable) */
    const taco_c128* obs_bar;      /* adjoint: G(<O>) per sample (nullable) */
    const taco_c128* r_final_bar;  /* adjoint: G(final state) (nullable) */
    taco_c128* L_bar;              /* adjoint out: [steps+1][D x D] */
    taco_c128* r0_bar;             /* adjoint out: [D] (nullable) */
    taco_c128* obs_vec_bar;        /* adjoint out: [D] (nullable) */
} taco_rk4_grad_job;
int taco_rk4_forward_checkpointed(const taco_rk4_grad_job* jobs, size_t n, size_t checkpoint_every, void* stream);
int taco_rk4_adjoint(const taco_rk4_grad_job* jobs, size_t n, size_t checkpoint_every, void* stream);

/* Adjoint of L4(t), t = 0..T-1 (build_TCL4_generator_cuda_fused_batch with all times), through
 * GW/MIKX (tcl4_assemble.cpp:53-230, tcl4_mikx.cpp:87-177) and the F/C/R kernels
 * (tcl4_kernels.cpp:105-281): accumulates G(gamma) ([nf][T], gamma[b*T + t]), dloss/domega_b
 * (host [nf]) and, when the forward F/C/R series ([nf^3][T] each) are given, G(ops) (host
 * [num_ops][N*N]).  nf <= 27. */
typedef struct {
    const taco_system_view* sys;
    const taco_c128* gamma;
    size_t T;
    double dt;
    const taco_c128* L_bar;        /* [T][N^2 x N^2] */
    const taco_c128* F;            /* nullable */
    const taco_c128* C;
    const taco_c128* R;
    taco_c128* gamma_bar;          /* accumulated */
    double* omega_bar;             /* host, accumulated (nullable) */
    taco_c128* ops_bar;            /* host, accumulated (nullable) */
} taco_tcl4_adjoint_job;
int taco_tcl4_adjoint(const taco_tcl4_adjoint_job* jobs, size_t n, void* stream);

/* Adjoint of the TCL2 generator series (generator.cpp:42-177, the example's kernel fill):
 * accumulates G(gamma), and (host) G(ops) and dloss/deps. */
typedef struct {
    const taco_system_view* sys;
    const double* eps;             /* host [N] eigenvalues */
    const taco_c128* gamma;        /* [nf][T] */
    size_t T;
    const taco_c128* L_bar;        /* [T][N^2 x N^2] */
    taco_c128* gamma_bar;          /* accumulated */
    taco_c128* ops_bar;            /* host, accumulated (nullable) */
    double* eps_bar;               /* host [N], accumulated (nullable) */
} taco_tcl2_adjoint_job;
int taco_tcl2_adjoint(const taco_tcl2_adjoint_job* jobs, size_t n, void* stream);

/* out[k] = sum_i Re(conj(a_k[i]) b_k[i]) for device vectors (host out). */
typedef struct {
    const taco_c128* a;
    const taco_c128* b;
    size_t n;
} taco_inner_job;
int taco_inner_re(const taco_inner_job* jobs, size_t n, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
