// engine.hpp -- host orchestration of the TCL4 device path (no torch types).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <memory>
#include <vector>

#include "common.cuh"

namespace taco {

struct SystemDesc {
    int N = 0, nf = 0, num_ops = 0;
    std::vector<double> omegas;
    std::vector<int> mirror;
    std::vector<int> p2f;       // column-major N x N
    std::vector<double2> ops;   // num_ops x (N x N) column-major
};

// Requested time indices of an instance.  Instances of one call that name the same caller
// array share one copy (share_with), so their time maps are derived and uploaded once.
class TimeList {
public:
    std::size_t size() const { return v_ ? v_->size() : 0; }
    bool empty() const { return size() == 0; }
    uint32_t operator[](std::size_t k) const { return (*v_)[k]; }
    const uint32_t* begin() const { return v_ ? v_->data() : nullptr; }
    const uint32_t* end() const { return v_ ? v_->data() + v_->size() : nullptr; }
    const std::vector<uint32_t>& vec() const { return v_ ? *v_ : empty_vec(); }
    const void* identity() const { return v_.get(); }
    void assign(const uint32_t* first, const uint32_t* last) {
        v_ = std::make_shared<std::vector<uint32_t>>(first, last);
    }
    void iota(std::size_t n) {  // 0, 1, ..., n-1
        auto v = std::make_shared<std::vector<uint32_t>>(n);
        for (std::size_t t = 0; t < n; ++t) (*v)[t] = static_cast<uint32_t>(t);
        v_ = std::move(v);
    }
    TimeList& operator=(const std::vector<uint32_t>& v) {
        v_ = std::make_shared<std::vector<uint32_t>>(v);
        return *this;
    }
    void share_with(const TimeList& o) { v_ = o.v_; }

private:
    static const std::vector<uint32_t>& empty_vec() {
        static const std::vector<uint32_t> e;
        return e;
    }
    std::shared_ptr<const std::vector<uint32_t>> v_;
};

struct Tcl4Instance {
    SystemDesc sys;
    const double2* gamma = nullptr;  // [nf][Nt] (column-major Nt x nf)
    bool gamma_on_device = false;
    std::size_t Nt = 0;
    double dt = 0.0;
    TimeList tidx;                   // explicit list of requested time indices
    void* out = nullptr;             // [T][N^2 x N^2] complex (FP64: double2, FP32: float2)
    bool out_on_device = false;
    bool internal = false;           // buffers allocated by the library itself (not re-checked)
};

// Launch schedule of the F/C/R passes for one FFT length and precision.
struct Tuning {
    int col_tile = 4096;                        // elements per column-pass tile
    int row_tile = 2048;                        // elements per row-pass tile
    std::size_t chunk_bytes = std::size_t(48) << 20;  // Z/W scratch per chunk of triples
    int inv_dft_rows = 0;  // pruned inverse column DFT up to this many rows (0: the column FFT always;
                           // measured slower than the FFT at 10 and 16 rows, in both precisions)
    int cluster_lm = 0;  // log2 points per CTA of the cluster path (0: multi-pass path, -1: automatic)
    int enabled = 1;     // 3 * 2^k and 5 * 2^k lengths: 0 removes the length from the causal rule's choice
};
void set_tuning(int L, bool fp32, const Tuning& t);
// Transient device memory one group of a build may use (0: 45% of the free memory, at
// most 64 GiB); an instance above it is processed in slices of its frequency triples.
void set_work_budget(std::size_t bytes);
// The fused F/C/R path (one CTA per triple and half, the transforms in shared memory) for the
// FFT lengths it fits; off: the four-step passes and the scan kernels for every length.
void set_fused_conv(bool on);
bool fused_conv();
// Frees the calling thread's grow-only transient buffers on the current device (after its
// streams finish); the next build allocates them again.
void release_workspace();
// FFT length of the F/C/R convolutions for n_in consumed samples, and its schedule key
// (the tuning-table key: log2 for powers of two, + 64 for 3 * 2^k, + 128 for 5 * 2^k).
std::size_t fft_length_for(std::size_t n_in, bool fp32, bool causal, std::size_t pad_factor, int* key);
Tuning get_tuning(int L, bool fp32);
void clear_tuning();

struct BuildOptions {
    bool fp32 = false;
    bool causal_truncation = false;  // FFT length from max(tidx)+1 instead of Nt
    std::size_t pad_factor = 0;      // Nfft = next_pow2(max(2 n - 1, pad * n))
    double* fcr_ms = nullptr;        // device time of the F/C/R stage
    // Called with a stream ordered after a group's contraction, which has written the rows
    // [T][E] of the whole (unsliced) instances it lists -- each with the device address of its
    // rows, the output itself or its staging for a host output -- and before any of those rows
    // is downloaded (the downloads follow on that stream).  A build lists every instance at
    // most once and has finished the hook's work when it returns.  Plans ignore it.
    std::function<void(const std::vector<std::pair<const Tcl4Instance*, void*>>&, cudaStream_t)> out_hook;
};

// Full L4 builds (build_TCL4_generator_cuda_fused[_batch]) for a set of instances.  In the
// FP32 form the precision guard (guard.cu) recomputes in FP64 the leading times at which
// the FP32 result misses the guard's tolerance.
void tcl4_build(std::vector<Tcl4Instance>& insts, const BuildOptions& opt, cudaStream_t stream);
// The same without the guard (one pass in the requested precision).
void tcl4_build_direct(std::vector<Tcl4Instance>& insts, const BuildOptions& opt, cudaStream_t stream);

// Prepared batched build: metadata resident on the device, launch sequence captured in a
// CUDA graph; execute replays it (stream-ordered, no host work).
struct Tcl4Plan;
Tcl4Plan* plan_create(std::vector<Tcl4Instance>& insts, const BuildOptions& opt);
// ext_work (optional): a caller's device buffer of ext_cap bytes for the plan's transient
// arrays, shared with plans that run one after another on the same stream.
// budget (optional, with ext_work): the group budget the plan's units are packed by.
Tcl4Plan* plan_create_direct(std::vector<Tcl4Instance>& insts, const BuildOptions& opt, void* ext_work = nullptr,
                             std::size_t ext_cap = 0, std::size_t budget = 0);
// Transient bytes a plan of these instances would allocate under the group budget.
std::size_t plan_work_bytes(std::vector<Tcl4Instance>& insts, const BuildOptions& opt, std::size_t budget);
// The group budget of a build started now (set, or the share of the free memory).
std::size_t work_budget_now();
// Frees the calling thread's precision-guard buffers on the current device.
void release_guard_scratch();
// Work enqueued on every execute before the plan's graph (`pre`, may be empty) and after it
// (`tail`), on the execute's stream; each owns what it captures.
void plan_set_tail(Tcl4Plan* plan, std::function<void(cudaStream_t)> pre, std::function<void(cudaStream_t)> tail,
                   uint64_t kernels);
void plan_execute(Tcl4Plan* plan, cudaStream_t stream);
void plan_destroy(Tcl4Plan* plan);
uint64_t plan_kernels(const Tcl4Plan* plan);

// L4 build of one instance with every scratch buffer in a fixed file-scope device array
// (noalloc.cu); gamma and out are device pointers.
// Precision guard of the FP32 form: the largest relative FP32-vs-FP64 error accepted on the
// checked window (0: off).
void set_fp32_guard(double tol);
double fp32_guard();
// Bytes of FP64 head rows the guard builds and patches at a time (0: the default, 1 GiB).
void set_guard_chunk_bytes(std::size_t bytes);
// What the guard did in the calling thread's last FP32 build or plan creation.
struct GuardStats {
    uint64_t instances = 0;  // instances of the call
    uint64_t heads = 0;      // instances whose leading times were rebuilt in FP64
    uint64_t head_rows = 0;  // requested times rebuilt in FP64
    uint64_t rows = 0;       // requested times of the instances with a head
    uint64_t full = 0;       // instances rebuilt in FP64 entirely
    uint64_t rounds = 0;     // head-growth rounds
};
GuardStats fp32_guard_stats();

void noalloc_tcl4_build(const SystemDesc& sys, const double2* gamma, std::size_t Nt, double dt,
                        const std::vector<uint32_t>& tidx, bool fp32, std::size_t pad_factor, void* out,
                        cudaStream_t stream);

// TCL2 generator at the requested times (tcl2.cu); gamma and out are device pointers.
void tcl2_series_device(const SystemDesc& sys, const double* eps, const double2* gamma, std::size_t Nt,
                        const std::vector<uint32_t>& tidx, double2* out, cudaStream_t st);
// Trapezoid Gamma(w_b, t_k) for all buckets: C [N] and G [nb][N] are device pointers.
struct GammaRequest {
    const double2* C = nullptr;
    std::size_t N = 0;
    double dt = 0.0;
    std::vector<double> omegas;
    double2* G = nullptr;
};
// Many requests in one pair of launches.
void gamma_trapz_batch_device(const std::vector<GammaRequest>& reqs, cudaStream_t st);
void gamma_trapz_device(const double2* C, std::size_t N, double dt, const std::vector<double>& omegas, double2* G,
                        cudaStream_t st);

// The unfused stages (mikx_gw.cu), batched over T times; all pointers are device pointers.
void mikx_device(const double2* F, const double2* C, const double2* R, const int* p2f_dev, int N, int nf, std::size_t T,
                 double2* M, double2* I, double2* K, double2* X, cudaStream_t st);
void gw_device(const double2* M, const double2* I, const double2* K, const double2* X, const double2* ops_dev, int N,
               int num_ops, std::size_t T, bool symmetrize, double2* GW, double2* tmp, cudaStream_t st);
void gw_to_l4_device(const double2* GW, int N, std::size_t T, double2* L4, cudaStream_t st);

// dst[k] += src[k] (complex64 into complex128), n entries, device pointers.
void add_c64_into_c128(const float2* src, double2* dst, std::size_t n, cudaStream_t st);

// compute_triple_kernels for many instances (device buffers): full F/C/R series [nf^3][Nt]
// (FP64) of each.
struct FcrRequest {
    SystemDesc sys;
    const double2* gamma = nullptr;  // device [nf][Nt]
    std::size_t Nt = 0;
    double dt = 0.0;
    double2 *F = nullptr, *C = nullptr, *R = nullptr;  // device [nf^3][Nt]
};
void triple_kernels_batch(const std::vector<FcrRequest>& reqs, const BuildOptions& opt, cudaStream_t stream);

// compute_triple_kernels: full F/C/R series [nf^3][Nt] (FP64) for one instance.
void triple_kernels(const SystemDesc& sys, const double2* gamma, bool gamma_on_device, std::size_t Nt,
                    double dt, double2* F, double2* Cc, double2* R, bool out_on_device,
                    const BuildOptions& opt, cudaStream_t stream);

struct Rk4Request {
    const void* L = nullptr;       // [steps+1][D x D]
    const void* L_half = nullptr;  // [steps][D x D] or nullptr
    const void* L_add = nullptr;   // [steps+1][D x D] or nullptr
    bool fp32_storage = false;     // L, L_half, L_add are complex64 when true
    std::size_t steps = 0;
    int D = 0;
    double dt = 0.0;
    double2* r = nullptr;          // [D]
    std::size_t sample_every = 0;
    double2* samples = nullptr;    // [n_samples][D]
    const double2* obs = nullptr;  // [D]
    double2* obs_out = nullptr;    // [n_samples]
};

// RK4 propagation; all pointers are device pointers.  Requests with equal D and storage
// type run in one launch.
void rk4_propagate_device(const std::vector<Rk4Request>& reqs, cudaStream_t stream);

std::size_t rk4_num_samples(std::size_t steps, std::size_t sample_every);

// ----------------------------------------------------------------- bath ---
// bcf_fft_fun (correlation_fft.hpp:153-214) on the device (bcf.cu); out is a device pointer.
struct BcfRequest {
    int model = 0;   // 0: Ohmic, 1: Ohmic + Drude-Lorentz
    int which = 0;   // 0: C(t); 1: dC/dalpha; 2: dC/domega_c; 3: dC/dbeta
    double alpha = 0.0, omega_c = 1.0, lambda = 0.0, gamma = 1.0, beta = 1.0;
    std::size_t N = 0;  // grid: N + 1 samples
    double dt = 0.0;
    double2* out = nullptr;
    std::size_t n_out = 0;
};
std::size_t bcf_nfft(std::size_t N);
void bcf_device(const std::vector<BcfRequest>& reqs, cudaStream_t st);

// ------------------------------------------------------------- adjoints ---
// (adjoint.cu) Real losses; G(z) = dloss/dRe z + i dloss/dIm z.  Device pointers unless noted.
struct Rk4GradJob {
    const double2* L = nullptr;      // [steps+1][D x D] column-major
    const double2* L_add = nullptr;  // optional, added to L (its gradient equals L_bar)
    std::size_t steps = 0;
    int D = 0;
    double dt = 0.0;
    const double2* r0 = nullptr;     // [D]
    const double2* obs = nullptr;    // [D]: <O> = sum_l obs_l r_l
    std::size_t sample_every = 0;
    double2* ckpt = nullptr;         // [rk4_num_checkpoints(steps, every)][D]
    double2* obs_out = nullptr;      // forward: [rk4_num_samples] samples of <O>
    double2* r_out = nullptr;        // forward: final state
    const double2* obs_bar = nullptr;      // adjoint: G(<O>) per sample
    const double2* r_final_bar = nullptr;  // adjoint: G(final state), optional
    double2* L_bar = nullptr;        // adjoint out: [steps+1][D x D]
    double2* r0_bar = nullptr;       // adjoint out: [D]
    double2* obs_vec_bar = nullptr;  // adjoint out: [D]
};
std::size_t rk4_num_checkpoints(std::size_t steps, std::size_t every);
void rk4_forward_checkpointed(const std::vector<Rk4GradJob>& jobs, std::size_t every, cudaStream_t st);
void rk4_adjoint(const std::vector<Rk4GradJob>& jobs, std::size_t every, cudaStream_t st);

// L4 adjoint through the MIKX/GW map and the F/C/R kernels of one instance.
struct Tcl4AdjointJob {
    const SystemDesc* sys = nullptr;
    const double2* gamma = nullptr;   // [nf][T]
    std::size_t T = 0;
    double dt = 0.0;
    const double2* L_bar = nullptr;   // [T][N^4]
    const double2* F = nullptr;       // [nf^3][T] forward sources (needed for ops_bar)
    const double2* C = nullptr;
    const double2* R = nullptr;
    double2* gamma_bar = nullptr;     // [nf][T], accumulated
    double* omega_bar = nullptr;      // host [nf], accumulated (nullable)
    double2* ops_bar = nullptr;       // host [num_ops][N x N], accumulated (nullable)
};
void tcl4_adjoint(const std::vector<Tcl4AdjointJob>& jobs, cudaStream_t st);

// TCL2 adjoint: L2(t) = L0 + sum_b 2 Re Gamma_b(t) D_b + Im Gamma_b(t) U_b.
struct Tcl2AdjointJob {
    const SystemDesc* sys = nullptr;
    const double* eps = nullptr;      // host [N]
    const double2* gamma = nullptr;   // [nf][T]
    std::size_t T = 0;
    const double2* L_bar = nullptr;   // [T][N^4]
    double2* gamma_bar = nullptr;     // [nf][T], accumulated
    double2* ops_bar = nullptr;       // host, accumulated (nullable)
    double* eps_bar = nullptr;        // host [N], accumulated (nullable)
};
void tcl2_adjoint(const std::vector<Tcl2AdjointJob>& jobs, cudaStream_t st);
// Host maps of the TCL2 generator (tcl2.cu) and the reverse of their construction.
void tcl2_maps(const SystemDesc& s, const double* eps, std::vector<double2>& L0, std::vector<double2>& Db,
               std::vector<double2>& Ub);
void tcl2_maps_grad(const SystemDesc& s, const double* eps, const std::vector<double2>& GL0,
                    const std::vector<double2>& GD, const std::vector<double2>& GU, double2* ops_bar, double* eps_bar);

struct InnerRequest {
    const double2* a = nullptr;
    const double2* b = nullptr;
    std::size_t n = 0;
};
// out[k] = sum_i Re(conj(a_i) b_i) (host out)
void inner_re_device(const std::vector<InnerRequest>& reqs, double* out, cudaStream_t st);

// Mirror map of cpp/src/tcl/tcl4.cpp:40-101.
void build_mirror(const std::vector<double>& omegas, double tol, std::vector<int>& mirror, int* zero_index);

// Per-host-thread CUDA stream of the current device (created on first use).
cudaStream_t default_stream();

// Kernel accounting: every launch increments a process-wide counter; when profiling is
// on, each launch is bracketed by CUDA events and its device time is accumulated per
// kernel name after the call's final synchronisation.
uint64_t kernel_launches();
// Raises a kernel's dynamic shared-memory limit to at least `bytes` (per device).  The
// limit only grows: launches prepared earlier, and replayed later from a captured graph,
// keep the room they were prepared with.
void raise_smem_limit(const void* kernel, std::size_t bytes);
// Adds n to the process-wide launch counter (kernels launched outside engine.cu).
void count_launches(uint64_t n);
// Host phase times of the build calls: with TACO_TRACE_HOST set in the environment each
// tcl4_build prints, on stderr, the milliseconds its host thread spent in each phase
// (argument conversion, metadata derivation, preparation, waits).  Diagnostic only.
bool host_trace_on();
void host_trace_add(const char* phase, double ms);
// Checks the launch just issued and counts it.
inline void launched(const char* what) {
    cuda_check(cudaGetLastError(), what);
    count_launches(1);
}
void profile_enable(bool on);
void profile_reset();
struct ProfileEntry {
    const char* name;
    uint64_t launches;
    double total_ms;
};
std::vector<ProfileEntry> profile_entries();

}  // namespace taco
