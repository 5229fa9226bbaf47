// engine.cu -- host orchestration of the TCL4 device path.
//
// Per call: validate, derive per-instance metadata (requested-time maps, FFT length,
// merged GW coefficient table), group instances with equal FFT length, and run
//   spectra (2 nf per instance) -> per-triple B1/B2/B3 chain in chunks -> scans and
//   F/C/R assembly -> fused MIKX/GW/L4 contraction,
// all on one stream.  Device memory comes from a per-thread, per-device arena that
// grows on demand and is reused across calls (like the reference's thread-local fused
// workspace, cpp/src/backend/cuda/tcl4_fused_cuda.cu:676-685).
#include "engine.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <cmath>
#include <mutex>
#include <string>
#include <cstring>
#include <cstdint>
#include <limits>
#include <map>
#include <memory>
#include <unordered_map>
#include <thread>
#include <exception>

#include "cluster_conv.cuh"
#include "contract.cuh"
#include "fcr_kernels.cuh"
#include "fused_conv.cuh"
#include "gw_coef.hpp"
#include "rk4.cuh"

namespace taco {

namespace {

std::atomic<uint64_t> g_launches{0};
std::atomic<bool> g_profile{false};

std::mutex g_tune_mu;
std::map<std::pair<int, int>, Tuning> g_tune;  // (L, fp32) -> schedule set by the autotuner

Tuning tuning_for(int L, bool fp32) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find({L, fp32 ? 1 : 0});
    if (it != g_tune.end()) return it->second;
    return Tuning{};
}

std::size_t align_up(std::size_t x, std::size_t a) { return (x + a - 1) / a * a; }

// Host phase accumulator of the calling thread (see host_trace_on).
struct HostPhases {
    std::vector<std::pair<const char*, double>> ms;
    void add(const char* phase, double v) {
        for (auto& e : ms)
            if (std::strcmp(e.first, phase) == 0) {
                e.second += v;
                return;
            }
        ms.emplace_back(phase, v);
    }
};
thread_local HostPhases t_phases;

// Milliseconds since the previous lap, added to `phase` when tracing is on.
struct Lap {
    bool on = host_trace_on();
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    void operator()(const char* phase) {
        if (!on) return;
        const auto now = std::chrono::steady_clock::now();
        t_phases.add(phase, std::chrono::duration<double, std::milli>(now - t).count());
        t = now;
    }
};

struct DeviceBuffer {
    void* p = nullptr;
    std::size_t cap = 0;
    bool owned = true;  // false: a caller's buffer lent to a plan (never grown or freed here)
    void release() {
        if (p && owned) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    // grow-only with 1/8 slack (transient buffers reused by later calls); exact: a plan's
    // buffer, sized once
    void ensure(std::size_t bytes, bool exact = false) {
        if (bytes <= cap) return;
        if (!owned) throw Error(kRuntime, "shared work buffer smaller than the build needs");
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const std::size_t want = align_up(exact ? bytes : bytes + bytes / 8, std::size_t(1) << 20);
        const cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            p = nullptr;
            std::size_t fr = 0, tot = 0;
            (void)cudaGetLastError();
            cudaMemGetInfo(&fr, &tot);
            throw Error(kCuda, "cudaMalloc(workspace): " + std::string(cudaGetErrorString(e)) + " (" +
                                   std::to_string(want >> 20) + " MiB requested, " + std::to_string(fr >> 20) +
                                   " MiB free)");
        }
        cap = want;
    }
    ~DeviceBuffer() {
        if (p && owned) cudaFree(p);
    }
};

struct PinnedBuffer {
    void* p = nullptr;
    std::size_t cap = 0;
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
    void ensure(std::size_t bytes) {
        if (bytes <= cap) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        const std::size_t want = align_up(bytes + bytes / 8, std::size_t(1) << 16);
        cuda_check(cudaMallocHost(&p, want), "cudaMallocHost(staging)");
        cap = want;
    }
    ~PinnedBuffer() {
        if (p) cudaFreeHost(p);
    }
};

// Bump layout over one buffer: first a measuring pass (base == nullptr), then the real one.
struct Layout {
    char* base = nullptr;
    std::size_t off = 0;
    template <class T>
    T* take(std::size_t count) {
        off = align_up(off, 256);
        T* r = reinterpret_cast<T*>(base ? base + off : nullptr);
        off += count * sizeof(T);
        return r;
    }
};

struct PlanTables {
    DeviceBuffer buf;
    int L = 0, L1 = 0, L2 = 0, s = 0, R = 1;
};

// FFT lengths Nfft = R * 2^L with R in {1, 3, 5}.  The key names a length in the plan and
// tuning tables: L for powers of two, L + 64 (R = 3), L + 128 (R = 5).
int odd_index(int R) { return R == 3 ? 1 : (R == 5 ? 2 : 0); }
int size_key(int L, int R) { return L + 64 * odd_index(R); }

// Four-step split: N2 = 2^L2 rows of the row pass, N1 = R * 2^L1 points per column, with
// N2 the smallest power of two >= sqrt(Nfft) for the mixed lengths (L2 = ceil(L/2) else).
void fft_split(int L, int R, int& L1, int& L2) {
    if (R == 1) {
        L2 = (L + 1) / 2;
    } else {
        const double lg = L + std::log2(static_cast<double>(R));
        L2 = static_cast<int>(std::ceil(lg / 2.0));
    }
    L1 = L - L2;
}

struct Workspace {
    int device = -1;
    cudaStream_t stream = nullptr;
    DeviceBuffer arena;  // metadata of the running group
    DeviceBuffer work;   // transient arrays of the running group
    PinnedBuffer staging;
    // further lanes of pipelined direct builds: their own streams and buffers
    struct ExtraLane {
        cudaStream_t s = nullptr;
        DeviceBuffer arena, work;
        PinnedBuffer staging;
    };
    ExtraLane extra[2];
    // per sub-batch buffers of pipelined direct builds (metadata, staged host input, pinned
    // staging, upload event) and the stream that carries every upload of such a build
    struct SubBuffers {
        DeviceBuffer arena, input;
        PinnedBuffer staging;
        cudaEvent_t uploaded = nullptr, done = nullptr;
        ~SubBuffers() {
            if (uploaded) cudaEventDestroy(uploaded);
            if (done) cudaEventDestroy(done);
        }
    };
    std::vector<std::unique_ptr<SubBuffers>> sub_bufs;
    cudaStream_t upload = nullptr;
    // the download side of each lane of pipelined direct builds: staged host outputs (reused
    // by the lane's next sub-batch once `done`), and the stream that carries their copies, so
    // that the lane's next kernels do not queue behind them
    struct Download {
        DeviceBuffer out;
        cudaStream_t s = nullptr;
        cudaEvent_t contracted = nullptr, done = nullptr;
        ~Download() {
            if (contracted) cudaEventDestroy(contracted);
            if (done) cudaEventDestroy(done);
            if (s) cudaStreamDestroy(s);
        }
    };
    Download down[3];
    std::map<std::pair<int, int>, std::unique_ptr<PlanTables>> plans;  // (L, fp32)
    std::map<std::pair<int, int>, std::unique_ptr<DeviceBuffer>> fz_tables;  // (N, fp32): fused-path roots
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~Workspace() {
        plans.clear();
        fz_tables.clear();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (auto& l : extra)
            if (l.s) cudaStreamDestroy(l.s);
        sub_bufs.clear();
        if (upload) cudaStreamDestroy(upload);
        if (stream) cudaStreamDestroy(stream);
    }
};

Workspace& workspace() {
    thread_local std::unordered_map<int, std::unique_ptr<Workspace>> tl;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    auto& w = tl[dev];
    if (!w) {
        w = std::make_unique<Workspace>();
        w->device = dev;
        cuda_check(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        cuda_check(cudaEventCreate(&w->ev0), "cudaEventCreate");
        cuda_check(cudaEventCreate(&w->ev1), "cudaEventCreate");
    }
    return *w;
}

template <class C>
__global__ void k_fill_twiddle(C* out, uint32_t count, double denom) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= count) return;
    double s, c;
    sincospi(-2.0 * static_cast<double>(m) / denom, &s, &c);
    out[m] = from_d2<C>(make_double2(c, s));
}

template <class R>
FftPlan<cplx_t<R>> get_plan(Workspace& ws, int L, int Rf, cudaStream_t st) {
    using C = cplx_t<R>;
    const bool fp32 = std::is_same<R, float>::value;
    auto& slot = ws.plans[{size_key(L, Rf), fp32 ? 1 : 0}];
    if (!slot) {
        auto pt = std::make_unique<PlanTables>();
        pt->L = L;
        pt->R = Rf;
        fft_split(L, Rf, pt->L1, pt->L2);
        pt->s = (L + 1) / 2;
        const std::size_t N = static_cast<std::size_t>(Rf) << L, N1 = static_cast<std::size_t>(Rf) << pt->L1,
                          N2 = std::size_t(1) << pt->L2;
        const std::size_t nc = N >> pt->s, nfine = std::size_t(1) << pt->s;
        pt->buf.ensure((N1 + N2 + nc + nfine) * sizeof(C) + 4 * 256);
        Layout lay{static_cast<char*>(pt->buf.p)};
        C* tw1 = lay.take<C>(N1);
        C* tw2 = lay.take<C>(N2);
        C* twc = lay.take<C>(nc);
        C* twf = lay.take<C>(nfine);
        auto fill = [&](C* p, std::size_t count, double denom) {
            k_fill_twiddle<C><<<static_cast<unsigned>((count + 255) / 256), 256, 0, st>>>(p, static_cast<uint32_t>(count), denom);
            cuda_check(cudaGetLastError(), "k_fill_twiddle");
            g_launches.fetch_add(1);
        };
        fill(tw1, N1, static_cast<double>(N1));
        fill(tw2, N2, static_cast<double>(N2));
        fill(twc, nc, static_cast<double>(nc));
        fill(twf, nfine, static_cast<double>(N));
        // kernels on other streams (pipelined lanes) read the tables: complete them first
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(twiddles)");
        slot = std::move(pt);
    }
    const PlanTables& pt = *slot;
    const std::size_t N = static_cast<std::size_t>(Rf) << L, N1 = static_cast<std::size_t>(Rf) << pt.L1,
                      N2 = std::size_t(1) << pt.L2;
    Layout lay{static_cast<char*>(pt.buf.p)};
    FftPlan<C> p;
    p.L = L;
    p.L1 = pt.L1;
    p.L2 = pt.L2;
    p.s = pt.s;
    p.R = Rf;
    p.tw1 = lay.take<C>(N1);
    p.tw2 = lay.take<C>(N2);
    p.twc = lay.take<C>(N >> pt.s);
    p.twf = lay.take<C>(std::size_t(1) << pt.s);
    return p;
}

// Fused-path plan of length N: its stage list and the table of N-th roots.
std::atomic<int> g_fused{0};

template <class R>
FzPlan<cplx_t<R>> get_fz_plan(Workspace& ws, int N, cudaStream_t st) {
    using C = cplx_t<R>;
    const bool fp32 = std::is_same<R, float>::value;
    FzPlan<C> p{};
    p.N = N;
    if (!fz_stages(N, fp32 ? 16 : 8, p.rad, p.nst)) throw Error(kRuntime, "fused path: unsupported FFT length");
    const std::size_t entries = fz_table_layout(p);
    auto& slot = ws.fz_tables[{N, fp32 ? 1 : 0}];
    if (!slot) {
        auto buf = std::make_unique<DeviceBuffer>();
        buf->ensure(std::max<std::size_t>(1, entries) * sizeof(C));
        k_fz_fill_tables<C><<<static_cast<unsigned>((entries + 255) / 256 + 1), 256, 0, st>>>(
            static_cast<C*>(buf->p), p, static_cast<uint32_t>(entries));
        cuda_check(cudaGetLastError(), "k_fz_fill_tables");
        g_launches.fetch_add(1);
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(twiddles)");
        slot = std::move(buf);
    }
    p.tw = static_cast<const C*>(slot->p);
    return p;
}

// Whether a group of FFT length N runs the fused path: its working array and the scan
// scratch fit one CTA's shared memory, and the stage list exists.
template <class R>
bool fused_fits(std::size_t N) {
    using C = cplx_t<R>;
    if (!g_fused.load() || N > (std::size_t(1) << 16)) return false;
    int rad[FZ_MAX_STAGES], nst = 0;
    if (!fz_stages(static_cast<int>(N), std::is_same<R, float>::value ? 16 : 8, rad, nst)) return false;
    return fz_smem<C>(static_cast<int>(N)) <= 227 * 1024;
}

// Tables of the cluster path: M-point twiddles and the N-point coarse/fine tables.
template <class R>
ClusterPlan<cplx_t<R>> get_cluster_plan(Workspace& ws, int L, int LM, cudaStream_t st) {
    using C = cplx_t<R>;
    const bool fp32 = std::is_same<R, float>::value;
    auto& slot = ws.plans[{L + 64 * (LM + 1), fp32 ? 1 : 0}];
    const int s = (L + 1) / 2;
    const std::size_t N = std::size_t(1) << L, M = std::size_t(1) << LM;
    const std::size_t nc = N >> s, nfine = std::size_t(1) << s;
    if (!slot) {
        auto pt = std::make_unique<PlanTables>();
        pt->buf.ensure((M + nc + nfine) * sizeof(C) + 3 * 256);
        Layout lay{static_cast<char*>(pt->buf.p)};
        C* twM = lay.take<C>(M);
        C* twc = lay.take<C>(nc);
        C* twf = lay.take<C>(nfine);
        auto fill = [&](C* p, std::size_t count, double denom) {
            k_fill_twiddle<C><<<static_cast<unsigned>((count + 255) / 256), 256, 0, st>>>(p, static_cast<uint32_t>(count), denom);
            cuda_check(cudaGetLastError(), "k_fill_twiddle");
            g_launches.fetch_add(1);
        };
        fill(twM, M, static_cast<double>(M));
        fill(twc, nc, static_cast<double>(nc));
        fill(twf, nfine, static_cast<double>(N));
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(twiddles)");
        slot = std::move(pt);
    }
    Layout lay{static_cast<char*>(slot->buf.p)};
    ClusterPlan<C> p;
    p.LN = L;
    p.LM = LM;
    p.s = s;
    p.twM = lay.take<C>(M);
    p.twc = lay.take<C>(nc);
    p.twf = lay.take<C>(nfine);
    return p;
}

template <class R, int KLOG>
void launch_cluster_k(const ClusterJob* jobs, std::size_t njobs, const ClusterPlan<cplx_t<R>>& plan, std::size_t smem,
                      cudaStream_t st) {
    cuda_check(cudaFuncSetAttribute(k_conv_cluster<R, KLOG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem)),
               "cudaFuncSetAttribute(cluster smem)");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(njobs << KLOG), 1, 1);
    cfg.blockDim = dim3(static_cast<unsigned>((1u << plan.LM) / 8), 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1u << KLOG;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cuda_check(cudaLaunchKernelEx(&cfg, k_conv_cluster<R, KLOG>, jobs, plan), "cudaLaunchKernelEx(k_conv_cluster)");
}

template <class R>
void launch_cluster(const ClusterJob* jobs, std::size_t njobs, const ClusterPlan<cplx_t<R>>& plan, cudaStream_t st) {
    using C = cplx_t<R>;
    const std::size_t smem = 2 * static_cast<std::size_t>(padded_size<C>(1 << plan.LM)) * sizeof(C);
    switch (plan.LN - plan.LM) {
        case 0: launch_cluster_k<R, 0>(jobs, njobs, plan, smem, st); break;
        case 1: launch_cluster_k<R, 1>(jobs, njobs, plan, smem, st); break;
        case 2: launch_cluster_k<R, 2>(jobs, njobs, plan, smem, st); break;
        case 3: launch_cluster_k<R, 3>(jobs, njobs, plan, smem, st); break;
        default: throw Error(kInvalidArgument, "cluster path: at most 8 CTAs per cluster");
    }
}

// Points per CTA of the cluster path for FFT length 2^L, or -1 when the multi-pass path runs.
int cluster_lm_for(int L, bool fp32, const Tuning& t) {
    const int lm_max = fp32 ? 13 : 12;  // 1024 / 512 threads, two padded tiles in shared memory
    if (t.cluster_lm == 0) return -1;
    int lm = t.cluster_lm > 0 ? std::min(t.cluster_lm, lm_max) : std::min(L, lm_max);
    lm = std::min(lm, L);
    if (lm < 3 || L - lm > 3) return -1;
    return lm;
}

template <class K>
void set_smem(K kernel, std::size_t bytes) {
    raise_smem_limit(reinterpret_cast<const void*>(kernel), bytes);
}

// FFT pass kernels with compile-time sizes for (log2 pass length, log2 tile count) with
// pass length 2^7..2^10 and tiles of 2^10..2^12 elements (FFT lengths 2^14..2^20 under
// the default and tuned schedules); the runtime-size kernels otherwise.
template <class R>
using ColFn = void (*)(const ColJob*, FftPlan<cplx_t<R>>, int);
template <class R>
using RowFn = void (*)(const RowJob*, FftPlan<cplx_t<R>>, int);
template <class R>
using InvFn = void (*)(const InvJob*, FftPlan<cplx_t<R>>, int);

#define TACO_CT_CASES(X) \
    X(4, 5) X(5, 4) X(5, 5) X(5, 6) X(6, 5) X(6, 6) \
    X(7, 3) X(7, 4) X(7, 5) X(8, 2) X(8, 3) X(8, 4) X(9, 1) X(9, 2) X(9, 3) X(10, 0) X(10, 1) X(10, 2)

// Column kernels of the mixed lengths N1 = R * 2^l for the tile widths the default and
// tuned schedules produce.
#define TACO_MX_CASES(X) \
    X(5, 4, 3) X(5, 4, 4) X(5, 4, 5) X(5, 5, 3) X(5, 5, 4) X(3, 5, 3) X(3, 5, 4) X(3, 5, 5) X(3, 4, 4) X(3, 4, 5)

bool mixed_column_kernels(int r, int l, int c) {
    switch (r * 256 + l * 16 + c) {
#define X(a, b, d) case a * 256 + b * 16 + d: return true;
        TACO_MX_CASES(X)
#undef X
        default: return false;
    }
}

template <class R>
ColFn<R> fwd_col_fn(int r, int l, int c) {
    if (r > 1) {
        switch (r * 256 + l * 16 + c) {
#define X(a, b, d) case a * 256 + b * 16 + d: return k_fwd_col_mx<R, a, b, d>;
            TACO_MX_CASES(X)
#undef X
            default: throw Error(kRuntime, "no column kernel for this mixed FFT length");
        }
    }
    switch (l * 16 + c) {
#define X(a, b) case a * 16 + b: return k_fwd_col_ct<R, a, b>;
        TACO_CT_CASES(X)
#undef X
        default: return k_fwd_col<R>;
    }
}

template <class R>
InvFn<R> inv_col_fn(int r, int l, int c) {
    if (r > 1) {
        switch (r * 256 + l * 16 + c) {
#define X(a, b, d) case a * 256 + b * 16 + d: return k_inv_col_mx<R, a, b, d>;
            TACO_MX_CASES(X)
#undef X
            default: throw Error(kRuntime, "no column kernel for this mixed FFT length");
        }
    }
    switch (l * 16 + c) {
#define X(a, b) case a * 16 + b: return k_inv_col_ct<R, a, b>;
        TACO_CT_CASES(X)
#undef X
        default: return k_inv_col<R>;
    }
}

template <class R>
RowFn<R> row_fn(int l, int c) {
    switch (l * 16 + c) {
#define X(a, b) case a * 16 + b: return k_row_ct<R, a, b>;
        TACO_CT_CASES(X)
#undef X
        default: return k_row<R>;
    }
}
#undef TACO_CT_CASES
#undef TACO_MX_CASES

struct ProfStore {
    std::mutex mu;
    std::map<std::string, std::pair<uint64_t, double>> acc;
    std::vector<std::string> order;
};
ProfStore& prof_store() {
    static ProfStore s;
    return s;
}

// Event pairs recorded around launches of one call; resolved after the final sync.
struct ProfRecorder {
    struct Rec {
        const char* name;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    cudaStream_t st = nullptr;
    const char* pending = nullptr;
    cudaEvent_t pend_a = nullptr;
    void before(const char* name) {
        if (!g_profile.load() || st == nullptr) return;
        cuda_check(cudaEventCreate(&pend_a), "cudaEventCreate(prof)");
        cuda_check(cudaEventRecord(pend_a, st), "cudaEventRecord(prof)");
        pending = name;
    }
    void after() {
        if (!pending) return;
        cudaEvent_t b;
        cuda_check(cudaEventCreate(&b), "cudaEventCreate(prof)");
        cuda_check(cudaEventRecord(b, st), "cudaEventRecord(prof)");
        recs.push_back({pending, pend_a, b});
        pending = nullptr;
    }
    void resolve() {
        if (recs.empty()) return;
        ProfStore& ps = prof_store();
        std::lock_guard<std::mutex> lk(ps.mu);
        for (auto& r : recs) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, r.a, r.b);
            auto it = ps.acc.find(r.name);
            if (it == ps.acc.end()) {
                ps.order.push_back(r.name);
                it = ps.acc.emplace(r.name, std::make_pair(uint64_t(0), 0.0)).first;
            }
            it->second.first += 1;
            it->second.second += ms;
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
        recs.clear();
    }
    ~ProfRecorder() {
        for (auto& r : recs) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
    }
};

void check_launch(const char* what, ProfRecorder* pr = nullptr) {
    cuda_check(cudaGetLastError(), what);
    g_launches.fetch_add(1);
    if (pr) pr->after();
}

// --------------------------------------------------------------- metadata --
// Maps of one list of requested times (shared by the instances of a call that name the
// same list): the unique times in increasing order and each request's position among them.
struct TimeMap {
    std::size_t T = 0, U = 0, t_count = 0;
    std::vector<int> tmap;        // [t_count] sample -> unique-time position, or -1
    std::vector<uint32_t> out_u;  // [T] request -> unique-time position
};

std::shared_ptr<const TimeMap> make_time_map(const TimeList& list) {
    auto m = std::make_shared<TimeMap>();
    const uint32_t* tidx = list.begin();
    m->T = list.size();
    uint32_t tmax = 0;
    bool increasing = true;
    for (std::size_t o = 0; o < m->T; ++o) {
        tmax = std::max(tmax, tidx[o]);
        if (o > 0 && tidx[o] <= tidx[o - 1]) increasing = false;
    }
    m->t_count = static_cast<std::size_t>(tmax) + 1;
    m->tmap.assign(m->t_count, -1);
    m->out_u.resize(m->T);
    if (increasing) {  // the unique times are the requested ones, in order
        m->U = m->T;
        for (std::size_t o = 0; o < m->T; ++o) {
            m->tmap[tidx[o]] = static_cast<int>(o);
            m->out_u[o] = static_cast<uint32_t>(o);
        }
    } else {
        std::vector<uint32_t> uniq(list.vec());
        std::sort(uniq.begin(), uniq.end());
        uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
        m->U = uniq.size();
        for (std::size_t u = 0; u < uniq.size(); ++u) m->tmap[uniq[u]] = static_cast<int>(u);
        for (std::size_t o = 0; o < m->T; ++o) m->out_u[o] = static_cast<uint32_t>(m->tmap[tidx[o]]);
    }
    return m;
}

struct InstMeta {
    std::size_t T = 0, U = 0, t_count = 0, n_in = 0;
    int L = 0, R = 1;  // FFT length R * 2^L
    std::shared_ptr<const TimeMap> times;   // tmap [t_count], out_u [T]
    std::shared_ptr<const CoefTable> coef;  // shared with the table cache (empty when unused)
};

// Coefficient tables by system content (N, nf, pair_to_freq, coupling operators): the
// table depends on nothing else, so repeated builds of the same systems (parameter sweeps
// over baths and times, repeated calls) skip the NAKZWAN walk.  Bounded by 2 GB in total;
// the cache is dropped when a new table would exceed the bound.
std::shared_ptr<const CoefTable> coef_table_for(const SystemDesc& s) {
    static std::mutex mu;
    static std::unordered_map<std::string, std::shared_ptr<const CoefTable>> cache;
    static std::size_t cached_bytes = 0;
    constexpr std::size_t kMaxBytes = std::size_t(2) << 30;
    std::string key;
    key.reserve(12 + s.p2f.size() * sizeof(int) + s.ops.size() * sizeof(double2));
    const int head[3] = {s.N, s.nf, s.num_ops};
    key.append(reinterpret_cast<const char*>(head), sizeof(head));
    key.append(reinterpret_cast<const char*>(s.p2f.data()), s.p2f.size() * sizeof(int));
    key.append(reinterpret_cast<const char*>(s.ops.data()), s.ops.size() * sizeof(double2));
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    auto t = std::make_shared<CoefTable>();
    build_coef_table(s.N, s.nf, s.p2f.data(), s.ops.data(), s.num_ops, *t);
    const std::size_t bytes = key.size() + t->rowptr.size() * 4 + t->src.size() * 4 + t->coef.size() * 16 +
                              t->triple_fc_used.size() + t->triple_r_used.size();
    std::lock_guard<std::mutex> lk(mu);
    if (cached_bytes + bytes > kMaxBytes) {
        cache.clear();
        cached_bytes = 0;
    }
    if (bytes <= kMaxBytes && cache.emplace(key, t).second) cached_bytes += bytes;
    return t;
}

// FFT length for a linear convolution of `target` outputs: the next power of two, or (when
// allowed: the causal rule) 3 * 2^k or 5 * 2^k if shorter and column kernels exist for
// the resulting split under the current schedule.
void choose_fft(std::size_t target, bool fp32, bool allow_mixed, int& L_out, int& R_out) {
    std::size_t nfft = std::max<std::size_t>(8, next_pow2(target));
    if (nfft > (std::size_t(1) << 22)) throw Error(kOverflow, "FFT length above 2^22 is not supported");
    L_out = ilog2(nfft);
    R_out = 1;
    if (!allow_mixed) return;
    for (int Rf : {5, 3}) {
        const std::size_t base = (target + Rf - 1) / Rf;
        const int L = std::max(3, ilog2(base));
        const std::size_t n = static_cast<std::size_t>(Rf) << L;
        if (n >= nfft || n < target) continue;
        const Tuning t = tuning_for(size_key(L, Rf), fp32);
        if (!t.enabled) continue;  // the autotuner measured a longer length faster
        if (fp32 ? fused_fits<float>(n) : fused_fits<double>(n)) {  // no column kernels needed
            nfft = n;
            L_out = L;
            R_out = Rf;
            continue;
        }
        int L1 = 0, L2 = 0;
        fft_split(L, Rf, L1, L2);
        if (L1 < 3) continue;
        const int log2c = fp32 ? geometry(FftPlan<float2>{L, L1, L2, 0, Rf, nullptr, nullptr, nullptr, nullptr},
                                          t.col_tile, t.row_tile).log2c
                               : geometry(FftPlan<double2>{L, L1, L2, 0, Rf, nullptr, nullptr, nullptr, nullptr},
                                          t.col_tile, t.row_tile).log2c;
        if (!mixed_column_kernels(Rf, L1, log2c)) continue;
        nfft = n;
        L_out = L;
        R_out = Rf;
    }
}

void derive_meta(const Tcl4Instance& in, const BuildOptions& opt, InstMeta& m, bool want_coef,
                 std::shared_ptr<const TimeMap> times = nullptr) {
    m.times = times ? std::move(times) : make_time_map(in.tidx);
    m.T = m.times->T;
    m.U = m.times->U;
    m.t_count = m.times->t_count;
    m.n_in = opt.causal_truncation ? m.t_count : in.Nt;
    std::size_t target = 2 * m.n_in - 1;
    if (opt.pad_factor > 0) target = std::max(target, opt.pad_factor * m.n_in);
    choose_fft(target, opt.fp32, opt.causal_truncation && opt.pad_factor == 0, m.L, m.R);
    static const std::shared_ptr<const CoefTable> kEmpty = std::make_shared<CoefTable>();
    m.coef = want_coef ? coef_table_for(in.sys) : kEmpty;
}

struct TripleRef {
    int unit;
    int tri;  // (i*nf + j)*nf + k
};

// A slice of one instance's triples, [lo, hi) of the nf^3, processed by one group.  The
// contraction uses the coefficients of the slice's sources only (local source index
// kind * (hi - lo) + (tri - lo)); every slice after an instance's first adds into its
// output, so an instance too large for one pass streams through device memory slice
// by slice.
struct WorkUnit {
    Tcl4Instance* in = nullptr;
    InstMeta* meta = nullptr;
    int lo = 0, hi = 0;
    bool accumulate = false;
    const CoefTable* coef = nullptr;
    std::shared_ptr<CoefTable> own;
    int nsub() const { return hi - lo; }
};

// Coefficients of the sources of triples [lo, hi), re-indexed to the slice.
std::shared_ptr<CoefTable> slice_table(const CoefTable& full, int lo, int hi) {
    auto t = std::make_shared<CoefTable>();
    const uint32_t nf3 = static_cast<uint32_t>(full.nf) * full.nf * full.nf;
    const uint32_t nsub = static_cast<uint32_t>(hi - lo);
    t->N = full.N;
    t->nf = full.nf;
    const std::size_t E = full.rowptr.size() - 1;
    t->rowptr.assign(E + 1, 0);
    for (std::size_t e = 0; e < E; ++e) {
        for (int32_t q = full.rowptr[e]; q < full.rowptr[e + 1]; ++q) {
            const uint32_t key = full.src[q], s = key & 0x7fffffffu;
            const uint32_t kind = s / nf3, tri = s % nf3;
            if (tri < static_cast<uint32_t>(lo) || tri >= static_cast<uint32_t>(hi)) continue;
            t->src.push_back((kind * nsub + (tri - lo)) | (key & 0x80000000u));
            t->coef.push_back(full.coef[q]);
        }
        t->rowptr[e + 1] = static_cast<int32_t>(t->src.size());
    }
    t->triple_fc_used.assign(full.triple_fc_used.begin() + lo, full.triple_fc_used.begin() + hi);
    t->triple_r_used.assign(full.triple_r_used.begin() + lo, full.triple_r_used.begin() + hi);
    return t;
}

// Launch geometry of one group (units with equal FFT length).
template <class R>
struct GroupGeom {
    int L = 0, Rf = 1;  // FFT length Rf * 2^L
    std::size_t Nfft = 0, ntri = 0, Q = 1, nchunks = 0, max_tcount = 0;
    Tuning tune;
    Geometry g;
    int clm = -1, inv_rows = 0, max_chunks = 0;
    bool use_cluster = false, inv_dft = false;
    bool fused = false;  // one CTA per (triple, half): transforms, scans and assembly in shared memory
};

template <class R>
GroupGeom<R> group_geom(const std::vector<WorkUnit*>& units) {
    using C = cplx_t<R>;
    GroupGeom<R> G;
    G.L = units[0]->meta->L;
    G.Rf = units[0]->meta->R;
    G.Nfft = static_cast<std::size_t>(G.Rf) << G.L;
    G.tune = tuning_for(size_key(G.L, G.Rf), std::is_same<R, float>::value);
    FftPlan<C> shape{};
    shape.L = G.L;
    shape.R = G.Rf;
    fft_split(G.L, G.Rf, shape.L1, shape.L2);
    G.g = geometry(shape, G.tune.col_tile, G.tune.row_tile);
    for (auto* u : units) G.ntri += static_cast<std::size_t>(u->nsub());
    G.clm = G.Rf == 1 ? cluster_lm_for(G.L, std::is_same<R, float>::value, G.tune) : -1;
    G.use_cluster = G.clm > 0;
    G.fused = !G.use_cluster && fused_fits<R>(G.Nfft);
    const std::size_t per_tri_scratch = 2 * G.Nfft * sizeof(C);
    G.Q = std::max<std::size_t>(1, G.tune.chunk_bytes / per_tri_scratch);
    G.Q = std::min<std::size_t>({G.Q, std::max<std::size_t>(1, G.ntri), 32767});
    G.nchunks = (G.ntri + G.Q - 1) / G.Q;
    for (auto* u : units) G.max_tcount = std::max(G.max_tcount, u->meta->t_count);
    const int N2 = 1 << shape.L2;
    G.inv_rows = static_cast<int>((G.max_tcount + N2 - 1) / N2);
    G.inv_dft = G.inv_rows <= std::min(G.tune.inv_dft_rows, INV_DFT_MAXR);
    G.max_chunks = static_cast<int>((G.max_tcount + SCAN_CHUNK - 1) / SCAN_CHUNK);
    return G;
}

// Transient device arrays of a group (reused by the next group): staged host gamma,
// spectra, convolution outputs, sources, staged host output, FFT scratch, scan partials.
template <class C>
struct WorkPtrs {
    std::vector<const double2*> gamma;
    std::vector<C*> spec, conv, v, out;
    C* scratch = nullptr;
    double* partial = nullptr;
};

template <class R>
void layout_work(const std::vector<WorkUnit*>& units, const GroupGeom<R>& G, bool fcr_only, bool fcr_out_dev,
                 Layout& lay, WorkPtrs<cplx_t<R>>& P, bool gamma_elsewhere = false, bool out_elsewhere = false) {
    using C = cplx_t<R>;
    const std::size_t ni = units.size();
    P.gamma.assign(ni, nullptr);
    P.spec.assign(ni, nullptr);
    P.conv.assign(ni, nullptr);
    P.v.assign(ni, nullptr);
    P.out.assign(ni, nullptr);
    for (std::size_t a = 0; a < ni; ++a) {
        const Tcl4Instance& in = *units[a]->in;
        const InstMeta& m = *units[a]->meta;
        const std::size_t nf = in.sys.nf, nsub = units[a]->nsub();
        if (!in.gamma_on_device && !gamma_elsewhere) P.gamma[a] = lay.take<double2>(nf * m.n_in);
        P.spec[a] = lay.take<C>(2 * nf * G.Nfft);
        if (!G.fused) P.conv[a] = lay.take<C>(nsub * 2 * m.t_count);
        if (!fcr_only) {
            P.v[a] = lay.take<C>(3 * nsub * m.U);
            if (!in.out_on_device && !out_elsewhere) {
                const std::size_t E = static_cast<std::size_t>(in.sys.N) * in.sys.N * in.sys.N * in.sys.N;
                P.out[a] = lay.take<C>(m.T * E);
            }
        } else if (!fcr_out_dev) {
            P.v[a] = lay.take<C>(3 * nsub * m.U);
        }
    }
    P.scratch = lay.take<C>(G.use_cluster || G.fused ? 1 : G.Q * 2 * G.Nfft);
    P.partial = lay.take<double>(G.fused ? 1 : std::max<std::size_t>(1, G.ntri) * G.max_chunks * SCAN_W);
}

template <class R>
std::size_t measure_work(const std::vector<WorkUnit*>& units, bool fcr_only, bool fcr_out_dev) {
    const GroupGeom<R> G = group_geom<R>(units);
    Layout meas;
    WorkPtrs<cplx_t<R>> P;
    layout_work<R>(units, G, fcr_only, fcr_out_dev, meas, P);
    return meas.off + 256;
}

// One group (units with equal FFT length): lays out its metadata in `meta_mem` and its
// transient arrays in `work_mem`, stages the small metadata and the host inputs
// (stream-ordered on `st`), and returns the closure that enqueues the group's kernels
// (and the D2H copies of host outputs) on a stream.  `fcr_out` (non-null) writes the
// F/C/R series (FP64) into caller buffers instead of running the contraction.
using Enqueue = std::function<void(cudaStream_t, ProfRecorder*, cudaEvent_t, cudaEvent_t)>;

template <class R>
Enqueue prepare_group(std::vector<WorkUnit*>& units, const BuildOptions& opt, cudaStream_t st, Workspace& ws,
                      DeviceBuffer& meta_mem, DeviceBuffer& work_mem, double2* const* fcr_out, bool fcr_out_dev,
                      PinnedBuffer* staging_buf = nullptr, DeviceBuffer* input_mem = nullptr,
                      cudaStream_t upload = nullptr, cudaEvent_t uploaded = nullptr,
                      Workspace::Download* down = nullptr) {
    using C = cplx_t<R>;
    const auto t_prep = std::chrono::steady_clock::now();
    const GroupGeom<R> G = group_geom<R>(units);
    const int L = G.L;
    const FftPlan<C> plan = get_plan<R>(ws, L, G.Rf, st);
    const Geometry g = G.g;
    const std::size_t Nfft = G.Nfft;
    const std::size_t ni = units.size();
    const bool fcr_only = (fcr_out != nullptr);
    std::vector<TripleRef> tris;
    for (std::size_t a = 0; a < ni; ++a)
        for (int t = units[a]->lo; t < units[a]->hi; ++t) tris.push_back({static_cast<int>(a), t});
    const std::size_t ntri = tris.size();
    const bool use_cluster = G.use_cluster;
    ClusterPlan<C> cplan{};
    if (use_cluster) cplan = get_cluster_plan<R>(ws, L, G.clm, st);
    const std::size_t Q = G.Q;
    const std::size_t nchunks = G.nchunks;
    const int N2 = 1 << plan.L2;
    const int inv_rows = G.inv_rows;
    const bool inv_dft = G.inv_dft;
    const int max_chunks = G.max_chunks;

    // ---- device layout: transient arrays in work_mem, metadata in meta_mem ----
    WorkPtrs<C> P;
    {
        // staged host gamma in `input_mem` when given (kept apart from the reused work arrays)
        const bool apart = input_mem != nullptr;
        const bool out_apart = down != nullptr && !fcr_only;
        Layout meas;
        layout_work<R>(units, G, fcr_only, fcr_out_dev, meas, P, apart, out_apart);
        work_mem.ensure(meas.off + 256);
        Layout lay{static_cast<char*>(work_mem.p)};
        layout_work<R>(units, G, fcr_only, fcr_out_dev, lay, P, apart, out_apart);
        if (out_apart) {
            // staged host outputs in the lane's download buffer
            Layout mo;
            for (auto* u : units)
                if (!u->in->out_on_device)
                    mo.take<C>(u->meta->T * static_cast<std::size_t>(u->in->sys.N) * u->in->sys.N * u->in->sys.N * u->in->sys.N);
            down->out.ensure(mo.off + 256);
            Layout lo{static_cast<char*>(down->out.p)};
            for (std::size_t a = 0; a < ni; ++a)
                if (!units[a]->in->out_on_device)
                    P.out[a] = lo.take<C>(units[a]->meta->T * static_cast<std::size_t>(units[a]->in->sys.N) *
                                          units[a]->in->sys.N * units[a]->in->sys.N * units[a]->in->sys.N);
        }
        if (apart) {
            Layout mi;
            for (auto* u : units)
                if (!u->in->gamma_on_device) mi.take<double2>(static_cast<std::size_t>(u->in->sys.nf) * u->meta->n_in);
            input_mem->ensure(mi.off + 256);
            Layout li{static_cast<char*>(input_mem->p)};
            for (std::size_t a = 0; a < ni; ++a)
                if (!units[a]->in->gamma_on_device)
                    P.gamma[a] = li.take<double2>(static_cast<std::size_t>(units[a]->in->sys.nf) * units[a]->meta->n_in);
        }
    }
    struct MetaPtrs {
        std::vector<int*> tmap;
        std::vector<uint32_t*> out_u;
        std::vector<int32_t*> rowptr;
        std::vector<uint32_t*> src;
        std::vector<C*> coef;
        ClusterJob* clj = nullptr;
        ColJob* colj = nullptr;
        RowJob* rowj = nullptr;
        InvJob* invj = nullptr;
        ScanJob* scanj = nullptr;
        ContractJob* conj = nullptr;
    } M;
    const std::size_t n_spec_jobs = [&] {
        std::size_t s = 0;
        for (auto* u : units) s += 2 * u->in->sys.nf;
        return s;
    }();
    const std::size_t n_col_jobs = n_spec_jobs + ntri;
    const std::size_t n_row_jobs = n_spec_jobs + ntri;
    // one device copy of each distinct time map: first_use[a] is true for the first unit
    // naming it, and the others reuse that unit's arrays
    std::vector<char> first_use(ni, 1);
    std::vector<std::size_t> owner(ni);
    {
        std::unordered_map<const TimeMap*, std::size_t> seen;
        for (std::size_t a = 0; a < ni; ++a) {
            auto r = seen.emplace(units[a]->meta->times.get(), a);
            owner[a] = r.first->second;
            first_use[a] = r.second;
        }
    }
    auto layout_meta = [&](Layout& lay) {
        M.tmap.assign(ni, nullptr);
        M.out_u.assign(ni, nullptr);
        M.rowptr.assign(ni, nullptr);
        M.src.assign(ni, nullptr);
        M.coef.assign(ni, nullptr);
        for (std::size_t a = 0; a < ni; ++a) {
            const InstMeta& m = *units[a]->meta;
            M.tmap[a] = first_use[a] ? lay.take<int>(m.t_count) : M.tmap[owner[a]];
            if (!fcr_only) {
                const CoefTable& ct = *units[a]->coef;
                M.out_u[a] = first_use[a] ? lay.take<uint32_t>(m.T) : M.out_u[owner[a]];
                M.rowptr[a] = lay.take<int32_t>(ct.rowptr.size());
                M.src[a] = lay.take<uint32_t>(std::max<std::size_t>(1, ct.src.size()));
                M.coef[a] = lay.take<C>(std::max<std::size_t>(1, ct.coef.size()));
            }
        }
        M.clj = lay.take<ClusterJob>(n_spec_jobs + ntri);
        M.colj = lay.take<ColJob>(n_col_jobs);
        M.rowj = lay.take<RowJob>(n_row_jobs);
        M.invj = lay.take<InvJob>(2 * ntri);
        M.scanj = lay.take<ScanJob>(ntri);
        M.conj = lay.take<ContractJob>(ni);
    };
    {
        Layout meas;
        layout_meta(meas);
        meta_mem.ensure(meas.off);
        Layout lay{static_cast<char*>(meta_mem.p)};
        layout_meta(lay);
    }
    // column stride of gamma on the device: Nt for caller buffers, n_in for staged host input
    std::vector<std::size_t> gs(ni);
    for (std::size_t a = 0; a < ni; ++a) {
        if (units[a]->in->gamma_on_device) P.gamma[a] = units[a]->in->gamma;
        gs[a] = units[a]->in->gamma_on_device ? units[a]->in->Nt : units[a]->meta->n_in;
    }

    // ---- host staging of small metadata (one pinned buffer, one copy per array) ----
    std::vector<ColJob> colj(n_col_jobs);
    std::vector<RowJob> rowj(n_row_jobs);
    std::vector<InvJob> invj(2 * ntri);
    std::vector<ScanJob> scanj(ntri);
    std::vector<ContractJob> conj(ni);
    std::size_t cj = 0;
    for (std::size_t a = 0; a < ni; ++a) {
        const Tcl4Instance& in = *units[a]->in;
        const InstMeta& m = *units[a]->meta;
        const int nf = in.sys.nf;
        for (int half = 0; half < 2; ++half)
            for (int b = 0; b < nf; ++b) {
                ColJob& c = colj[cj];
                c.g = P.gamma[a] + static_cast<std::size_t>(b) * gs[a];
                c.omega = 0.0;
                c.dt = in.dt;
                c.has_phase = 0;
                c.conj = half;
                c.n_in = static_cast<uint32_t>(m.n_in);
                c.out = P.spec[a] + (static_cast<std::size_t>(half) * nf + b) * Nfft;
                rowj[cj] = RowJob{c.out, nullptr, nullptr, nullptr};
                ++cj;
            }
    }
    auto r_spec_f = [&](std::size_t a, int jm) { return P.spec[a] + static_cast<std::size_t>(jm) * Nfft; };
    auto r_spec_c = [&](std::size_t a, int j) {
        return P.spec[a] + static_cast<std::size_t>(units[a]->in->sys.nf + j) * Nfft;
    };
    for (std::size_t q = 0; q < ntri; ++q) {
        const int a = tris[q].unit, tri = tris[q].tri;
        const Tcl4Instance& in = *units[a]->in;
        const InstMeta& m = *units[a]->meta;
        const std::size_t lo = static_cast<std::size_t>(units[a]->lo), nsub = units[a]->nsub();
        const std::size_t lt = tri - lo;  // triple index within the slice
        const int nf = in.sys.nf;
        const int i = tri / (nf * nf), j = (tri / nf) % nf, k = tri % nf;
        const int jm = in.sys.mirror[j] >= 0 ? in.sys.mirror[j] : j;
        const double w = in.sys.omegas[i] + in.sys.omegas[j] + in.sys.omegas[k];
        const std::size_t slot = q % Q;
        C* z = P.scratch + slot * 2 * Nfft;
        C* wcb = z + Nfft;
        ColJob& c = colj[n_spec_jobs + q];
        c.g = P.gamma[a] + static_cast<std::size_t>(i) * gs[a];
        c.omega = w;
        c.dt = in.dt;
        c.has_phase = 1;
        c.conj = 0;
        c.n_in = static_cast<uint32_t>(m.n_in);
        c.out = z;
        rowj[n_spec_jobs + q] = RowJob{z, wcb, P.spec[a] + static_cast<std::size_t>(jm) * Nfft,
                                       P.spec[a] + static_cast<std::size_t>(nf + j) * Nfft};
        C* cf = G.fused ? nullptr : P.conv[a] + lt * 2 * m.t_count;
        C* cc = G.fused ? nullptr : cf + m.t_count;
        const double scale = in.dt / static_cast<double>(Nfft);
        invj[2 * q] = InvJob{z, cf, static_cast<uint32_t>(m.t_count), scale};
        invj[2 * q + 1] = InvJob{wcb, cc, static_cast<uint32_t>(m.t_count), scale};
        ScanJob& s = scanj[q];
        s.gi = P.gamma[a] + static_cast<std::size_t>(i) * gs[a];
        s.gj = P.gamma[a] + static_cast<std::size_t>(j) * gs[a];
        s.gmj = P.gamma[a] + static_cast<std::size_t>(jm) * gs[a];
        s.omega = w;
        s.dt = in.dt;
        s.n_in = static_cast<uint32_t>(m.n_in);
        s.t_count = static_cast<uint32_t>(m.t_count);
        s.conv_f = cf;
        s.conv_c = cc;
        s.spec_f = r_spec_f(a, jm);
        s.spec_c = r_spec_c(a, j);
        s.tmap = M.tmap[a];
        if (fcr_only && fcr_out_dev) {
            s.vf = fcr_out[3 * a + 0] + static_cast<std::size_t>(tri) * m.U;  // three outputs per unit
            s.vc = fcr_out[3 * a + 1] + static_cast<std::size_t>(tri) * m.U;
            s.vr = fcr_out[3 * a + 2] + static_cast<std::size_t>(tri) * m.U;
        } else {
            s.vf = P.v[a] + lt * m.U;
            s.vc = P.v[a] + (nsub + lt) * m.U;
            s.vr = P.v[a] + (2 * nsub + lt) * m.U;
        }
    }
    // the same jobs for the cluster path (spectra in its [K][M] order)
    std::vector<ClusterJob> clj(n_spec_jobs + ntri);
    for (std::size_t k = 0; k < n_spec_jobs; ++k) {
        const ColJob& c = colj[k];
        clj[k] = ClusterJob{c.g, 0.0, c.dt, 0, c.conj, c.n_in, 0u, 0.0, nullptr, nullptr, c.out, nullptr};
    }
    for (std::size_t q = 0; q < ntri; ++q) {
        const ColJob& c = colj[n_spec_jobs + q];
        const RowJob& r = rowj[n_spec_jobs + q];
        clj[n_spec_jobs + q] = ClusterJob{c.g, c.omega, c.dt, 1, 0, c.n_in, invj[2 * q].t_count, invj[2 * q].scale,
                                          r.spec_f, r.spec_c, invj[2 * q].out, invj[2 * q + 1].out};
    }
    if (!fcr_only) {
        for (std::size_t a = 0; a < ni; ++a) {
            const Tcl4Instance& in = *units[a]->in;
            const InstMeta& m = *units[a]->meta;
            ContractJob& c = conj[a];
            c.rowptr = M.rowptr[a];
            c.src = M.src[a];
            c.coef = M.coef[a];
            c.v = P.v[a];
            c.out_u = M.out_u[a];
            c.out = in.out_on_device ? in.out : P.out[a];
            c.T = static_cast<uint32_t>(m.T);
            c.U = static_cast<uint32_t>(m.U);
            c.E = static_cast<uint32_t>(in.sys.N * in.sys.N * in.sys.N * in.sys.N);
            c.accumulate = units[a]->accumulate ? 1u : 0u;
        }
    }
    // pack everything small into the pinned staging buffer as an image of the metadata
    // buffer's layout (offset of each array = its offset in meta_mem), copied in one piece
    struct Copy {
        std::size_t off, bytes;
    };
    std::vector<Copy> copies;
    std::size_t soff = 0;
    auto plan_copy = [&](void* dst, std::size_t bytes) {
        if (!bytes) return;
        const std::size_t o = static_cast<std::size_t>(static_cast<char*>(dst) - static_cast<char*>(meta_mem.p));
        copies.push_back({o, bytes});
        soff = std::max(soff, o + bytes);
    };
    plan_copy(M.colj, colj.size() * sizeof(ColJob));
    plan_copy(M.rowj, rowj.size() * sizeof(RowJob));
    plan_copy(M.invj, invj.size() * sizeof(InvJob));
    plan_copy(M.scanj, scanj.size() * sizeof(ScanJob));
    plan_copy(M.clj, clj.size() * sizeof(ClusterJob));
    if (!fcr_only) plan_copy(M.conj, conj.size() * sizeof(ContractJob));
    for (std::size_t a = 0; a < ni; ++a) {
        const InstMeta& m = *units[a]->meta;
        if (first_use[a]) plan_copy(M.tmap[a], m.times->tmap.size() * sizeof(int));
        if (!fcr_only) {
            const CoefTable& ct = *units[a]->coef;
            if (first_use[a]) plan_copy(M.out_u[a], m.times->out_u.size() * sizeof(uint32_t));
            plan_copy(M.rowptr[a], ct.rowptr.size() * sizeof(int32_t));
            plan_copy(M.src[a], ct.src.size() * sizeof(uint32_t));
            plan_copy(M.coef[a], ct.coef.size() * sizeof(C));
        }
    }
    PinnedBuffer& staging = staging_buf ? *staging_buf : ws.staging;
    staging.ensure(soff);
    char* sb = static_cast<char*>(staging.p);
    {
        std::size_t k = 0;
        auto put = [&](const void* src, std::size_t bytes) {
            if (!bytes) return;
            std::memcpy(sb + copies[k].off, src, bytes);
            ++k;
        };
        put(colj.data(), colj.size() * sizeof(ColJob));
        put(rowj.data(), rowj.size() * sizeof(RowJob));
        put(invj.data(), invj.size() * sizeof(InvJob));
        put(scanj.data(), scanj.size() * sizeof(ScanJob));
        put(clj.data(), clj.size() * sizeof(ClusterJob));
        if (!fcr_only) put(conj.data(), conj.size() * sizeof(ContractJob));
        for (std::size_t a = 0; a < ni; ++a) {
            const InstMeta& m = *units[a]->meta;
            if (first_use[a]) put(m.times->tmap.data(), m.times->tmap.size() * sizeof(int));
            if (!fcr_only) {
                const CoefTable& ct = *units[a]->coef;
                if (first_use[a]) put(m.times->out_u.data(), m.times->out_u.size() * sizeof(uint32_t));
                put(ct.rowptr.data(), ct.rowptr.size() * sizeof(int32_t));
                put(ct.src.data(), ct.src.size() * sizeof(uint32_t));
                if (std::is_same<R, double>::value) {
                    put(ct.coef.data(), ct.coef.size() * sizeof(C));
                } else {
                    std::vector<float2> cf(ct.coef.size());
                    for (std::size_t e = 0; e < cf.size(); ++e) cf[e] = to_f2(ct.coef[e]);
                    put(cf.data(), cf.size() * sizeof(float2));
                }
            }
        }
    }
    // uploads on `upload` when given, else on st
    cudaStream_t cs = upload ? upload : st;
    if (soff) cuda_check(cudaMemcpyAsync(meta_mem.p, sb, soff, cudaMemcpyHostToDevice, cs), "cudaMemcpyAsync(meta)");
    // host gamma: only the n_in leading samples of each bucket are consumed
    for (std::size_t a = 0; a < ni; ++a)
        if (!units[a]->in->gamma_on_device)
            cuda_check(cudaMemcpy2DAsync(const_cast<double2*>(P.gamma[a]), gs[a] * sizeof(double2), units[a]->in->gamma,
                                         units[a]->in->Nt * sizeof(double2), units[a]->meta->n_in * sizeof(double2),
                                         units[a]->in->sys.nf, cudaMemcpyHostToDevice, cs),
                       "cudaMemcpy2DAsync(gamma)");
    // the caller makes the kernels' stream wait for `uploaded` before it enqueues them
    if (upload) cuda_check(cudaEventRecord(uploaded, upload), "cudaEventRecord(uploaded)");

    host_trace_add("prepare.host", std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_prep).count());
    // the pinned staging buffer is reused by the next call: wait for the copies (a caller
    // that passes its own staging buffer synchronises the stream before reusing it)
    if (!staging_buf) cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(meta)");

    // ---- launches ----
    // the four-step kernels (none on the fused path, whose mixed lengths may have no
    // column kernel)
    const ColFn<R> fwd_col = G.fused ? nullptr : fwd_col_fn<R>(plan.R, plan.L1, g.log2c);
    const InvFn<R> inv_col = G.fused ? nullptr : inv_col_fn<R>(plan.R, plan.L1, g.log2c);
    const RowFn<R> row = G.fused ? nullptr : row_fn<R>(plan.L2, g.log2r);
    // 256-point rows: one warp per row with the transform in registers
    const bool row_warp = plan.L2 == 8;
    const int n_rows = plan.R << plan.L1;  // N1
    const unsigned wrow_grid = static_cast<unsigned>((n_rows + WROW_WARPS - 1) / WROW_WARPS);
    if (!G.fused) {
        set_smem(fwd_col, g.col_smem);
        set_smem(inv_col, g.col_smem);
        set_smem(row, g.row_smem);
    }
    int maxE = 0, maxS = 0;
    std::size_t maxNnz = 1;
    for (auto* u : units) {
        maxE = std::max(maxE, u->in->sys.N * u->in->sys.N * u->in->sys.N * u->in->sys.N);
        maxS = std::max(maxS, 3 * u->nsub());
        if (!fcr_only) maxNnz = std::max(maxNnz, u->coef->src.size());
    }
    std::size_t maxT = 0;
    for (auto* u : units) maxT = std::max(maxT, u->meta->T);
    // contraction: one thread per output time while a [threads][E+1] result tile fits in
    // shared memory (d <= 3); the staged-source kernel for small tables; one warp per
    // (32 entries x 32 times) tile otherwise
    const std::size_t rows_smem = static_cast<std::size_t>(CONTRACT_ROW_THREADS) * (maxE + 1) * sizeof(C);
    const bool contract_rows = rows_smem <= 100 * 1024;
    int maxN = 0;
    for (auto* u : units) maxN = std::max(maxN, u->in->sys.N);
    const bool same_N = [&] {
        for (auto* u : units)
            if (u->in->sys.N != maxN) return false;
        return true;
    }();
    const std::size_t smem_budget = 100 * 1024;
    const std::size_t csr_bytes = maxNnz * (sizeof(C) + 4) + (maxE + 1) * 4 + 64;
    int OTs = 128;
    auto smem_need = [&](int ot) {
        return (static_cast<std::size_t>(maxS) + maxE) * ot * sizeof(C) + csr_bytes;
    };
    while (OTs > 16 && smem_need(OTs) > smem_budget) OTs /= 2;
    // one thread per time leaves a small group (a single instance) with too few CTAs: the
    // staged-source kernel spreads its entries over the threads instead
    const std::size_t row_ctas = (maxT + CONTRACT_ROW_THREADS - 1) / CONTRACT_ROW_THREADS * ni;
    const bool use_rows = contract_rows && same_N && row_ctas >= 2 * 148;
    // the rows kernel with its table preprocessed into shared memory when the table fits and
    // every source offset s * U fits 32 bits
    const std::size_t staged_smem = rows_staged_smem<R>(CONTRACT_ROW_THREADS, maxE, maxNnz);
    const bool offsets_32 = [&] {
        for (auto* u : units)
            if (static_cast<std::size_t>(3) * u->nsub() * u->meta->U >= (std::size_t(1) << 32)) return false;
        return true;
    }();
    const bool rows_staged = use_rows && offsets_32 && staged_smem <= 100 * 1024;
    const bool rows_d2 = rows_staged && maxN == 2;  // results in registers
    const bool contract_smem = !use_rows && maxE < 256 && smem_need(OTs) <= smem_budget;
    const int OT = use_rows ? CONTRACT_ROW_THREADS : OTs;
    const std::size_t csmem = rows_staged ? staged_smem : use_rows ? rows_smem : contract_smem ? smem_need(OT) : 0;
    const std::size_t d2smem = rows_d2_smem<R>(maxNnz);
    if (rows_d2) set_smem(k_contract_rows_d2<R>, d2smem);
    if (rows_staged) set_smem(k_contract_rows_staged<R>, csmem);
    else if (use_rows) set_smem(k_contract_rows<R>, csmem);
    else if (contract_smem) set_smem(k_contract_smem<R>, csmem);
    const int nnz_cap = static_cast<int>(maxNnz);
    struct D2H {
        void* dst;
        const void* src;
        std::size_t bytes;
    };
    std::vector<D2H> d2h;
    if (!fcr_only) {
        for (std::size_t a = 0; a < ni; ++a) {
            if (units[a]->in->out_on_device) continue;
            const Tcl4Instance& in = *units[a]->in;
            const std::size_t E = static_cast<std::size_t>(in.sys.N) * in.sys.N * in.sys.N * in.sys.N;
            d2h.push_back({in.out, P.out[a], units[a]->meta->T * E * sizeof(C)});
        }
    } else if (!fcr_out_dev) {
        const Tcl4Instance& in = *units[0]->in;
        const std::size_t nf3 = static_cast<std::size_t>(in.sys.nf) * in.sys.nf * in.sys.nf;
        const std::size_t U = units[0]->meta->U;
        for (int kind = 0; kind < 3; ++kind)
            d2h.push_back({fcr_out[kind], P.v[0] + kind * nf3 * U, nf3 * U * sizeof(C)});
    }
    // whole instances of the group with the device address of their rows, for opt.out_hook
    std::vector<std::pair<const Tcl4Instance*, void*>> hooked;
    if (!fcr_only && opt.out_hook)
        for (std::size_t a = 0; a < ni; ++a) {
            const WorkUnit& u = *units[a];
            if (u.accumulate || u.lo != 0 || u.hi != u.in->sys.nf * u.in->sys.nf * u.in->sys.nf) continue;
            hooked.emplace_back(u.in, u.in->out_on_device ? u.in->out : static_cast<void*>(P.out[a]));
        }
    const auto out_hook = opt.out_hook;
    const std::size_t n_scan = ntri;
    // single-pass scan (one CTA per triple) once the triples alone fill the GPU four times
    // over; the chunked reduce-then-scan otherwise
    const bool scan_single = n_scan >= static_cast<std::size_t>(148 * 2 * 4);
    const bool fused = G.fused;
    FzPlan<C> fzp{};
    std::size_t fz_bytes = 0;
    if (fused) {
        fzp = get_fz_plan<R>(ws, static_cast<int>(Nfft), st);
        fz_bytes = fz_smem<C>(static_cast<int>(Nfft));
        set_smem(k_fz_spectrum<R>, fz_bytes);
        set_smem(k_fz_conv_scan<R>, fz_bytes);
    }
    const MetaPtrs Mc = M;
    const WorkPtrs<C> Pc = P;
    return [=](cudaStream_t st, ProfRecorder* prp, cudaEvent_t ev0, cudaEvent_t ev1) {
    ProfRecorder dummy;
    ProfRecorder& pr = prp ? *prp : dummy;
    const bool f32 = std::is_same<R, float>::value;
    if (ev0) cuda_check(cudaEventRecord(ev0, st), "cudaEventRecord");
    if (fused) {
        pr.before(f32 ? "fz_spectra_f32" : "fz_spectra_f64");
        k_fz_spectrum<R><<<static_cast<unsigned>(n_spec_jobs), FZ_THREADS, fz_bytes, st>>>(Mc.colj, fzp);
        check_launch("k_fz_spectrum", &pr);
        pr.before(f32 ? "fz_conv_scan_f32" : "fz_conv_scan_f64");
        k_fz_conv_scan<R><<<static_cast<unsigned>(2 * ntri), FZ_THREADS, fz_bytes, st>>>(Mc.scanj, fzp);
        check_launch("k_fz_conv_scan", &pr);
    } else if (use_cluster) {
        pr.before(f32 ? "spectra_cluster_f32" : "spectra_cluster_f64");
        launch_cluster<R>(Mc.clj, n_spec_jobs, cplan, st);
        check_launch("k_conv_cluster(spectra)", &pr);
        pr.before(f32 ? "conv_cluster_f32" : "conv_cluster_f64");
        launch_cluster<R>(Mc.clj + n_spec_jobs, ntri, cplan, st);
        check_launch("k_conv_cluster", &pr);
    } else {
        pr.before(f32 ? "spectra_col_f32" : "spectra_col_f64");
        fwd_col<<<dim3(g.col_grid, static_cast<unsigned>(n_spec_jobs)), g.col_threads, g.col_smem, st>>>(
            Mc.colj, plan, g.log2c);
        check_launch("k_fwd_col(spectra)", &pr);
        pr.before(f32 ? "spectra_row_f32" : "spectra_row_f64");
        if (row_warp)
            k_row_warp256<R><<<dim3(wrow_grid, static_cast<unsigned>(n_spec_jobs)), WROW_THREADS, 0, st>>>(
                Mc.rowj, plan, n_rows);
        else
            row<<<dim3(g.row_grid, static_cast<unsigned>(n_spec_jobs)), g.row_threads, g.row_smem, st>>>(
                Mc.rowj, plan, g.log2r);
        check_launch("k_row(spectra)", &pr);
        const unsigned dft_grid = static_cast<unsigned>((N2 + INV_DFT_THREADS - 1) / INV_DFT_THREADS);
        for (std::size_t ch = 0; ch < nchunks; ++ch) {
            const std::size_t q0 = ch * Q, nq = std::min(Q, ntri - q0);
            pr.before(f32 ? "fwd_col_f32" : "fwd_col_f64");
            fwd_col<<<dim3(g.col_grid, static_cast<unsigned>(nq)), g.col_threads, g.col_smem, st>>>(
                Mc.colj + n_spec_jobs + q0, plan, g.log2c);
            check_launch("k_fwd_col", &pr);
            pr.before(f32 ? "row_conv_f32" : "row_conv_f64");
            if (row_warp)
                k_row_warp256<R><<<dim3(wrow_grid, static_cast<unsigned>(nq)), WROW_THREADS, 0, st>>>(
                    Mc.rowj + n_spec_jobs + q0, plan, n_rows);
            else
                row<<<dim3(g.row_grid, static_cast<unsigned>(nq)), g.row_threads, g.row_smem, st>>>(
                    Mc.rowj + n_spec_jobs + q0, plan, g.log2r);
            check_launch("k_row", &pr);
            pr.before(f32 ? "inv_col_f32" : "inv_col_f64");
            if (inv_dft) {
                k_inv_col_dft<R><<<dim3(dft_grid, static_cast<unsigned>(2 * nq)), INV_DFT_THREADS, 0, st>>>(
                    Mc.invj + 2 * q0, plan, inv_rows);
                check_launch("k_inv_col_dft", &pr);
            } else {
                inv_col<<<dim3(g.col_grid, static_cast<unsigned>(2 * nq)), g.col_threads, g.col_smem, st>>>(
                    Mc.invj + 2 * q0, plan, g.log2c);
                check_launch("k_inv_col", &pr);
            }
        }
    }
    if (fused) {
        // the fused kernel assembled F, C, R already
    } else if (scan_single) {
        // enough triples to fill the GPU: one CTA per triple walks its whole time axis
        pr.before(f32 ? "scan_assemble_f32" : "scan_assemble_f64");
        k_scan_assemble<R, 2, 4><<<static_cast<unsigned>(n_scan), SCAN_THREADS, 0, st>>>(Mc.scanj);
        check_launch("k_scan_assemble", &pr);
    }
    for (std::size_t s0 = 0; !fused && !scan_single && s0 < n_scan; s0 += 65535) {
        const unsigned ns = static_cast<unsigned>(std::min<std::size_t>(65535, n_scan - s0));
        pr.before(f32 ? "scan_reduce_f32" : "scan_reduce_f64");
        k_scan_reduce<R><<<dim3(static_cast<unsigned>(max_chunks), ns), SCAN_THREADS, 0, st>>>(
            Mc.scanj + s0, Pc.partial + s0 * max_chunks * SCAN_W, max_chunks);
        check_launch("k_scan_reduce", &pr);
        pr.before(f32 ? "scan_assemble_f32" : "scan_assemble_f64");
        k_scan_chunks<R><<<dim3(static_cast<unsigned>(max_chunks), ns), SCAN_THREADS, 0, st>>>(
            Mc.scanj + s0, Pc.partial + s0 * max_chunks * SCAN_W, max_chunks);
        check_launch("k_scan_chunks", &pr);
    }
    if (ev1) cuda_check(cudaEventRecord(ev1, st), "cudaEventRecord");
    if (!fcr_only) {
        // the lane's previous sub-batch has left the output staging
        if (down && !d2h.empty()) cuda_check(cudaStreamWaitEvent(st, down->done, 0), "cudaStreamWaitEvent(download)");
        pr.before(f32 ? "contract_f32" : "contract_f64");
        if (rows_d2) {
            const unsigned gx = static_cast<unsigned>((maxT + OT - 1) / OT);
            k_contract_rows_d2<R><<<dim3(gx, static_cast<unsigned>(ni)), CONTRACT_ROW_THREADS, d2smem, st>>>(Mc.conj,
                                                                                                       nnz_cap);
        } else if (rows_staged) {
            const unsigned gx = static_cast<unsigned>((maxT + OT - 1) / OT);
            k_contract_rows_staged<R><<<dim3(gx, static_cast<unsigned>(ni)), CONTRACT_ROW_THREADS, csmem, st>>>(
                Mc.conj, maxN, nnz_cap);
        } else if (use_rows) {
            const unsigned gx = static_cast<unsigned>((maxT + OT - 1) / OT);
            k_contract_rows<R><<<dim3(gx, static_cast<unsigned>(ni)), CONTRACT_ROW_THREADS, csmem, st>>>(Mc.conj, maxN);
        } else if (contract_smem) {
            const unsigned gx = static_cast<unsigned>((maxT + OT - 1) / OT);
            k_contract_smem<R><<<dim3(gx, static_cast<unsigned>(ni)), 256, csmem, st>>>(Mc.conj, OT, maxS, nnz_cap);
        } else {
            const unsigned gx = static_cast<unsigned>((maxT + CONTRACT_TILE - 1) / CONTRACT_TILE);
            const unsigned gy = static_cast<unsigned>((maxE + CONTRACT_TILE - 1) / CONTRACT_TILE);
            k_contract_tiles<R><<<dim3(gx, gy, static_cast<unsigned>(ni)), CONTRACT_TILE_THREADS, 0, st>>>(Mc.conj);
        }
        check_launch("k_contract", &pr);
    }
    cudaStream_t ds = st;
    if (down && !d2h.empty()) {
        cuda_check(cudaEventRecord(down->contracted, st), "cudaEventRecord(contracted)");
        cuda_check(cudaStreamWaitEvent(down->s, down->contracted, 0), "cudaStreamWaitEvent(contracted)");
        ds = down->s;
    }
    // the hook's work goes where the downloads go: it does not hold up the lane's next kernels
    if (!hooked.empty()) out_hook(hooked, ds);
    for (const D2H& c : d2h)
        cuda_check(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, ds), "cudaMemcpyAsync(out)");
    if (ds != st) cuda_check(cudaEventRecord(down->done, ds), "cudaEventRecord(download)");
    };
}

template <class R>
void run_group(std::vector<WorkUnit*>& units, const BuildOptions& opt, cudaStream_t st, Workspace& ws,
               double2* const* fcr_out, bool fcr_out_dev) {
    Enqueue enq = prepare_group<R>(units, opt, st, ws, ws.arena, ws.work, fcr_out, fcr_out_dev);
    ProfRecorder pr;
    pr.st = st;
    enq(st, &pr, opt.fcr_ms ? ws.ev0 : nullptr, opt.fcr_ms ? ws.ev1 : nullptr);
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    pr.resolve();
    if (opt.fcr_ms) {
        float ms = 0.f;
        cuda_check(cudaEventElapsedTime(&ms, ws.ev0, ws.ev1), "cudaEventElapsedTime");
        *opt.fcr_ms += ms;
    }
}

// Transient-memory budget of one group: set explicitly, or 45% of the free device memory
// (at most 64 GiB) at the time of the call.
std::atomic<std::size_t> g_work_budget{0};

std::size_t work_budget() {
    const std::size_t set = g_work_budget.load();
    if (set) return set;
    std::size_t fr = 0, tot = 0;
    cuda_check(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
    return std::min<std::size_t>(fr / 100 * 45, std::size_t(64) << 30);
}

// Work units for a set of instances: instances with equal FFT length are packed into
// groups while their transient arrays fit the budget; an instance that alone exceeds it
// is cut into triple slices, each its own group, run in order (the first overwrites the
// output, the rest accumulate).
template <class R>
std::vector<std::vector<WorkUnit*>> plan_units(std::vector<Tcl4Instance>& insts, std::vector<InstMeta>& metas,
                                               std::size_t budget, std::vector<std::unique_ptr<WorkUnit>>& store) {
    std::map<int, std::vector<std::size_t>> byL;
    for (std::size_t a = 0; a < insts.size(); ++a)
        if (!insts[a].tidx.empty()) byL[size_key(metas[a].L, metas[a].R)].push_back(a);
    std::vector<std::vector<WorkUnit*>> groups;
    for (auto& kv : byL) {
        std::vector<WorkUnit*> cur;
        for (std::size_t a : kv.second) {
            const int nf3 = insts[a].sys.nf * insts[a].sys.nf * insts[a].sys.nf;
            auto unit = std::make_unique<WorkUnit>();
            unit->in = &insts[a];
            unit->meta = &metas[a];
            unit->lo = 0;
            unit->hi = nf3;
            unit->coef = metas[a].coef.get();
            std::vector<WorkUnit*> one{unit.get()};
            const std::size_t need = measure_work<R>(one, false, false);
            if (need > budget) {
                // slices sized from the per-triple cost of a probe slice
                WorkUnit probe = *unit;
                probe.hi = 1;
                std::vector<WorkUnit*> p1{&probe};
                const std::size_t base = measure_work<R>(p1, false, false);
                probe.hi = std::min(nf3, 2);
                const std::size_t two = measure_work<R>(p1, false, false);
                if (base > budget)  // not even one frequency triple fits: the budget is a hard cap
                    throw Error(kOverflow, "one frequency triple needs " + std::to_string(base) +
                                               " bytes of transient device memory, above the work budget of " +
                                               std::to_string(budget) + " bytes");
                const std::size_t per = std::max<std::size_t>(1, two > base ? two - base : base);
                const std::size_t nsub = budget > base ? std::max<std::size_t>(1, (budget - base) / per + 1) : 1;
                if (!insts[a].gamma_on_device || !insts[a].out_on_device)
                    throw Error(kRuntime, "sliced instances need device inputs and outputs");
                for (int lo = 0; lo < nf3; lo += static_cast<int>(nsub)) {
                    auto u = std::make_unique<WorkUnit>();
                    u->in = &insts[a];
                    u->meta = &metas[a];
                    u->lo = lo;
                    u->hi = std::min(nf3, lo + static_cast<int>(nsub));
                    u->accumulate = lo > 0;
                    u->own = slice_table(*metas[a].coef, u->lo, u->hi);
                    u->coef = u->own.get();
                    groups.push_back({u.get()});
                    store.push_back(std::move(u));
                }
                continue;
            }
            cur.push_back(unit.get());
            store.push_back(std::move(unit));
            if (cur.size() > 1 && measure_work<R>(cur, false, false) > budget) {
                WorkUnit* last = cur.back();
                cur.pop_back();
                groups.push_back(cur);
                cur = {last};
            }
        }
        if (!cur.empty()) groups.push_back(cur);
    }
    return groups;
}

// Instances that will be sliced read and write device memory: host gamma and host
// outputs go through device copies made here (and copied back by the caller).
struct HostIoStage {
    std::vector<void*> bufs;
    struct Back {
        void* host;
        const void* dev;
        std::size_t bytes;
    };
    std::vector<Back> back;
    ~HostIoStage() {
        for (void* p : bufs) cudaFree(p);
    }
};

template <class R>
void stage_sliced_io(std::vector<Tcl4Instance>& insts, std::vector<InstMeta>& metas, std::size_t budget,
                     HostIoStage& io, cudaStream_t st) {
    using C = cplx_t<R>;
    for (std::size_t a = 0; a < insts.size(); ++a) {
        Tcl4Instance& in = insts[a];
        if (in.tidx.empty() || (in.gamma_on_device && in.out_on_device)) continue;
        WorkUnit u;
        u.in = &in;
        u.meta = &metas[a];
        u.hi = in.sys.nf * in.sys.nf * in.sys.nf;
        u.coef = metas[a].coef.get();
        std::vector<WorkUnit*> one{&u};
        if (measure_work<R>(one, false, false) <= budget) continue;
        if (!in.gamma_on_device) {
            const std::size_t bytes = static_cast<std::size_t>(in.sys.nf) * in.Nt * sizeof(double2);
            void* d = nullptr;
            cuda_check(cudaMalloc(&d, bytes), "cudaMalloc(sliced gamma)");
            io.bufs.push_back(d);
            cuda_check(cudaMemcpyAsync(d, in.gamma, bytes, cudaMemcpyHostToDevice, st), "sliced gamma");
            in.gamma = static_cast<const double2*>(d);
            in.gamma_on_device = true;
        }
        if (!in.out_on_device) {
            const std::size_t E = static_cast<std::size_t>(in.sys.N) * in.sys.N * in.sys.N * in.sys.N;
            const std::size_t bytes = metas[a].T * E * sizeof(C);
            void* d = nullptr;
            cuda_check(cudaMalloc(&d, bytes), "cudaMalloc(sliced out)");
            io.bufs.push_back(d);
            io.back.push_back({in.out, d, bytes});
            in.out = d;
            in.out_on_device = true;
        }
    }
}

}  // namespace

void set_work_budget(std::size_t bytes) { g_work_budget.store(bytes); }
void set_fused_conv(bool on) { g_fused.store(on ? 1 : 0); }

void release_workspace() {
    Workspace& ws = workspace();
    cuda_check(cudaStreamSynchronize(ws.stream), "cudaStreamSynchronize(release)");
    for (auto& l : ws.extra)
        if (l.s) cuda_check(cudaStreamSynchronize(l.s), "cudaStreamSynchronize(release)");
    if (ws.upload) cuda_check(cudaStreamSynchronize(ws.upload), "cudaStreamSynchronize(release)");
    ws.work.release();
    ws.arena.release();
    ws.staging.release();
    for (auto& l : ws.extra) {
        l.work.release();
        l.arena.release();
        l.staging.release();
    }
    for (auto& b : ws.sub_bufs) {
        b->arena.release();
        b->input.release();
        b->staging.release();
    }
    for (auto& d : ws.down) {
        if (d.s) cuda_check(cudaStreamSynchronize(d.s), "cudaStreamSynchronize(release)");
        d.out.release();
    }
}
bool fused_conv() { return g_fused.load() != 0; }

std::size_t fft_length_for(std::size_t n_in, bool fp32, bool causal, std::size_t pad_factor, int* key) {
    std::size_t target = 2 * n_in - 1;
    if (pad_factor > 0) target = std::max(target, pad_factor * n_in);
    int L = 0, R = 1;
    choose_fft(target, fp32, causal && pad_factor == 0, L, R);
    if (key) *key = size_key(L, R);
    return static_cast<std::size_t>(R) << L;
}

namespace {

void validate_system(const SystemDesc& s) {
    if (s.N <= 0) throw Error(kInvalidArgument, "system: N must be > 0");
    if (s.nf <= 0) throw Error(kInvalidArgument, "system: nf must be > 0");
    if (s.num_ops <= 0) throw Error(kInvalidArgument, "coupling_ops must be non-empty");
    if (static_cast<int>(s.omegas.size()) != s.nf || static_cast<int>(s.mirror.size()) != s.nf)
        throw Error(kInvalidArgument, "system: frequency metadata has wrong size");
    if (static_cast<int>(s.p2f.size()) != s.N * s.N) throw Error(kInvalidArgument, "system: pair_to_freq has wrong shape");
    for (int v : s.p2f) {
        if (v < 0) throw Error(kRuntime, "pair_to_freq contains -1 (missing frequency buckets)");
        if (v >= s.nf) throw Error(kInvalidArgument, "pair_to_freq entry out of range");
    }
    for (int v : s.mirror)
        if (v < 0 || v >= s.nf) throw Error(kInvalidArgument, "mirror entry out of range");
    if (static_cast<std::size_t>(s.num_ops) * s.N * s.N != s.ops.size())
        throw Error(kInvalidArgument, "coupling operator has wrong shape");
    const double nf3 = static_cast<double>(s.nf) * s.nf * s.nf;
    if (3.0 * nf3 >= 2147483647.0) throw Error(kOverflow, "nf too large");
}

}  // namespace

cudaStream_t default_stream() { return workspace().stream; }

void set_tuning(int L, bool fp32, const Tuning& t) {
    if (t.col_tile < 8 || t.row_tile < 8 || (t.col_tile & (t.col_tile - 1)) || (t.row_tile & (t.row_tile - 1)) ||
        t.col_tile > 8192 || t.row_tile > 8192 || t.chunk_bytes == 0)
        throw Error(kInvalidArgument, "tuning: tiles must be powers of two in [8, 8192] and chunk_bytes > 0");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[{L, fp32 ? 1 : 0}] = t;
}

Tuning get_tuning(int L, bool fp32) { return tuning_for(L, fp32); }

void clear_tuning() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
}

uint64_t kernel_launches() { return g_launches.load(); }

void raise_smem_limit(const void* kernel, std::size_t bytes) {
    if (bytes <= 48 * 1024) return;
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, std::size_t> granted;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lk(mu);
    std::size_t& g = granted[{dev, kernel}];
    if (bytes <= g) return;
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)),
               "cudaFuncSetAttribute(smem)");
    g = bytes;
}
void count_launches(uint64_t n) { g_launches.fetch_add(n); }
bool host_trace_on() {
    static const bool on = std::getenv("TACO_TRACE_HOST") != nullptr;
    return on;
}
void host_trace_add(const char* phase, double ms) {
    if (host_trace_on()) t_phases.add(phase, ms);
}
void profile_enable(bool on) { g_profile.store(on); }
void profile_reset() {
    ProfStore& ps = prof_store();
    std::lock_guard<std::mutex> lk(ps.mu);
    ps.acc.clear();
    ps.order.clear();
}
std::vector<ProfileEntry> profile_entries() {
    ProfStore& ps = prof_store();
    std::lock_guard<std::mutex> lk(ps.mu);
    std::vector<ProfileEntry> out;
    for (const auto& n : ps.order) {
        const auto& v = ps.acc.at(n);
        out.push_back({n.c_str(), v.first, v.second});
    }
    return out;
}

void build_mirror(const std::vector<double>& omegas, double tol, std::vector<int>& mirror, int* zero_index) {
    const double t = std::max(1e-12, tol);
    const int nf = static_cast<int>(omegas.size());
    mirror.assign(nf, -1);
    int zero = -1;
    for (int b = 0; b < nf; ++b) {
        const double w = omegas[b];
        int best = -1;
        if (std::abs(w) <= t) {
            best = b;
            if (zero < 0) zero = b;
        } else {
            double ba = std::numeric_limits<double>::infinity();
            for (int bp = 0; bp < nf; ++bp) {
                const double d = std::abs(omegas[bp] - (-w));
                if (d < ba) {
                    ba = d;
                    best = bp;
                }
            }
        }
        mirror[b] = best;
    }
    if (zero < 0) {
        double ba = std::numeric_limits<double>::infinity();
        for (int b = 0; b < nf; ++b)
            if (std::abs(omegas[b]) < ba) {
                ba = std::abs(omegas[b]);
                zero = b;
            }
        if (zero < 0) zero = 0;
    }
    if (zero_index) *zero_index = zero;
}

namespace {
void validate_and_derive(std::vector<Tcl4Instance>& insts, const BuildOptions& opt, std::vector<InstMeta>& metas);
}

void tcl4_build_direct(std::vector<Tcl4Instance>& insts, const BuildOptions& opt, cudaStream_t stream) {
    Workspace& ws = workspace();
    cudaStream_t st = stream ? stream : ws.stream;
    if (opt.fcr_ms) *opt.fcr_ms = 0.0;
    Lap lap;
    std::vector<InstMeta> metas;
    validate_and_derive(insts, opt, metas);
    lap("derive");
    const std::size_t budget = work_budget();
    HostIoStage io;
    std::vector<std::unique_ptr<WorkUnit>> store;
    std::vector<std::vector<WorkUnit*>> groups;
    if (opt.fp32) {
        stage_sliced_io<float>(insts, metas, budget, io, st);
        groups = plan_units<float>(insts, metas, budget, store);
    } else {
        stage_sliced_io<double>(insts, metas, budget, io, st);
        groups = plan_units<double>(insts, metas, budget, store);
    }
    lap("plan");
    // Large builds of whole instances run as sub-batches of about kPipeSub instances on two
    // or three lanes (streams with their own buffers): the host preparation and the input
    // upload of one sub-batch overlap the kernels and the output download of the others.
    // Slices (ordered accumulation), profiling and F/C/R timing keep the single-lane order.
    constexpr std::size_t kPipeSub = 48;
    std::size_t nunits = 0;
    bool whole = true;
    for (auto& gu : groups)
        for (auto* u : gu) {
            ++nunits;
            whole = whole && !u->accumulate && u->lo == 0 && u->hi == u->in->sys.nf * u->in->sys.nf * u->in->sys.nf;
        }
    bool pipeline = whole && io.back.empty() && !opt.fcr_ms && !g_profile.load() && nunits >= kPipeSub;
    if (pipeline) {
        // two lanes' transient arrays must fit the group budget together (large instances,
        // whose sub-batches each fill the budget, run on one lane)
        std::size_t mw = 0;
        for (auto& gu : groups) {
            const std::size_t n = gu.size(), parts = std::max<std::size_t>(1, (n + kPipeSub / 2) / kPipeSub);
            for (std::size_t p = 0; p < parts; ++p) {
                std::vector<WorkUnit*> sub(gu.begin() + p * n / parts, gu.begin() + (p + 1) * n / parts);
                mw = std::max(mw, opt.fp32 ? measure_work<float>(sub, false, false) : measure_work<double>(sub, false, false));
            }
        }
        pipeline = 2 * mw <= budget;
    }
    if (!pipeline) {
        for (auto& gu : groups) {
            if (opt.fp32) run_group<float>(gu, opt, st, ws, nullptr, false);
            else run_group<double>(gu, opt, st, ws, nullptr, false);
        }
        lap("groups");
    } else {
        // sub-batches of kPipeSub instances or more (rounded count per group)
        // (the first group starts with a third of that: its outputs start downloading early)
        std::vector<std::vector<WorkUnit*>> subs;
        std::size_t max_work = 0, max_input = 0;
        bool first = true;
        for (auto& gu : groups) {
            const std::size_t b0 = first && gu.size() > kPipeSub ? kPipeSub / 3 : 0;
            first = false;
            const std::size_t n = gu.size() - b0, parts = std::max<std::size_t>(1, (n + kPipeSub / 2) / kPipeSub);
            for (std::size_t p = 0; p < parts + (b0 ? 1 : 0); ++p) {
                if (b0 && p == 0) subs.emplace_back(gu.begin(), gu.begin() + b0);
                else {
                    const std::size_t q = b0 ? p - 1 : p;
                    subs.emplace_back(gu.begin() + b0 + q * n / parts, gu.begin() + b0 + (q + 1) * n / parts);
                }
                max_work = std::max(max_work, opt.fp32 ? measure_work<float>(subs.back(), false, false)
                                                       : measure_work<double>(subs.back(), false, false));
                std::size_t in_bytes = 0;
                for (auto* u : subs.back())
                    if (!u->in->gamma_on_device)
                        in_bytes += static_cast<std::size_t>(u->in->sys.nf) * u->meta->n_in * sizeof(double2) + 256;
                max_input = std::max(max_input, in_bytes);
            }
        }
        // a third lane while three sub-batches' transient arrays fit the group budget
        const std::size_t nlanes = subs.size() >= 3 && 3 * max_work <= budget ? 3 : 2;
        // sub-batch buffer slots (metadata, staged input): up to two per lane, while the
        // lanes' work arrays and the slots' inputs fit the group budget; a slot is reused
        // once the sub-batch that held it has finished
        std::size_t nslots = std::min<std::size_t>(subs.size(), 2 * nlanes);
        while (nslots > 1 && nlanes * max_work + nslots * max_input > budget) --nslots;
        struct Lane {
            cudaStream_t s;
            DeviceBuffer* work;
        };
        std::vector<Lane> lanes{{st, &ws.work}};
        if (!ws.upload) cuda_check(cudaStreamCreateWithFlags(&ws.upload, cudaStreamNonBlocking), "cudaStreamCreate");
        // the other lanes and the uploads start after the work already queued on the caller's stream
        cuda_check(cudaEventRecord(ws.ev0, st), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(ws.upload, ws.ev0, 0), "cudaStreamWaitEvent");
        for (std::size_t l = 1; l < nlanes; ++l) {
            auto& x = ws.extra[l - 1];
            if (!x.s) cuda_check(cudaStreamCreateWithFlags(&x.s, cudaStreamNonBlocking), "cudaStreamCreate");
            cuda_check(cudaStreamWaitEvent(x.s, ws.ev0, 0), "cudaStreamWaitEvent");
            lanes.push_back({x.s, &x.work});
        }
        // Every buffer a sub-batch writes from the host (metadata, staged input) is its own, so
        // the host never waits inside the loop: all uploads queue on the upload stream ahead of
        // the downloads, each lane's kernels wait for their sub-batch's upload event, and a
        // lane's work arrays (sized here for the largest sub-batch) are reused in its stream order.
        while (ws.sub_bufs.size() < nslots) {
            ws.sub_bufs.push_back(std::make_unique<Workspace::SubBuffers>());
            cuda_check(cudaEventCreateWithFlags(&ws.sub_bufs.back()->uploaded, cudaEventDisableTiming), "cudaEventCreate");
            cuda_check(cudaEventCreateWithFlags(&ws.sub_bufs.back()->done, cudaEventDisableTiming), "cudaEventCreate");
        }
        for (auto& L : lanes) L.work->ensure(max_work);
        // each lane downloads on its own stream (created once)
        for (std::size_t l = 0; l < nlanes; ++l) {
            auto& d = ws.down[l];
            if (!d.s) {
                cuda_check(cudaStreamCreateWithFlags(&d.s, cudaStreamNonBlocking), "cudaStreamCreate");
                cuda_check(cudaEventCreateWithFlags(&d.contracted, cudaEventDisableTiming), "cudaEventCreate");
                cuda_check(cudaEventCreateWithFlags(&d.done, cudaEventDisableTiming), "cudaEventCreate");
            }
            // the previous build's downloads are complete (the build ended with them); a
            // fresh event makes the first wait of this build a no-op
            cuda_check(cudaEventRecord(d.done, d.s), "cudaEventRecord");
        }
        // traced calls time each sub-batch on the device: lane start, inputs uploaded,
        // F/C/R done, outputs downloaded
        std::vector<cudaEvent_t> evs(lap.on ? 4 * subs.size() : 0);
        for (auto& e : evs) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
        // each sub-batch is enqueued as soon as it is prepared: its upload on the upload stream,
        // its kernels on its lane (after the upload), its download on the lane's download
        // stream (the lane's next kernels do not wait for it)
        for (std::size_t k = 0; k < subs.size(); ++k) {
            const Lane& L = lanes[k % nlanes];
            Workspace::SubBuffers& sb = *ws.sub_bufs[k % nslots];
            if (k >= nslots) {
                cuda_check(cudaEventSynchronize(sb.done), "cudaEventSynchronize(slot)");
                lap("slot_wait");
            }
            Workspace::Download* dl = &ws.down[k % nlanes];
            Enqueue enq = opt.fp32 ? prepare_group<float>(subs[k], opt, L.s, ws, sb.arena, *L.work, nullptr, false,
                                                          &sb.staging, &sb.input, ws.upload, sb.uploaded, dl)
                                   : prepare_group<double>(subs[k], opt, L.s, ws, sb.arena, *L.work, nullptr, false,
                                                           &sb.staging, &sb.input, ws.upload, sb.uploaded, dl);
            lap("prepare");
            if (lap.on) cuda_check(cudaEventRecord(evs[4 * k], L.s), "cudaEventRecord");
            cuda_check(cudaStreamWaitEvent(L.s, sb.uploaded, 0), "cudaStreamWaitEvent(uploaded)");
            if (lap.on) cuda_check(cudaEventRecord(evs[4 * k + 1], L.s), "cudaEventRecord");
            enq(L.s, nullptr, nullptr, lap.on ? evs[4 * k + 2] : nullptr);
            cuda_check(cudaEventRecord(sb.done, L.s), "cudaEventRecord(slot)");
            if (lap.on) cuda_check(cudaEventRecord(evs[4 * k + 3], dl->s), "cudaEventRecord");
            lap("enqueue");
        }
        for (std::size_t l = 1; l < nlanes; ++l)
            cuda_check(cudaStreamSynchronize(lanes[l].s), "cudaStreamSynchronize(lane)");
        cuda_check(cudaStreamSynchronize(ws.upload), "cudaStreamSynchronize(upload)");
        for (std::size_t l = 0; l < nlanes; ++l)
            cuda_check(cudaStreamSynchronize(ws.down[l].s), "cudaStreamSynchronize(download)");
        lap("lane_wait");
        if (lap.on) {
            cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(build)");
            std::string line = "taco sub-batch device times (ms from the first lane event; queued/uploaded/fcr/done):";
            for (std::size_t k = 0; k < subs.size(); ++k) {
                line += " [" + std::to_string(subs[k].size()) + " inst, lane " + std::to_string(k % nlanes) + ":";
                for (int q = 0; q < 4; ++q) {
                    float ms = 0.f;
                    cuda_check(cudaEventElapsedTime(&ms, evs[0], evs[4 * k + q]), "cudaEventElapsedTime");
                    line += " " + std::to_string(ms);
                }
                line += "]";
            }
            std::fprintf(stderr, "%s\n", line.c_str());
        }
        for (auto& e : evs) cudaEventDestroy(e);
    }
    for (const auto& b : io.back)
        cuda_check(cudaMemcpyAsync(b.host, b.dev, b.bytes, cudaMemcpyDeviceToHost, st), "cudaMemcpyAsync(sliced out)");
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(build)");
    lap("final_wait");
    if (lap.on) {
        std::string line = "taco host phases (ms, " + std::to_string(insts.size()) + " instances):";
        for (const auto& e : t_phases.ms) line += " " + std::string(e.first) + "=" + std::to_string(e.second);
        std::fprintf(stderr, "%s\n", line.c_str());
        t_phases.ms.clear();
    }
}

// F/C/R series of many instances with device buffers: instances of equal Nt share build
// groups (within the work budget), each unit writing its own three outputs.
void triple_kernels_batch(const std::vector<FcrRequest>& reqs, const BuildOptions& opt, cudaStream_t stream) {
    if (reqs.empty()) return;
    Workspace& ws = workspace();
    cudaStream_t st = stream ? stream : ws.stream;
    std::vector<Tcl4Instance> insts(reqs.size());
    std::vector<InstMeta> metas(reqs.size());
    BuildOptions o = opt;
    o.fp32 = false;
    o.causal_truncation = false;
    o.fcr_ms = nullptr;
    for (std::size_t k = 0; k < reqs.size(); ++k) {
        const FcrRequest& r = reqs[k];
        SystemDesc s = r.sys;
        if (s.num_ops <= 0) {  // F/C/R do not depend on the coupling operators
            s.num_ops = 1;
            s.ops.assign(static_cast<std::size_t>(s.N) * s.N, make_double2(0.0, 0.0));
        }
        validate_system(s);
        if (r.Nt == 0) throw Error(kInvalidArgument, "empty gamma_series");
        if (r.Nt >= (std::size_t(1) << 31)) throw Error(kOverflow, "Nt too large");
        if (!(r.dt > 0.0)) throw Error(kInvalidArgument, "dt must be > 0");
        if (!r.gamma || !r.F || !r.C || !r.R) throw Error(kInvalidArgument, "null pointer");
        Tcl4Instance& in = insts[k];
        in.sys = s;
        in.gamma = r.gamma;
        in.gamma_on_device = true;
        in.Nt = r.Nt;
        in.dt = r.dt;
        in.tidx.iota(r.Nt);
        derive_meta(in, o, metas[k], false);
    }
    std::vector<WorkUnit> units(reqs.size());
    std::map<std::size_t, std::vector<std::size_t>> by_nt;
    for (std::size_t k = 0; k < reqs.size(); ++k) {
        units[k].in = &insts[k];
        units[k].meta = &metas[k];
        units[k].hi = insts[k].sys.nf * insts[k].sys.nf * insts[k].sys.nf;
        units[k].coef = metas[k].coef.get();
        by_nt[reqs[k].Nt].push_back(k);
    }
    const std::size_t budget = work_budget();
    for (auto& kv : by_nt) {
        std::vector<WorkUnit*> gu;
        std::vector<double2*> outs;
        auto flush = [&] {
            if (gu.empty()) return;
            run_group<double>(gu, o, st, ws, outs.data(), true);
            gu.clear();
            outs.clear();
        };
        for (std::size_t k : kv.second) {
            gu.push_back(&units[k]);
            if (gu.size() > 1 && measure_work<double>(gu, true, true) > budget) {
                gu.pop_back();
                flush();
                gu.push_back(&units[k]);
            }
            outs.insert(outs.end(), {reqs[k].F, reqs[k].C, reqs[k].R});
        }
        flush();
    }
}

void triple_kernels(const SystemDesc& sys, const double2* gamma, bool gamma_on_device, std::size_t Nt, double dt,
                    double2* F, double2* Cc, double2* R, bool out_on_device, const BuildOptions& opt,
                    cudaStream_t stream) {
    Workspace& ws = workspace();
    cudaStream_t st = stream ? stream : ws.stream;
    SystemDesc s = sys;
    if (s.num_ops <= 0) {  // F/C/R do not depend on the coupling operators
        s.num_ops = 1;
        s.ops.assign(static_cast<std::size_t>(s.N) * s.N, make_double2(0.0, 0.0));
    }
    validate_system(s);
    if (Nt == 0) throw Error(kInvalidArgument, "empty gamma_series");
    if (Nt >= (std::size_t(1) << 31)) throw Error(kOverflow, "Nt too large");
    if (!(dt > 0.0)) throw Error(kInvalidArgument, "dt must be > 0");
    if (!gamma || !F || !Cc || !R) throw Error(kInvalidArgument, "null pointer");
    Tcl4Instance in;
    in.sys = s;
    in.gamma = gamma;
    in.gamma_on_device = gamma_on_device;
    in.Nt = Nt;
    in.dt = dt;
    in.tidx.iota(Nt);
    BuildOptions o = opt;
    o.fp32 = false;
    o.causal_truncation = false;
    InstMeta m;
    derive_meta(in, o, m, false);
    WorkUnit u;
    u.in = &in;
    u.meta = &m;
    u.hi = s.nf * s.nf * s.nf;
    u.coef = m.coef.get();
    std::vector<WorkUnit*> gu{&u};
    double2* outs[3] = {F, Cc, R};
    if (opt.fcr_ms) *opt.fcr_ms = 0.0;
    run_group<double>(gu, o, st, ws, outs, out_on_device);
}

struct Tcl4Plan {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<std::unique_ptr<DeviceBuffer>> mems;  // per-group metadata
    DeviceBuffer work;                                 // transient arrays, shared
    std::vector<std::unique_ptr<WorkUnit>> units;
    std::vector<Enqueue> enqs;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t kernels = 0;
    // work enqueued after the graph on every execute (the FP64 heads of the FP32 form),
    // holding the buffers and plans it uses; its kernel count
    std::function<void(cudaStream_t)> pre, tail;
    uint64_t tail_kernels = 0;
    ~Tcl4Plan() {
        pre = nullptr;  // the pre and tail work's plans and buffers go before the stream
        tail = nullptr;
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {
// A buffer flagged as device memory must be device (or managed) memory of the current device
// and aligned for its element type: a host address or a misaligned one handed to the kernels
// would fault instead of failing.  The last accepted pointer is remembered per thread
// (consecutive instances often share one buffer).
void check_device_buffer(const void* p, std::size_t align, const char* what) {
    if (reinterpret_cast<std::uintptr_t>(p) % align != 0)
        throw Error(kInvalidArgument, std::string(what) + " (device) is not " + std::to_string(align) + "-byte aligned");
    thread_local const void* last_ok = nullptr;
    thread_local int last_dev = -1;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (p == last_ok && dev == last_dev) return;
    cudaPointerAttributes a{};
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw Error(kInvalidArgument, std::string(what) + " is flagged as device memory but is not a CUDA allocation");
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)
        throw Error(kInvalidArgument, std::string(what) + " is flagged as device memory but is host memory");
    if (a.type == cudaMemoryTypeDevice && a.device != dev)
        throw Error(kInvalidArgument, std::string(what) + " is on device " + std::to_string(a.device) +
                                          ", not the current device " + std::to_string(dev));
    last_ok = p;
    last_dev = dev;
}

void validate_and_derive(std::vector<Tcl4Instance>& insts, const BuildOptions& opt, std::vector<InstMeta>& metas) {
    const std::size_t n = insts.size();
    metas.resize(n);
    const unsigned nthreads =
        n >= 16 ? std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency())) : 1u;
    // fn(k) for k in [0, count) on the host threads (round robin)
    auto spread = [&](std::size_t count, const std::function<void(std::size_t)>& fn) {
        const unsigned nt = static_cast<unsigned>(std::min<std::size_t>(nthreads, count));
        if (nt <= 1) {
            for (std::size_t k = 0; k < count; ++k) fn(k);
            return;
        }
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nt; ++t)
            pool.emplace_back([&, t] {
                for (std::size_t k = t; k < count; k += nt) fn(k);
            });
        for (auto& th : pool) th.join();
    };
    // distinct time lists (instances sharing a caller's array share one list)
    constexpr std::size_t kNone = ~std::size_t(0);
    std::unordered_map<const void*, std::size_t> list_index;
    std::vector<std::size_t> first;          // first instance of each distinct list
    std::vector<std::size_t> lid(n, kNone);  // list of each instance
    for (std::size_t a = 0; a < n; ++a) {
        Tcl4Instance& in = insts[a];
        validate_system(in.sys);
        if (in.Nt == 0) throw Error(kInvalidArgument, "empty gamma_series");
        if (in.Nt >= (std::size_t(1) << 31)) throw Error(kOverflow, "Nt too large");
        if (!(in.dt > 0.0)) throw Error(kInvalidArgument, "dt must be > 0");
        if (!in.gamma) throw Error(kInvalidArgument, "gamma is null");
        if (in.gamma_on_device) check_device_buffer(in.gamma, sizeof(double2), "gamma");
        if (in.tidx.empty()) continue;
        if (!in.out) throw Error(kInvalidArgument, "output pointer is null");
        if (in.out_on_device && !in.internal)
            check_device_buffer(in.out, opt.fp32 ? sizeof(float2) : sizeof(double2), "output");
        auto r = list_index.emplace(in.tidx.identity(), first.size());
        if (r.second) first.push_back(a);
        lid[a] = r.first->second;
    }
    // every requested index below the instance's Nt, checked before any map is sized by it
    std::vector<uint32_t> tmax(first.size(), 0);
    for (std::size_t k = 0; k < first.size(); ++k)
        for (uint32_t t : insts[first[k]].tidx) tmax[k] = std::max(tmax[k], t);
    for (std::size_t a = 0; a < n; ++a)
        if (lid[a] != kNone && tmax[lid[a]] >= insts[a].Nt) throw Error(kOutOfRange, "time_index out of range");
    std::vector<std::shared_ptr<const TimeMap>> maps(first.size());
    std::vector<std::exception_ptr> map_errs(first.size());
    spread(first.size(), [&](std::size_t k) {
        try {
            maps[k] = make_time_map(insts[first[k]].tidx);
        } catch (...) {
            map_errs[k] = std::current_exception();
        }
    });
    for (auto& e : map_errs)
        if (e) std::rethrow_exception(e);
    // per-instance metadata (FFT length, coefficient table) on several host threads for
    // large batches; the first failing instance's error is rethrown.  Systems with large
    // coefficient maps (nf >= 21, d >= 5) one at a time, each map built on several threads;
    // the others spread over the threads, one map per thread.
    std::vector<std::exception_ptr> errs(n);
    auto large = [&](std::size_t a) { return insts[a].sys.nf >= 21; };
    auto derive = [&](std::size_t a) {
        if (lid[a] == kNone) return;
        try {
            derive_meta(insts[a], opt, metas[a], true, maps[lid[a]]);
        } catch (...) {
            errs[a] = std::current_exception();
        }
    };
    for (std::size_t a = 0; a < n; ++a)
        if (large(a)) derive(a);
    auto work = [&](std::size_t a0, std::size_t step) {
        set_coef_table_threads(nthreads > 1 ? 1 : 0);
        for (std::size_t a = a0; a < n; a += step)
            if (!large(a)) derive(a);
        set_coef_table_threads(0);
    };
    if (nthreads <= 1) {
        work(0, 1);
    } else {
        std::vector<std::thread> pool;
        for (unsigned k = 0; k < nthreads; ++k) pool.emplace_back(work, k, nthreads);
        for (auto& th : pool) th.join();
    }
    for (auto& e : errs)
        if (e) std::rethrow_exception(e);
}
}  // namespace

std::size_t work_budget_now() { return work_budget(); }

// Transient arrays of a plan's groups.  Groups of whole instances run concurrently (branches
// of the plan's graph, each group in its own region of the buffer) when their sum fits a
// quarter of the group budget `cap` (the plan keeps its buffer: large batches of long series
// would otherwise hold several groups' worth of memory for the plan's lifetime) and the
// buffer the plan is lent (`avail`); otherwise, or when an instance is built in slices (its
// slices accumulate into one output in order), one after another in one shared region.
struct PlanWork {
    std::vector<std::size_t> each;  // bytes of each group
    std::size_t total = 0;
    bool concurrent = false;
};
PlanWork plan_work(const std::vector<std::vector<WorkUnit*>>& groups, bool fp32, std::size_t cap,
                   std::size_t avail = ~std::size_t(0)) {
    PlanWork w;
    std::size_t most = 0, sum = 0;
    bool whole = true;
    for (auto& gu : groups) {
        std::vector<WorkUnit*> g(gu);
        const std::size_t b = fp32 ? measure_work<float>(g, false, false) : measure_work<double>(g, false, false);
        w.each.push_back(b);
        most = std::max(most, b);
        sum += align_up(b, std::size_t(256));
        for (auto* u : gu)
            whole = whole && !u->accumulate && u->lo == 0 && u->hi == u->in->sys.nf * u->in->sys.nf * u->in->sys.nf;
    }
    w.concurrent = groups.size() > 1 && whole && sum <= cap / 4 && sum <= avail;
    w.total = w.concurrent ? sum : most;
    return w;
}

std::size_t plan_work_bytes(std::vector<Tcl4Instance>& insts, const BuildOptions& opt, std::size_t budget) {
    std::vector<InstMeta> metas;
    validate_and_derive(insts, opt, metas);
    std::vector<std::unique_ptr<WorkUnit>> store;
    std::vector<std::vector<WorkUnit*>> groups =
        opt.fp32 ? plan_units<float>(insts, metas, budget, store) : plan_units<double>(insts, metas, budget, store);
    return plan_work(groups, opt.fp32, budget).total;
}

Tcl4Plan* plan_create_direct(std::vector<Tcl4Instance>& insts, const BuildOptions& opt, void* ext_work,
                             std::size_t ext_cap, std::size_t budget_in) {
    for (const auto& in : insts)
        if (!in.gamma_on_device || !in.out_on_device)
            throw Error(kInvalidArgument, "plans take device inputs and outputs (TACO_IN_DEVICE | TACO_OUT_DEVICE)");
    std::vector<InstMeta> metas;
    validate_and_derive(insts, opt, metas);
    BuildOptions popt = opt;
    popt.out_hook = nullptr;  // a replayed graph calls no host code
    auto plan = std::make_unique<Tcl4Plan>();
    cuda_check(cudaGetDevice(&plan->device), "cudaGetDevice");
    cuda_check(cudaStreamCreateWithFlags(&plan->stream, cudaStreamNonBlocking), "cudaStreamCreate(plan)");
    Workspace& ws = workspace();
    // a lent buffer is the budget (the caller sized it for these instances); else the
    // share of the free memory
    const std::size_t budget = ext_work ? (budget_in ? budget_in : ext_cap) : work_budget();
    std::vector<std::vector<WorkUnit*>> groups =
        opt.fp32 ? plan_units<float>(insts, metas, budget, plan->units) : plan_units<double>(insts, metas, budget, plan->units);
    // one transient buffer, sized before any group records its pointers: a region per group
    // when the groups run concurrently, else one region they share in order
    const PlanWork pw = plan_work(groups, opt.fp32, budget, ext_work ? ext_cap : ~std::size_t(0));
    if (ext_work) {  // a caller's buffer shared by plans that run one after another
        plan->work.p = ext_work;
        plan->work.cap = ext_cap;
        plan->work.owned = false;
    }
    plan->work.ensure(pw.total, true);
    std::size_t region = 0;
    for (std::size_t gi = 0; gi < groups.size(); ++gi) {
        auto& gu = groups[gi];
        DeviceBuffer view;  // the group's region (prepare_group records pointers into it)
        view.owned = false;
        view.p = static_cast<char*>(plan->work.p) + region;
        view.cap = pw.concurrent ? pw.each[gi] : plan->work.cap;
        if (pw.concurrent) region += align_up(pw.each[gi], std::size_t(256));
        plan->mems.push_back(std::make_unique<DeviceBuffer>());
        if (opt.fp32)
            plan->enqs.push_back(prepare_group<float>(gu, popt, plan->stream, ws, *plan->mems.back(), view, nullptr, false));
        else
            plan->enqs.push_back(prepare_group<double>(gu, popt, plan->stream, ws, *plan->mems.back(), view, nullptr, false));
    }
    // concurrent groups: captured as branches forked from and joined into the plan's stream
    struct Branches {
        std::vector<cudaStream_t> s;
        std::vector<cudaEvent_t> e;
        ~Branches() {
            for (auto x : s) cudaStreamDestroy(x);
            for (auto x : e) cudaEventDestroy(x);
        }
    } br;
    if (pw.concurrent) {
        br.s.assign(groups.size() - 1, nullptr);
        br.e.assign(groups.size(), nullptr);
        for (auto& x : br.s) cuda_check(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking), "cudaStreamCreate(branch)");
        for (auto& x : br.e) cuda_check(cudaEventCreateWithFlags(&x, cudaEventDisableTiming), "cudaEventCreate(branch)");
    }
    const uint64_t k0 = g_launches.load();
    cuda_check(cudaStreamBeginCapture(plan->stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    try {
        if (pw.concurrent) {
            cuda_check(cudaEventRecord(br.e[0], plan->stream), "cudaEventRecord(fork)");
            for (auto x : br.s) cuda_check(cudaStreamWaitEvent(x, br.e[0], 0), "cudaStreamWaitEvent(fork)");
            plan->enqs[0](plan->stream, nullptr, nullptr, nullptr);
            for (std::size_t gi = 1; gi < groups.size(); ++gi) {
                plan->enqs[gi](br.s[gi - 1], nullptr, nullptr, nullptr);
                cuda_check(cudaEventRecord(br.e[gi], br.s[gi - 1]), "cudaEventRecord(join)");
                cuda_check(cudaStreamWaitEvent(plan->stream, br.e[gi], 0), "cudaStreamWaitEvent(join)");
            }
        } else {
            for (auto& e : plan->enqs) e(plan->stream, nullptr, nullptr, nullptr);
        }
    } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(plan->stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    cuda_check(cudaStreamEndCapture(plan->stream, &plan->graph), "cudaStreamEndCapture");
    plan->kernels = g_launches.load() - k0;
    g_launches.fetch_sub(plan->kernels);  // captured, not launched
    cuda_check(cudaGraphInstantiate(&plan->exec, plan->graph, 0), "cudaGraphInstantiate");
    return plan.release();
}

void plan_execute(Tcl4Plan* plan, cudaStream_t stream) {
    if (!plan) throw Error(kInvalidArgument, "plan is null");
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev != plan->device) throw Error(kInvalidArgument, "plan belongs to another device");
    // asynchronous on exactly the caller's stream (0 is the legacy default stream)
    if (plan->pre) plan->pre(stream);
    cuda_check(cudaGraphLaunch(plan->exec, stream), "cudaGraphLaunch");
    g_launches.fetch_add(plan->kernels);
    if (plan->tail) plan->tail(stream);
}

void plan_set_tail(Tcl4Plan* plan, std::function<void(cudaStream_t)> pre, std::function<void(cudaStream_t)> tail,
                   uint64_t kernels) {
    plan->pre = std::move(pre);
    plan->tail = std::move(tail);
    plan->tail_kernels = kernels;
}

void plan_destroy(Tcl4Plan* plan) { delete plan; }

uint64_t plan_kernels(const Tcl4Plan* plan) { return plan ? plan->kernels + plan->tail_kernels : 0; }

std::size_t rk4_num_samples(std::size_t steps, std::size_t sample_every) {
    if (sample_every == 0) return 0;
    return (steps + sample_every - 1) / sample_every + 1;
}

void rk4_propagate_device(const std::vector<Rk4Request>& reqs, cudaStream_t stream) {
    if (reqs.empty()) return;
    Workspace& ws = workspace();
    cudaStream_t st = stream ? stream : ws.stream;
    // group by (D, storage)
    std::map<std::pair<int, int>, std::vector<std::size_t>> groups;
    for (std::size_t k = 0; k < reqs.size(); ++k) {
        const Rk4Request& r = reqs[k];
        if (r.D <= 0) throw Error(kInvalidArgument, "rk4: dimension must be > 0");
        if (!(r.dt > 0.0)) throw Error(kInvalidArgument, "rk4: dt must be > 0");
        if (r.steps < 1) throw Error(kInvalidArgument, "rk4: L_series must have at least 2 matrices (endpoints)");
        if (!r.L || !r.r) throw Error(kInvalidArgument, "rk4: null pointer");
        if (r.obs_out && !r.obs) throw Error(kInvalidArgument, "rk4: obs_out needs obs");
        if ((r.samples || r.obs_out) && r.sample_every == 0)
            throw Error(kInvalidArgument, "rk4: sample_every must be > 0");
        groups[{r.D, r.fp32_storage ? 1 : 0}].push_back(k);
    }
    std::vector<Rk4Job> jobs(reqs.size());
    for (std::size_t k = 0; k < reqs.size(); ++k) {
        const Rk4Request& r = reqs[k];
        jobs[k] = Rk4Job{r.L, r.L_half, r.L_add, r.steps, r.dt, r.r, r.sample_every, r.samples, r.obs, r.obs_out};
    }
    // reorder jobs group-contiguously and upload once
    std::vector<Rk4Job> ordered;
    std::vector<std::pair<std::size_t, std::size_t>> ranges;
    for (auto& kv : groups) {
        ranges.push_back({ordered.size(), kv.second.size()});
        for (std::size_t k : kv.second) ordered.push_back(jobs[k]);
    }
    ws.arena.ensure(ordered.size() * sizeof(Rk4Job) + 256);
    ws.staging.ensure(ordered.size() * sizeof(Rk4Job));
    std::memcpy(ws.staging.p, ordered.data(), ordered.size() * sizeof(Rk4Job));
    Rk4Job* dj = static_cast<Rk4Job*>(ws.arena.p);
    cuda_check(cudaMemcpyAsync(dj, ws.staging.p, ordered.size() * sizeof(Rk4Job), cudaMemcpyHostToDevice, st),
               "cudaMemcpyAsync(rk4 jobs)");
    std::size_t gi = 0;
    ProfRecorder pr;
    pr.st = st;
    for (auto& kv : groups) {
        const int D = kv.first.first;
        pr.before(D <= 16 ? "rk4_warp" : "rk4_cta");
        const bool f32 = kv.first.second != 0;
        const auto rg = ranges[gi++];
        Rk4Job* base = dj + rg.first;
        const int n = static_cast<int>(rg.second);
        if (D <= 16) {
            const int warps_per_block = 4;
            const unsigned grid = static_cast<unsigned>((n + warps_per_block - 1) / warps_per_block);
            if (D <= 4) {
                // step matrices built in parallel, one matrix per sequential step
                uint64_t mstride = 1, sstride = 1;
                for (std::size_t k = 0; k < rg.second; ++k) {
                    const Rk4Job& jk = ordered[rg.first + k];
                    mstride = std::max<uint64_t>(mstride, jk.steps);
                    if (jk.sample_every)
                        sstride = std::max<uint64_t>(sstride, (jk.steps + jk.sample_every - 1) / jk.sample_every + 1);
                }
                const std::size_t mbytes = static_cast<std::size_t>(n) * mstride * RK_REC * sizeof(double2);
                const std::size_t sbytes = static_cast<std::size_t>(n) * sstride * 4 * sizeof(double2);
                ws.work.ensure(mbytes + sbytes + 512);
                double2* M = static_cast<double2*>(ws.work.p);
                double2* Rs = reinterpret_cast<double2*>(static_cast<char*>(ws.work.p) + align_up(mbytes, 256));
                const dim3 mgrid(static_cast<unsigned>((mstride + 127) / 128), static_cast<unsigned>(n));
                if (f32) k_rk4_stepmat<float2><<<mgrid, 128, 0, st>>>(base, D, mstride, M);
                else k_rk4_stepmat<double2><<<mgrid, 128, 0, st>>>(base, D, mstride, M);
                check_launch("k_rk4_stepmat", &pr);
                pr.before("rk4_chain");
                k_rk4_chain<<<grid, 32 * warps_per_block, 0, st>>>(base, n, D, M, mstride, Rs, sstride);
                check_launch("k_rk4_chain", &pr);
                pr.before("rk4_samples");
                k_rk4_samples<<<dim3(static_cast<unsigned>((sstride + 127) / 128), static_cast<unsigned>(n)), 128, 0, st>>>(
                    base, D, Rs, sstride);
                check_launch("k_rk4_samples", &pr);
            } else {
                if (f32) k_rk4_warp<float2, 16><<<grid, 32 * warps_per_block, 0, st>>>(base, n, D);
                else k_rk4_warp<double2, 16><<<grid, 32 * warps_per_block, 0, st>>>(base, n, D);
                check_launch("k_rk4_warp", &pr);
            }
        } else {
            const std::size_t smem = 6 * static_cast<std::size_t>(D) * sizeof(double2);
            const int threads = std::min(256, ((D + 31) / 32) * 32);
            if (f32) {
                set_smem(k_rk4_cta<float2>, smem);
                k_rk4_cta<float2><<<static_cast<unsigned>(n), threads, smem, st>>>(base, D);
            } else {
                set_smem(k_rk4_cta<double2>, smem);
                k_rk4_cta<double2><<<static_cast<unsigned>(n), threads, smem, st>>>(base, D);
            }
            check_launch("k_rk4_cta", &pr);
        }
    }
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(rk4)");
    pr.resolve();
}

}  // namespace taco
