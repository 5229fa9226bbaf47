// capi.cpp -- extern "C" entry points of libtaco_b200.so (see include/taco_b200.h).
#include "taco_b200.h"

#include <chrono>
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "engine.hpp"
#include "gw_coef.hpp"

namespace {

thread_local std::string g_last_error;
std::atomic<std::size_t> g_pad_factor{0};

template <class Fn>
int guarded(Fn&& fn) {
    try {
        fn();
        return TACO_OK;
    } catch (const taco::Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return TACO_ERR_RUNTIME;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return TACO_ERR_RUNTIME;
    }
}

void require_device() {
    int n = 0;
    const cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        throw taco::Error(taco::kNoDevice, std::string("no CUDA device: ") + cudaGetErrorString(e));
}

taco::SystemDesc to_desc(const taco_system_view* v, bool need_ops = true) {
    if (!v) throw taco::Error(taco::kInvalidArgument, "system view is null");
    taco::SystemDesc s;
    s.N = v->N;
    s.nf = v->nf;
    s.num_ops = v->num_ops;
    if (s.N <= 0) throw taco::Error(taco::kInvalidArgument, "system: N must be > 0");
    if (s.nf <= 0) throw taco::Error(taco::kInvalidArgument, "system: nf must be > 0");
    if (!v->omegas || !v->pair_to_freq) throw taco::Error(taco::kInvalidArgument, "system: null metadata");
    s.omegas.assign(v->omegas, v->omegas + s.nf);
    s.p2f.assign(v->pair_to_freq, v->pair_to_freq + static_cast<std::size_t>(s.N) * s.N);
    if (v->mirror) {
        s.mirror.assign(v->mirror, v->mirror + s.nf);
    } else {
        taco::build_mirror(s.omegas, v->tol > 0 ? v->tol : 1e-9, s.mirror, nullptr);
    }
    if (need_ops) {
        if (s.num_ops <= 0) throw taco::Error(taco::kInvalidArgument, "coupling_ops must be non-empty");
        if (!v->ops) throw taco::Error(taco::kInvalidArgument, "coupling_ops is null");
        const double2* o = reinterpret_cast<const double2*>(v->ops);
        s.ops.assign(o, o + static_cast<std::size_t>(s.num_ops) * s.N * s.N);
    } else if (s.num_ops > 0 && v->ops) {
        const double2* o = reinterpret_cast<const double2*>(v->ops);
        s.ops.assign(o, o + static_cast<std::size_t>(s.num_ops) * s.N * s.N);
    } else {
        s.num_ops = 0;
    }
    return s;
}

void check_method(int method) {
    if (method != TACO_FCR_CONVOLUTION)
        throw taco::Error(taco::kInvalidArgument, "only FCRMethod::Convolution is supported on the device path");
}

taco::BuildOptions options(int precision, int flags, double* fcr_ms) {
    if (precision != TACO_PREC_FP64 && precision != TACO_PREC_FP32)
        throw taco::Error(taco::kInvalidArgument, "precision must be TACO_PREC_FP64 or TACO_PREC_FP32");
    taco::BuildOptions o;
    o.fp32 = (precision == TACO_PREC_FP32);
    o.causal_truncation = (flags & TACO_FULL_LENGTH_FFT) == 0;
    o.pad_factor = g_pad_factor.load();
    o.fcr_ms = fcr_ms;
    return o;
}

void fill_tidx(taco::Tcl4Instance& in, const uint32_t* tidx, std::size_t T) {
    if (tidx == nullptr || T == 0) in.tidx.iota(in.Nt);
    else in.tidx.assign(tidx, tidx + T);
}

std::vector<taco::Tcl4Instance> to_instances(const taco_tcl4_instance* inst, size_t count, int flags) {
    if (count > 0 && !inst) throw taco::Error(taco::kInvalidArgument, "instances is null");
    std::vector<taco::Tcl4Instance> insts(count);
    // instances naming the same caller array (pointer and length) share one copy of it
    std::map<std::pair<const uint32_t*, std::size_t>, std::size_t> first_of;
    for (std::size_t k = 0; k < count; ++k) {
        taco::Tcl4Instance& in = insts[k];
        in.sys = to_desc(&inst[k].sys);
        in.gamma = reinterpret_cast<const double2*>(inst[k].gamma);
        in.gamma_on_device = (flags & TACO_IN_DEVICE) != 0;
        in.Nt = inst[k].Nt;
        in.dt = inst[k].dt;
        if (in.Nt == 0) throw taco::Error(taco::kInvalidArgument, "empty gamma_series");
        const bool listed = inst[k].tidx != nullptr && inst[k].T > 0;
        const std::pair<const uint32_t*, std::size_t> key{listed ? inst[k].tidx : nullptr,
                                                          listed ? inst[k].T : inst[k].Nt};
        auto it = first_of.find(key);
        if (it != first_of.end()) {
            in.tidx.share_with(insts[it->second].tidx);
        } else {
            fill_tidx(in, inst[k].tidx, inst[k].T);
            first_of.emplace(key, k);
        }
        in.out = inst[k].L4_out;
        in.out_on_device = (flags & TACO_OUT_DEVICE) != 0;
    }
    return insts;
}

}  // namespace

extern "C" {

const char* taco_version(void) { return TACO_B200_VERSION; }

const char* taco_last_error(void) { return g_last_error.c_str(); }

int taco_device_count(int* count) {
    return guarded([&] {
        int n = 0;
        const cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess) n = 0;
        if (count) *count = n;
    });
}

int taco_set_device(int gpu_id) {
    return guarded([&] {
        require_device();
        taco::cuda_check(cudaSetDevice(gpu_id), "cudaSetDevice");
    });
}

void taco_set_fcr_fft_pad_factor(size_t factor) { g_pad_factor.store(factor); }
size_t taco_get_fcr_fft_pad_factor(void) { return g_pad_factor.load(); }

int taco_compute_triple_kernels(const taco_system_view* sys, const taco_c128* gamma, size_t Nt, double dt,
                                int method, taco_c128* F, taco_c128* C, taco_c128* R, int flags, void* stream) {
    return guarded([&] {
        check_method(method);
        require_device();
        taco::SystemDesc s = to_desc(sys, false);
        taco::BuildOptions o = options(TACO_PREC_FP64, 0, nullptr);
        taco::triple_kernels(s, reinterpret_cast<const double2*>(gamma), (flags & TACO_IN_DEVICE) != 0, Nt, dt,
                             reinterpret_cast<double2*>(F), reinterpret_cast<double2*>(C),
                             reinterpret_cast<double2*>(R), (flags & TACO_OUT_DEVICE) != 0, o,
                             static_cast<cudaStream_t>(stream));
    });
}

int taco_compute_triple_kernels_batch(const taco_fcr_request* reqs, size_t n, int method, void* stream) {
    return guarded([&] {
        check_method(method);
        require_device();
        if (n && !reqs) throw taco::Error(taco::kInvalidArgument, "null request array");
        std::vector<taco::FcrRequest> rs(n);
        for (size_t k = 0; k < n; ++k) {
            rs[k].sys = to_desc(&reqs[k].sys, false);
            rs[k].gamma = reinterpret_cast<const double2*>(reqs[k].gamma);
            rs[k].Nt = reqs[k].Nt;
            rs[k].dt = reqs[k].dt;
            rs[k].F = reinterpret_cast<double2*>(reqs[k].F);
            rs[k].C = reinterpret_cast<double2*>(reqs[k].C);
            rs[k].R = reinterpret_cast<double2*>(reqs[k].R);
        }
        taco::triple_kernels_batch(rs, options(TACO_PREC_FP64, 0, nullptr), static_cast<cudaStream_t>(stream));
    });
}

int taco_tcl4_build_batch(const taco_system_view* sys, const taco_c128* gamma, size_t Nt, double dt,
                          const uint32_t* tidx, size_t T, int method, int precision, void* L4_out, int flags,
                          void* stream, double* fcr_ms) {
    return guarded([&] {
        check_method(method);
        require_device();
        std::vector<taco::Tcl4Instance> insts(1);
        taco::Tcl4Instance& in = insts[0];
        in.sys = to_desc(sys);
        in.gamma = reinterpret_cast<const double2*>(gamma);
        in.gamma_on_device = (flags & TACO_IN_DEVICE) != 0;
        in.Nt = Nt;
        in.dt = dt;
        if (Nt == 0) throw taco::Error(taco::kInvalidArgument, "empty gamma_series");
        fill_tidx(in, tidx, T);
        in.out = L4_out;
        in.out_on_device = (flags & TACO_OUT_DEVICE) != 0;
        taco::tcl4_build(insts, options(precision, flags, fcr_ms), static_cast<cudaStream_t>(stream));
    });
}

int taco_tcl4_build(const taco_system_view* sys, const taco_c128* gamma, size_t Nt, double dt, size_t time_index,
                    int method, taco_c128* L4_out, int flags, void* stream) {
    if (time_index >= Nt) {
        g_last_error = "build_TCL4_generator: time_index out of range";
        return TACO_ERR_OUT_OF_RANGE;
    }
    const uint32_t t = static_cast<uint32_t>(time_index);
    return taco_tcl4_build_batch(sys, gamma, Nt, dt, &t, 1, method, TACO_PREC_FP64, L4_out, flags, stream, nullptr);
}

int taco_tcl4_correction_series(const taco_system_view* sys, const taco_c128* gamma, size_t Nt, double dt,
                                int method, taco_c128* L4_out, int flags, void* stream) {
    return taco_tcl4_build_batch(sys, gamma, Nt, dt, nullptr, 0, method, TACO_PREC_FP64, L4_out, flags, stream,
                                 nullptr);
}

int taco_tcl4_build_instances(const taco_tcl4_instance* inst, size_t count, int method, int precision, int flags,
                              void* stream) {
    return guarded([&] {
        check_method(method);
        require_device();
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<taco::Tcl4Instance> insts = to_instances(inst, count, flags);
        taco::host_trace_add("abi", std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
        taco::tcl4_build(insts, options(precision, flags, nullptr), static_cast<cudaStream_t>(stream));
    });
}

struct taco_tcl4_plan {
    taco::Tcl4Plan* p;
};

int taco_tcl4_plan_create(const taco_tcl4_instance* inst, size_t count, int method, int precision, int flags,
                          taco_tcl4_plan** plan) {
    return guarded([&] {
        if (!plan) throw taco::Error(taco::kInvalidArgument, "plan is null");
        *plan = nullptr;
        check_method(method);
        require_device();
        std::vector<taco::Tcl4Instance> insts = to_instances(inst, count, flags);
        taco::Tcl4Plan* p = taco::plan_create(insts, options(precision, flags, nullptr));
        *plan = new taco_tcl4_plan{p};
    });
}

int taco_tcl4_plan_execute(taco_tcl4_plan* plan, void* stream) {
    return guarded([&] {
        if (!plan) throw taco::Error(taco::kInvalidArgument, "plan is null");
        taco::plan_execute(plan->p, static_cast<cudaStream_t>(stream));
    });
}

int taco_tcl4_plan_destroy(taco_tcl4_plan* plan) {
    return guarded([&] {
        if (!plan) return;
        taco::plan_destroy(plan->p);
        delete plan;
    });
}

int taco_tcl4_build_batch_noalloc(const taco_system_view* sys, const taco_c128* gamma, size_t Nt, double dt,
                                  const uint32_t* tidx, size_t T, int precision, void* L4_out, void* stream) {
    return guarded([&] {
        require_device();
        if (precision != TACO_PREC_FP64 && precision != TACO_PREC_FP32)
            throw taco::Error(taco::kInvalidArgument, "precision must be TACO_PREC_FP64 or TACO_PREC_FP32");
        taco::SystemDesc s = to_desc(sys);
        std::vector<uint32_t> t;
        if (tidx == nullptr || T == 0) {
            t.resize(Nt);
            for (std::size_t k = 0; k < Nt; ++k) t[k] = static_cast<uint32_t>(k);
        } else {
            t.assign(tidx, tidx + T);
        }
        taco::noalloc_tcl4_build(s, reinterpret_cast<const double2*>(gamma), Nt, dt, t, precision == TACO_PREC_FP32,
                                 g_pad_factor.load(), L4_out, static_cast<cudaStream_t>(stream));
    });
}

int taco_rk4_propagate(const void* L_series, const void* L_half, const void* L_add, int l_is_fp32, size_t steps,
                       int D, double dt, taco_c128* r, size_t sample_every, taco_c128* samples,
                       const taco_c128* obs, taco_c128* obs_out, int flags, void* stream) {
    return guarded([&] {
        require_device();
        if (D <= 0) throw taco::Error(taco::kInvalidArgument, "rk4: dimension must be > 0");
        if (!(dt > 0.0)) throw taco::Error(taco::kInvalidArgument, "propagate_rk4_dense: dt must be > 0");
        if (steps < 1)
            throw taco::Error(taco::kInvalidArgument,
                              "propagate_rk4_dense: L_series must have at least 2 matrices (endpoints)");
        if ((samples || obs_out) && sample_every == 0)
            throw taco::Error(taco::kInvalidArgument, "propagate_rk4_dense: sample_every must be > 0");
        if (!L_series || !r) throw taco::Error(taco::kInvalidArgument, "rk4: null pointer");
        const bool dev = (flags & TACO_IN_DEVICE) != 0;
        const std::size_t esz = l_is_fp32 ? sizeof(float2) : sizeof(double2);
        const std::size_t DD = static_cast<std::size_t>(D) * D;
        const std::size_t ns = taco::rk4_num_samples(steps, sample_every);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        taco::Rk4Request q;
        q.fp32_storage = l_is_fp32 != 0;
        q.steps = steps;
        q.D = D;
        q.dt = dt;
        q.sample_every = (samples || obs_out) ? sample_every : 0;
        if (dev) {
            q.L = L_series;
            q.L_half = L_half;
            q.L_add = L_add;
            q.r = reinterpret_cast<double2*>(r);
            q.samples = reinterpret_cast<double2*>(samples);
            q.obs = reinterpret_cast<const double2*>(obs);
            q.obs_out = reinterpret_cast<double2*>(obs_out);
            taco::rk4_propagate_device({q}, st);
            return;
        }
        // host buffers: stage through device memory owned by this call
        std::vector<void*> allocs;
        auto dalloc = [&](std::size_t bytes) {
            void* p = nullptr;
            taco::cuda_check(cudaMalloc(&p, bytes), "cudaMalloc(rk4)");
            allocs.push_back(p);
            return p;
        };
        try {
            auto up = [&](const void* h, std::size_t bytes) -> void* {
                if (!h) return nullptr;
                void* d = dalloc(bytes);
                taco::cuda_check(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(rk4 in)");
                return d;
            };
            q.L = up(L_series, (steps + 1) * DD * esz);
            q.L_half = up(L_half, steps * DD * esz);
            q.L_add = up(L_add, (steps + 1) * DD * esz);
            q.r = static_cast<double2*>(up(r, D * sizeof(double2)));
            q.obs = static_cast<const double2*>(up(obs, D * sizeof(double2)));
            if (samples) q.samples = static_cast<double2*>(dalloc(ns * D * sizeof(double2)));
            if (obs_out) q.obs_out = static_cast<double2*>(dalloc(ns * sizeof(double2)));
            taco::rk4_propagate_device({q}, st);
            taco::cuda_check(cudaMemcpyAsync(r, q.r, D * sizeof(double2), cudaMemcpyDeviceToHost, st), "rk4 out");
            if (samples)
                taco::cuda_check(cudaMemcpyAsync(samples, q.samples, ns * D * sizeof(double2), cudaMemcpyDeviceToHost, st),
                                 "rk4 samples");
            if (obs_out)
                taco::cuda_check(cudaMemcpyAsync(obs_out, q.obs_out, ns * sizeof(double2), cudaMemcpyDeviceToHost, st),
                                 "rk4 obs");
            taco::cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(rk4)");
        } catch (...) {
            cudaStreamSynchronize(st);
            for (void* p : allocs) cudaFree(p);
            throw;
        }
        for (void* p : allocs) cudaFree(p);
    });
}

namespace {
// device staging for host buffers of the convenience paths
struct DevAllocs {
    std::vector<void*> ptrs;
    void* take(std::size_t bytes) {
        void* p = nullptr;
        taco::cuda_check(cudaMalloc(&p, bytes ? bytes : 16), "cudaMalloc(staging)");
        ptrs.push_back(p);
        return p;
    }
    ~DevAllocs() {
        for (void* p : ptrs) cudaFree(p);
    }
};
}  // namespace

int taco_tcl2_generator_series(const taco_system_view* sys, const double* eps, const taco_c128* gamma, size_t Nt,
                               const uint32_t* tidx, size_t T, taco_c128* L2_out, int flags, void* stream) {
    return guarded([&] {
        require_device();
        taco::SystemDesc s = to_desc(sys);
        if (!eps || !gamma || !L2_out) throw taco::Error(taco::kInvalidArgument, "tcl2 series: null pointer");
        if (Nt == 0) throw taco::Error(taco::kInvalidArgument, "empty gamma_series");
        std::vector<uint32_t> t;
        if (!tidx || T == 0) {
            t.resize(Nt);
            for (std::size_t k = 0; k < Nt; ++k) t[k] = static_cast<uint32_t>(k);
        } else {
            t.assign(tidx, tidx + T);
        }
        for (uint32_t k : t)
            if (k >= Nt) throw taco::Error(taco::kOutOfRange, "time_index out of range");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        const std::size_t E = static_cast<std::size_t>(s.N) * s.N * s.N * s.N;
        DevAllocs da;
        const double2* g = reinterpret_cast<const double2*>(gamma);
        if (!(flags & TACO_IN_DEVICE)) {
            void* dg = da.take(s.nf * Nt * sizeof(double2));
            taco::cuda_check(cudaMemcpyAsync(dg, gamma, s.nf * Nt * sizeof(double2), cudaMemcpyHostToDevice, st), "gamma");
            g = static_cast<const double2*>(dg);
        }
        double2* out = reinterpret_cast<double2*>(L2_out);
        if (!(flags & TACO_OUT_DEVICE)) out = static_cast<double2*>(da.take(t.size() * E * sizeof(double2)));
        taco::tcl2_series_device(s, eps, g, Nt, t, out, st);
        if (!(flags & TACO_OUT_DEVICE)) {
            taco::cuda_check(cudaMemcpyAsync(L2_out, out, t.size() * E * sizeof(double2), cudaMemcpyDeviceToHost, st),
                             "L2 out");
            taco::cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        }
    });
}

int taco_gamma_trapz(const taco_c128* C, size_t N, double dt, const double* omegas, size_t M, taco_c128* G, int flags,
                     void* stream) {
    return guarded([&] {
        require_device();
        if (!C || !G || (M > 0 && !omegas)) throw taco::Error(taco::kInvalidArgument, "gamma_trapz: null pointer");
        if (N == 0 || M == 0 || !(dt > 0.0)) throw taco::Error(taco::kInvalidArgument, "gamma_trapz: empty input");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        DevAllocs da;
        const double2* c = reinterpret_cast<const double2*>(C);
        if (!(flags & TACO_IN_DEVICE)) {
            void* dc = da.take(N * sizeof(double2));
            taco::cuda_check(cudaMemcpyAsync(dc, C, N * sizeof(double2), cudaMemcpyHostToDevice, st), "C");
            c = static_cast<const double2*>(dc);
        }
        double2* g = reinterpret_cast<double2*>(G);
        if (!(flags & TACO_OUT_DEVICE)) g = static_cast<double2*>(da.take(M * N * sizeof(double2)));
        taco::gamma_trapz_device(c, N, dt, std::vector<double>(omegas, omegas + M), g, st);
        if (!(flags & TACO_OUT_DEVICE)) {
            taco::cuda_check(cudaMemcpyAsync(G, g, M * N * sizeof(double2), cudaMemcpyDeviceToHost, st), "G out");
            taco::cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        }
    });
}

int taco_gamma_trapz_batch(const taco_gamma_request* reqs, size_t n, void* stream) {
    return guarded([&] {
        require_device();
        if (!reqs && n) throw taco::Error(taco::kInvalidArgument, "gamma_trapz: null requests");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        std::vector<taco::GammaRequest> rs(n);
        for (size_t k = 0; k < n; ++k) {
            const taco_gamma_request& q = reqs[k];
            if (!q.omegas && q.M) throw taco::Error(taco::kInvalidArgument, "gamma_trapz: null omegas");
            rs[k].C = reinterpret_cast<const double2*>(q.C);
            rs[k].N = q.N;
            rs[k].dt = q.dt;
            rs[k].omegas.assign(q.omegas, q.omegas + q.M);
            rs[k].G = reinterpret_cast<double2*>(q.G);
        }
        taco::gamma_trapz_batch_device(rs, st);
    });
}

int taco_propagate_tcl(const taco_system_view* sys, const double* eps, const taco_c128* gamma, size_t Nt, double dt,
                       size_t steps, int order, int precision, const taco_c128* rho0, const taco_c128* obs,
                       size_t sample_every, taco_c128* obs_out, taco_c128* rho_out, int flags, void* stream) {
    return guarded([&] {
        require_device();
        if (order != 0 && order != 2 && order != 4) throw taco::Error(taco::kInvalidArgument, "order must be 0, 2, or 4");
        if (steps < 1) throw taco::Error(taco::kInvalidArgument, "propagate: steps must be >= 1");
        if (steps >= Nt) throw taco::Error(taco::kOutOfRange, "propagate: steps must be < Nt");
        if (!eps || !gamma || !rho0) throw taco::Error(taco::kInvalidArgument, "propagate: null pointer");
        if (obs_out && !obs) throw taco::Error(taco::kInvalidArgument, "propagate: obs_out needs obs");
        if (obs_out && sample_every == 0) throw taco::Error(taco::kInvalidArgument, "sample_every must be > 0");
        taco::SystemDesc s = to_desc(sys);
        const int D = s.N * s.N;
        const std::size_t E = static_cast<std::size_t>(D) * D, ns = taco::rk4_num_samples(steps, sample_every);
        const bool dev_in = (flags & TACO_IN_DEVICE) != 0, dev_out = (flags & TACO_OUT_DEVICE) != 0;
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        DevAllocs da;
        const double2* g = reinterpret_cast<const double2*>(gamma);
        if (!dev_in) {
            void* dg = da.take(s.nf * Nt * sizeof(double2));
            taco::cuda_check(cudaMemcpyAsync(dg, gamma, s.nf * Nt * sizeof(double2), cudaMemcpyHostToDevice, st), "gamma");
            g = static_cast<const double2*>(dg);
        }
        std::vector<uint32_t> t(steps + 1);
        for (std::size_t k = 0; k <= steps; ++k) t[k] = static_cast<uint32_t>(k);
        // L2 (or L0 alone for order 0: L2 with gamma = 0 is the unitary part)
        double2* L2 = static_cast<double2*>(da.take((steps + 1) * E * sizeof(double2)));
        if (order == 0) {
            double2* zero = static_cast<double2*>(da.take(s.nf * Nt * sizeof(double2)));
            taco::cuda_check(cudaMemsetAsync(zero, 0, s.nf * Nt * sizeof(double2), st), "cudaMemsetAsync");
            taco::tcl2_series_device(s, eps, zero, Nt, t, L2, st);
        } else {
            taco::tcl2_series_device(s, eps, g, Nt, t, L2, st);
        }
        const bool fp32 = precision == TACO_PREC_FP32;
        void* L4 = nullptr;
        if (order == 4) {
            L4 = da.take((steps + 1) * E * (fp32 ? sizeof(float2) : sizeof(double2)));
            std::vector<taco::Tcl4Instance> insts(1);
            insts[0].sys = s;
            insts[0].gamma = g;
            insts[0].gamma_on_device = true;
            insts[0].Nt = Nt;
            insts[0].dt = dt;
            insts[0].tidx = t;
            insts[0].out = L4;
            insts[0].out_on_device = true;
            taco::tcl4_build(insts, options(precision, 0, nullptr), st);
        }
        double2* r = static_cast<double2*>(da.take(D * sizeof(double2)));
        taco::cuda_check(cudaMemcpyAsync(r, rho0, D * sizeof(double2), dev_in ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st), "rho0");
        const double2* o = nullptr;
        if (obs) {
            void* d_o = da.take(D * sizeof(double2));
            taco::cuda_check(cudaMemcpyAsync(d_o, obs, D * sizeof(double2), dev_in ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st), "obs");
            o = static_cast<const double2*>(d_o);
        }
        double2* oo = obs_out ? static_cast<double2*>(da.take(ns * sizeof(double2))) : nullptr;
        if (order == 4 && fp32) {
            // the RK4 kernel reads one storage type: widen the complex64 L4 into the FP64 L2
            taco::add_c64_into_c128(static_cast<const float2*>(L4), L2, (steps + 1) * E, st);
            L4 = nullptr;
        }
        taco::Rk4Request q;
        q.L = L2;
        q.L_add = L4;
        q.fp32_storage = false;
        q.steps = steps;
        q.D = D;
        q.dt = dt;
        q.r = r;
        q.sample_every = obs_out ? sample_every : 0;
        q.obs = o;
        q.obs_out = oo;
        taco::rk4_propagate_device({q}, st);
        if (obs_out)
            taco::cuda_check(cudaMemcpyAsync(obs_out, oo, ns * sizeof(double2), dev_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st), "obs out");
        if (rho_out)
            taco::cuda_check(cudaMemcpyAsync(rho_out, r, D * sizeof(double2), dev_out ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st), "rho out");
        taco::cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(propagate)");
    });
}

namespace {
// Device view of a caller array: the pointer itself (device flag) or a staged copy.
const void* dev_in(DevAllocs& da, const void* p, std::size_t bytes, bool on_device, cudaStream_t st) {
    if (on_device || p == nullptr) return p;
    void* d = da.take(bytes);
    taco::cuda_check(cudaMemcpyAsync(d, p, bytes, cudaMemcpyHostToDevice, st), "cudaMemcpyAsync(stage in)");
    return d;
}
}  // namespace

int taco_build_mikx(const taco_c128* F, const taco_c128* C, const taco_c128* R, const int* pair_to_freq, int N,
                    int nf, size_t T, taco_c128* M, taco_c128* I, taco_c128* K, taco_c128* X, int flags, void* stream) {
    return guarded([&] {
        require_device();
        if (N <= 0) throw taco::Error(taco::kInvalidArgument, "build_mikx: N must be > 0");
        if (nf <= 0 || T == 0) throw taco::Error(taco::kInvalidArgument, "build_mikx: empty input");
        if (!F || !C || !R || !pair_to_freq || !M || !I || !K || !X)
            throw taco::Error(taco::kInvalidArgument, "build_mikx: null pointer");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        const bool din = (flags & TACO_IN_DEVICE) != 0, dout = (flags & TACO_OUT_DEVICE) != 0;
        const std::size_t NN = static_cast<std::size_t>(N) * N;
        std::vector<int> p2f(NN);
        taco::cuda_check(cudaMemcpy(p2f.data(), pair_to_freq, NN * sizeof(int), din ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost),
                         "pair_to_freq");
        for (int v : p2f) {
            if (v < 0) throw taco::Error(taco::kRuntime, "tcl4::build_mikx: pair_to_freq contains -1 for a required pair");
            if (v >= nf) throw taco::Error(taco::kInvalidArgument, "build_mikx: pair_to_freq entry out of range");
        }
        const std::size_t nf3 = static_cast<std::size_t>(nf) * nf * nf, N4 = NN * NN, N6 = N4 * NN;
        DevAllocs da;
        auto f = static_cast<const double2*>(dev_in(da, F, T * nf3 * 16, din, st));
        auto c = static_cast<const double2*>(dev_in(da, C, T * nf3 * 16, din, st));
        auto r = static_cast<const double2*>(dev_in(da, R, T * nf3 * 16, din, st));
        auto pf = static_cast<const int*>(dev_in(da, p2f.data(), NN * sizeof(int), false, st));
        double2* outs[4];
        taco_c128* host[4] = {M, I, K, X};
        const std::size_t sz[4] = {T * N4, T * N4, T * N4, T * N6};
        for (int k = 0; k < 4; ++k)
            outs[k] = dout ? reinterpret_cast<double2*>(host[k]) : static_cast<double2*>(da.take(sz[k] * 16));
        taco::mikx_device(f, c, r, pf, N, nf, T, outs[0], outs[1], outs[2], outs[3], st);
        if (!dout)
            for (int k = 0; k < 4; ++k)
                taco::cuda_check(cudaMemcpyAsync(host[k], outs[k], sz[k] * 16, cudaMemcpyDeviceToHost, st), "mikx out");
        taco::cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(mikx)");
    });
}

int taco_assemble_liouvillian(const taco_c128* M, const taco_c128* I, const taco_c128* K, const taco_c128* X,
                              const taco_c128* ops, int N, int num_ops, size_t T, int symmetrize, taco_c128* GW,
                              int flags, void* stream) {
    return guarded([&] {
        require_device();
        if (N <= 0) throw taco::Error(taco::kInvalidArgument, "assemble_liouvillian: tensors.N must be > 0");
        if (num_ops <= 0) throw taco::Error(taco::kInvalidArgument, "assemble_liouvillian: coupling_ops must be non-empty");
        if (!M || !I || !K || !X || !ops || !GW || T == 0)
            throw taco::Error(taco::kInvalidArgument, "assemble_liouvillian: null or empty input");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        const bool din = (flags & TACO_IN_DEVICE) != 0, dout = (flags & TACO_OUT_DEVICE) != 0;
        const std::size_t NN = static_cast<std::size_t>(N) * N, N4 = NN * NN, N6 = N4 * NN;
        DevAllocs da;
        auto m = static_cast<const double2*>(dev_in(da, M, T * N4 * 16, din, st));
        auto i = static_cast<const double2*>(dev_in(da, I, T * N4 * 16, din, st));
        auto k = static_cast<const double2*>(dev_in(da, K, T * N4 * 16, din, st));
        auto x = static_cast<const double2*>(dev_in(da, X, T * N6 * 16, din, st));
        auto o = static_cast<const double2*>(dev_in(da, ops, num_ops * NN * 16, din, st));
        double2* gw = dout ? reinterpret_cast<double2*>(GW) : static_cast<double2*>(da.take(T * N4 * 16));
        double2* tmp = symmetrize ? static_cast<double2*>(da.take(T * N4 * 16)) : nullptr;
        taco::gw_device(m, i, k, x, o, N, num_ops, T, symmetrize != 0, gw, tmp, st);
        if (!dout) taco::cuda_check(cudaMemcpyAsync(GW, gw, T * N4 * 16, cudaMemcpyDeviceToHost, st), "GW out");
        taco::cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(assemble)");
    });
}

int taco_gw_to_liouvillian(const taco_c128* GW, int N, size_t T, taco_c128* L4, int flags, void* stream) {
    return guarded([&] {
        require_device();
        if (N <= 0) throw taco::Error(taco::kInvalidArgument, "gw_to_liouvillian: N must be > 0");
        if (!GW || !L4 || T == 0) throw taco::Error(taco::kInvalidArgument, "gw_to_liouvillian: null or empty input");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        const bool din = (flags & TACO_IN_DEVICE) != 0, dout = (flags & TACO_OUT_DEVICE) != 0;
        const std::size_t N4 = static_cast<std::size_t>(N) * N * N * N;
        DevAllocs da;
        auto g = static_cast<const double2*>(dev_in(da, GW, T * N4 * 16, din, st));
        double2* l = dout ? reinterpret_cast<double2*>(L4) : static_cast<double2*>(da.take(T * N4 * 16));
        taco::gw_to_l4_device(g, N, T, l, st);
        if (!dout) taco::cuda_check(cudaMemcpyAsync(L4, l, T * N4 * 16, cudaMemcpyDeviceToHost, st), "L4 out");
        taco::cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(gw_to_l4)");
    });
}

int taco_set_work_budget(size_t bytes) {
    return guarded([&] { taco::set_work_budget(bytes); });
}

int taco_release_workspace(void) {
    return guarded([&] {
        require_device();
        taco::release_workspace();
        taco::release_guard_scratch();
    });
}

int taco_set_fused_conv(int on) {
    return guarded([&] { taco::set_fused_conv(on != 0); });
}

int taco_get_fused_conv(int* on) {
    return guarded([&] {
        if (!on) throw taco::Error(taco::kInvalidArgument, "on is null");
        *on = taco::fused_conv() ? 1 : 0;
    });
}

int taco_set_fp32_guard(double tol) {
    return guarded([&] {
        if (!(tol >= 0.0)) throw taco::Error(taco::kInvalidArgument, "fp32 guard tolerance must be >= 0");
        taco::set_fp32_guard(tol);
    });
}

int taco_set_guard_chunk_bytes(size_t bytes) {
    return guarded([&] { taco::set_guard_chunk_bytes(bytes); });
}

int taco_fp32_guard_stats(uint64_t* counts6) {
    return guarded([&] {
        if (!counts6) throw taco::Error(taco::kInvalidArgument, "counts is null");
        const taco::GuardStats g = taco::fp32_guard_stats();
        const uint64_t v[6] = {g.instances, g.heads, g.head_rows, g.rows, g.full, g.rounds};
        for (int k = 0; k < 6; ++k) counts6[k] = v[k];
    });
}

int taco_get_fp32_guard(double* tol) {
    return guarded([&] {
        if (!tol) throw taco::Error(taco::kInvalidArgument, "tol is null");
        *tol = taco::fp32_guard();
    });
}

int taco_fft_length(size_t n_in, int precision, int flags, size_t* nfft, int* key) {
    return guarded([&] {
        if (n_in == 0) throw taco::Error(taco::kInvalidArgument, "fft_length: n_in must be > 0");
        const bool full = (flags & TACO_FULL_LENGTH_FFT) != 0;
        const std::size_t n = taco::fft_length_for(n_in, precision == TACO_PREC_FP32, !full, taco_get_fcr_fft_pad_factor(), key);
        if (nfft) *nfft = n;
    });
}

int taco_bcf_fft(const taco_bcf_request* reqs, size_t n, int flags, void* stream) {
    return guarded([&] {
        require_device();
        if (!reqs && n) throw taco::Error(taco::kInvalidArgument, "bcf: null requests");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        const bool dout = (flags & TACO_OUT_DEVICE) != 0;
        std::vector<taco::BcfRequest> rs(n);
        DevAllocs da;
        for (size_t k = 0; k < n; ++k) {
            const taco_bcf_request& q = reqs[k];
            taco::BcfRequest& r = rs[k];
            r.model = q.model;
            r.which = q.which;
            r.alpha = q.alpha;
            r.omega_c = q.omega_c;
            r.lambda = q.lambda;
            r.gamma = q.gamma;
            r.beta = q.beta;
            r.N = q.N;
            r.dt = q.dt;
            r.n_out = q.n_out;
            if (!q.out) throw taco::Error(taco::kInvalidArgument, "bcf: null output");
            r.out = dout ? reinterpret_cast<double2*>(q.out) : static_cast<double2*>(da.take(q.n_out * sizeof(double2)));
        }
        taco::bcf_device(rs, st);
        if (!dout)
            for (size_t k = 0; k < n; ++k)
                taco::cuda_check(cudaMemcpyAsync(reqs[k].out, rs[k].out, reqs[k].n_out * sizeof(double2),
                                                 cudaMemcpyDeviceToHost, st),
                                 "bcf out");
        taco::cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(bcf)");
    });
}

namespace {
std::vector<taco::Rk4GradJob> to_rk4g(const taco_rk4_grad_job* jobs, size_t n) {
    if (!jobs && n) throw taco::Error(taco::kInvalidArgument, "rk4 gradient: null jobs");
    std::vector<taco::Rk4GradJob> out(n);
    auto d2 = [](const taco_c128* p) { return reinterpret_cast<const double2*>(p); };
    auto m2 = [](taco_c128* p) { return reinterpret_cast<double2*>(p); };
    for (size_t k = 0; k < n; ++k) {
        const taco_rk4_grad_job& j = jobs[k];
        taco::Rk4GradJob& o = out[k];
        o.L = d2(j.L);
        o.L_add = d2(j.L_add);
        o.steps = j.steps;
        o.D = j.D;
        o.dt = j.dt;
        o.r0 = d2(j.r0);
        o.obs = d2(j.obs);
        o.sample_every = j.sample_every;
        o.ckpt = m2(j.ckpt);
        o.obs_out = m2(j.obs_out);
        o.r_out = m2(j.r_out);
        o.obs_bar = d2(j.obs_bar);
        o.r_final_bar = d2(j.r_final_bar);
        o.L_bar = m2(j.L_bar);
        o.r0_bar = m2(j.r0_bar);
        o.obs_vec_bar = m2(j.obs_vec_bar);
    }
    return out;
}
}  // namespace

int taco_rk4_forward_checkpointed(const taco_rk4_grad_job* jobs, size_t n, size_t checkpoint_every, void* stream) {
    return guarded([&] {
        require_device();
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        taco::rk4_forward_checkpointed(to_rk4g(jobs, n), checkpoint_every, st);
    });
}

int taco_rk4_adjoint(const taco_rk4_grad_job* jobs, size_t n, size_t checkpoint_every, void* stream) {
    return guarded([&] {
        require_device();
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        taco::rk4_adjoint(to_rk4g(jobs, n), checkpoint_every, st);
    });
}

int taco_tcl4_adjoint(const taco_tcl4_adjoint_job* jobs, size_t n, void* stream) {
    return guarded([&] {
        require_device();
        if (!jobs && n) throw taco::Error(taco::kInvalidArgument, "tcl4 adjoint: null jobs");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        std::vector<taco::SystemDesc> sys(n);
        std::vector<taco::Tcl4AdjointJob> js(n);
        for (size_t k = 0; k < n; ++k) {
            const taco_tcl4_adjoint_job& j = jobs[k];
            sys[k] = to_desc(j.sys);
            taco::Tcl4AdjointJob& o = js[k];
            o.sys = &sys[k];
            o.gamma = reinterpret_cast<const double2*>(j.gamma);
            o.T = j.T;
            o.dt = j.dt;
            o.L_bar = reinterpret_cast<const double2*>(j.L_bar);
            o.F = reinterpret_cast<const double2*>(j.F);
            o.C = reinterpret_cast<const double2*>(j.C);
            o.R = reinterpret_cast<const double2*>(j.R);
            o.gamma_bar = reinterpret_cast<double2*>(j.gamma_bar);
            o.omega_bar = j.omega_bar;
            o.ops_bar = reinterpret_cast<double2*>(j.ops_bar);
        }
        taco::tcl4_adjoint(js, st);
    });
}

int taco_tcl2_adjoint(const taco_tcl2_adjoint_job* jobs, size_t n, void* stream) {
    return guarded([&] {
        require_device();
        if (!jobs && n) throw taco::Error(taco::kInvalidArgument, "tcl2 adjoint: null jobs");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        std::vector<taco::SystemDesc> sys(n);
        std::vector<taco::Tcl2AdjointJob> js(n);
        for (size_t k = 0; k < n; ++k) {
            const taco_tcl2_adjoint_job& j = jobs[k];
            sys[k] = to_desc(j.sys);
            taco::Tcl2AdjointJob& o = js[k];
            o.sys = &sys[k];
            o.eps = j.eps;
            o.gamma = reinterpret_cast<const double2*>(j.gamma);
            o.T = j.T;
            o.L_bar = reinterpret_cast<const double2*>(j.L_bar);
            o.gamma_bar = reinterpret_cast<double2*>(j.gamma_bar);
            o.ops_bar = reinterpret_cast<double2*>(j.ops_bar);
            o.eps_bar = j.eps_bar;
        }
        taco::tcl2_adjoint(js, st);
    });
}

int taco_inner_re(const taco_inner_job* jobs, size_t n, double* out, void* stream) {
    return guarded([&] {
        require_device();
        if ((!jobs || !out) && n) throw taco::Error(taco::kInvalidArgument, "inner: null pointer");
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : taco::default_stream();
        std::vector<taco::InnerRequest> rs(n);
        for (size_t k = 0; k < n; ++k)
            rs[k] = taco::InnerRequest{reinterpret_cast<const double2*>(jobs[k].a),
                                       reinterpret_cast<const double2*>(jobs[k].b), jobs[k].n};
        taco::inner_re_device(rs, out, st);
    });
}

int taco_l4_coefficients(const taco_system_view* sys, int32_t* rowptr, uint32_t* src, taco_c128* coef, size_t cap,
                         size_t* nnz) {
    return guarded([&] {
        taco::SystemDesc s = to_desc(sys);
        for (int v : s.p2f)
            if (v < 0 || v >= s.nf) throw taco::Error(taco::kRuntime, "pair_to_freq contains -1 or an invalid bucket");
        taco::CoefTable t;
        taco::build_coef_table(s.N, s.nf, s.p2f.data(), s.ops.data(), s.num_ops, t);
        if (nnz) *nnz = t.src.size();
        if (rowptr) std::memcpy(rowptr, t.rowptr.data(), t.rowptr.size() * sizeof(int32_t));
        if (t.src.size() <= cap) {
            if (src) std::memcpy(src, t.src.data(), t.src.size() * sizeof(uint32_t));
            if (coef) std::memcpy(coef, t.coef.data(), t.coef.size() * sizeof(taco_c128));
        }
    });
}

int taco_set_tuning(int log2_nfft, int precision, int col_tile, int row_tile, size_t chunk_bytes, int inv_dft_rows) {
    return guarded([&] {
        // schedule key: log2 of a power-of-two length (3..22), + 64 for 3 * 2^k, + 128 for 5 * 2^k
        if ((log2_nfft & 63) < 3 || (log2_nfft & 63) > 22 || log2_nfft >= 192)
            throw taco::Error(taco::kInvalidArgument, "tuning: schedule key out of range");
        taco::Tuning t = taco::get_tuning(log2_nfft, precision == TACO_PREC_FP32);
        t.col_tile = col_tile;
        t.row_tile = row_tile;
        t.chunk_bytes = chunk_bytes;
        t.inv_dft_rows = inv_dft_rows;
        taco::set_tuning(log2_nfft, precision == TACO_PREC_FP32, t);
    });
}

int taco_set_fft_length_enabled(int key, int precision, int enabled) {
    return guarded([&] {
        if ((key & 63) < 3 || (key & 63) > 22 || key >= 192 || key < 64)
            throw taco::Error(taco::kInvalidArgument, "fft length key must name a 3*2^k or 5*2^k length");
        taco::Tuning t = taco::get_tuning(key, precision == TACO_PREC_FP32);
        t.enabled = enabled ? 1 : 0;
        taco::set_tuning(key, precision == TACO_PREC_FP32, t);
    });
}

int taco_get_tuning(int log2_nfft, int precision, int* col_tile, int* row_tile, size_t* chunk_bytes,
                    int* inv_dft_rows) {
    return guarded([&] {
        const taco::Tuning t = taco::get_tuning(log2_nfft, precision == TACO_PREC_FP32);
        if (col_tile) *col_tile = t.col_tile;
        if (row_tile) *row_tile = t.row_tile;
        if (chunk_bytes) *chunk_bytes = t.chunk_bytes;
        if (inv_dft_rows) *inv_dft_rows = t.inv_dft_rows;
    });
}

int taco_set_cluster_points(int log2_nfft, int precision, int log2_points) {
    return guarded([&] {
        // schedule key: log2 of a power-of-two length (3..22), + 64 for 3 * 2^k, + 128 for 5 * 2^k
        if ((log2_nfft & 63) < 3 || (log2_nfft & 63) > 22 || log2_nfft >= 192)
            throw taco::Error(taco::kInvalidArgument, "tuning: schedule key out of range");
        if (log2_points < -1 || log2_points > 13)
            throw taco::Error(taco::kInvalidArgument, "tuning: log2_points must be -1 (automatic), 0 (off) or 3..13");
        taco::Tuning t = taco::get_tuning(log2_nfft, precision == TACO_PREC_FP32);
        t.cluster_lm = log2_points;
        taco::set_tuning(log2_nfft, precision == TACO_PREC_FP32, t);
    });
}

int taco_clear_tuning(void) {
    return guarded([&] { taco::clear_tuning(); });
}

int taco_kernel_launches(uint64_t* launches) {
    return guarded([&] {
        if (launches) *launches = taco::kernel_launches();
    });
}

int taco_profile_enable(int on) {
    return guarded([&] { taco::profile_enable(on != 0); });
}

int taco_profile_reset(void) {
    return guarded([&] { taco::profile_reset(); });
}

int taco_profile_get(size_t index, const char** name, uint64_t* launches, double* total_ms, size_t* count) {
    return guarded([&] {
        const auto e = taco::profile_entries();
        if (count) *count = e.size();
        if (index < e.size()) {
            if (name) *name = e[index].name;
            if (launches) *launches = e[index].launches;
            if (total_ms) *total_ms = e[index].total_ms;
        }
    });
}

}  // extern "C"
