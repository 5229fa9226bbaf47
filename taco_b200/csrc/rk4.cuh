// rk4.cuh -- fixed-step RK4 for r' = L(t) r with the generator series resident on the
// device (cpp/src/core/rk4_dense.cpp:133-160 and :246-321):
//   k1 = L_i r; k2 = Lh (r + dt/2 k1); k3 = Lh (r + dt/2 k2); k4 = L_{i+1} (r + dt k3);
//   r += dt/6 (k1 + 2 k2 + 2 k3 + k4),   Lh = L_half[i] or (L_i + L_{i+1}) / 2.
// The state and its accumulation are FP64 whatever the storage type of L.  Optional
// L_add is added entrywise to L (the propagated generator L2 + L4).  Samples of r (and
// of <O> = sum_l obs_l r_l) are written every sample_every steps plus the final state.
#pragma once

#include "common.cuh"

namespace taco {

struct Rk4Job {
    const void* L;       // [steps+1][D*D] column-major, storage complex type
    const void* L_half;  // [steps][D*D] or nullptr
    const void* L_add;   // [steps+1][D*D] or nullptr (added to L; midpoints by averaging)
    uint64_t steps;
    double dt;
    double2* r;          // [D] in/out
    uint64_t sample_every;  // 0: no samples
    double2* samples;    // [n_samples][D] or nullptr
    const double2* obs;  // [D] or nullptr
    double2* obs_out;    // [n_samples] or nullptr
};

template <class S>
__device__ __forceinline__ double2 ld_d2(const S* p, size_t i) { return to_d2(p[i]); }

// Row `row` of the generator at endpoint `step` (entries (row, c), c < D).
template <class S, int DMAX>
__device__ __forceinline__ void load_row(const Rk4Job& j, int D, uint64_t step, int row, double2* out) {
    const size_t base = static_cast<size_t>(step) * D * D + row;
    const S* L = static_cast<const S*>(j.L);
    const S* La = static_cast<const S*>(j.L_add);
#pragma unroll
    for (int c = 0; c < DMAX; ++c) {
        if (c < D) {
            double2 v = to_d2(L[base + static_cast<size_t>(c) * D]);
            if (La) v = cadd(v, to_d2(La[base + static_cast<size_t>(c) * D]));
            out[c] = v;
        }
    }
}

template <int DMAX>
__device__ __forceinline__ double2 warp_matvec(const double2* row, double2 x, int D) {
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < DMAX; ++c) {
        if (c < D) {
            double2 xc;
            xc.x = __shfl_sync(0xffffffffu, x.x, c);
            xc.y = __shfl_sync(0xffffffffu, x.y, c);
            acc = cadd(acc, cmul(row[c], xc));
        }
    }
    return acc;
}

__device__ __forceinline__ void write_sample(const Rk4Job& j, int D, uint64_t s, double2 r, int lane) {
    if (j.samples && lane < D) j.samples[s * D + lane] = r;
    if (j.obs_out) {
        double2 v = lane < D ? cmul(j.obs[lane], r) : make_double2(0.0, 0.0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
            v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
        }
        if (lane == 0) j.obs_out[s] = v;
    }
}

// One warp per instance, lane l < D owns row l; rows of L_i and L_{i+1} live in
// registers and the row of L_{i+2} is fetched while step i runs.
template <class S, int DMAX>
__global__ void k_rk4_warp(const Rk4Job* __restrict__ jobs, int njobs, int D) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= njobs) return;
    const Rk4Job j = jobs[w];
    const int row = lane < D ? lane : 0;
    double2 l0[DMAX], l1[DMAX], l2[DMAX];
    load_row<S, DMAX>(j, D, 0, row, l0);
    load_row<S, DMAX>(j, D, 1, row, l1);
    double2 r = lane < D ? j.r[lane] : make_double2(0.0, 0.0);
    const double dt = j.dt;
    uint64_t ns = 0;
    const S* Lh = static_cast<const S*>(j.L_half);
    for (uint64_t i = 0; i < j.steps; ++i) {
        if (j.sample_every && (i % j.sample_every) == 0) write_sample(j, D, ns++, r, lane);
        if (i + 2 <= j.steps) load_row<S, DMAX>(j, D, i + 2, row, l2);
        double2 lh[DMAX];
        if (Lh) {
            const size_t base = static_cast<size_t>(i) * D * D + row;
#pragma unroll
            for (int c = 0; c < DMAX; ++c)
                if (c < D) lh[c] = to_d2(Lh[base + static_cast<size_t>(c) * D]);
        } else {
#pragma unroll
            for (int c = 0; c < DMAX; ++c)
                if (c < D) lh[c] = make_double2(0.5 * (l0[c].x + l1[c].x), 0.5 * (l0[c].y + l1[c].y));
        }
        const double2 k1 = warp_matvec<DMAX>(l0, r, D);
        const double2 k2 = warp_matvec<DMAX>(lh, cadd(r, cscale(k1, 0.5 * dt)), D);
        const double2 k3 = warp_matvec<DMAX>(lh, cadd(r, cscale(k2, 0.5 * dt)), D);
        const double2 k4 = warp_matvec<DMAX>(l1, cadd(r, cscale(k3, dt)), D);
        const double2 sum = cadd(cadd(k1, cscale(k2, 2.0)), cadd(cscale(k3, 2.0), k4));
        r = cadd(r, cscale(sum, dt / 6.0));
#pragma unroll
        for (int c = 0; c < DMAX; ++c) {
            l0[c] = l1[c];
            l1[c] = l2[c];
        }
    }
    if (j.sample_every) write_sample(j, D, ns, r, lane);
    if (lane < D) j.r[lane] = r;
}

// ------------------------------------------------ step matrices (D <= 4) --
// For r' = L(t) r one RK4 step is r_{n+1} = M_n r_n, M_n = I + dt/6 (K1 + 2 K2 + 2 K3 + K4)
// with K1 = L0, K2 = Lh + dt/2 Lh K1, K3 = Lh + dt/2 Lh K2, K4 = L1 + dt L1 K3 (Lh the given
// midpoint, or (L0 + L1)/2).  k_rk4_stepmat builds every M_n in parallel (FP64 from the
// storage type); k_rk4_chain applies one matrix per sequential step, the matrices streamed
// through a per-warp shared-memory ring by cp.async, and stores the sampled states;
// k_rk4_samples writes the samples and observables.  Records of 16 entries, column-major.
constexpr int RK_RING = 8;
constexpr int RK_REC = 16;

template <class S>
__device__ __forceinline__ void rk_load(const Rk4Job& j, int D, uint64_t t, double2* A) {
    const S* L = static_cast<const S*>(j.L);
    const S* La = static_cast<const S*>(j.L_add);
    const size_t DD = static_cast<size_t>(D) * D;
    for (size_t e = 0; e < DD; ++e) {
        double2 v = to_d2(L[t * DD + e]);
        if (La) v = cadd(v, to_d2(La[t * DD + e]));
        A[e] = v;
    }
}

// C = A + a A B (column-major D x D)
__device__ __forceinline__ void rk_stage(const double2* A, const double2* B, double a, int D, double2* C) {
    for (int c = 0; c < D; ++c)
        for (int r = 0; r < D; ++r) {
            double2 acc = make_double2(0.0, 0.0);
            for (int k = 0; k < D; ++k) acc = cadd(acc, cmul(A[r + k * D], B[k + c * D]));
            C[r + c * D] = cadd(A[r + c * D], cscale(acc, a));
        }
}

template <class S>
__global__ void k_rk4_stepmat(const Rk4Job* __restrict__ jobs, int D, uint64_t mstride, double2* __restrict__ M) {
    const Rk4Job& j = jobs[blockIdx.y];
    const uint64_t n = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n >= j.steps) return;
    const int DD = D * D;
    const double dt = j.dt;
    double2 L0[RK_REC], L1[RK_REC], Lh[RK_REC], Ka[RK_REC], Kb[RK_REC], Sm[RK_REC];
    rk_load<S>(j, D, n, L0);
    rk_load<S>(j, D, n + 1, L1);
    const S* Lhalf = static_cast<const S*>(j.L_half);
    for (int e = 0; e < DD; ++e) {
        Lh[e] = Lhalf ? to_d2(Lhalf[n * DD + e]) : make_double2(0.5 * (L0[e].x + L1[e].x), 0.5 * (L0[e].y + L1[e].y));
        Sm[e] = L0[e];  // K1
    }
    rk_stage(Lh, L0, 0.5 * dt, D, Ka);  // K2
    for (int e = 0; e < DD; ++e) Sm[e] = cadd(Sm[e], cscale(Ka[e], 2.0));
    rk_stage(Lh, Ka, 0.5 * dt, D, Kb);  // K3
    for (int e = 0; e < DD; ++e) Sm[e] = cadd(Sm[e], cscale(Kb[e], 2.0));
    rk_stage(L1, Kb, dt, D, Ka);  // K4
    double2* out = M + (static_cast<size_t>(blockIdx.y) * mstride + n) * RK_REC;
    for (int c = 0; c < D; ++c)
        for (int r = 0; r < D; ++r) {
            double2 v = cscale(cadd(Sm[r + c * D], Ka[r + c * D]), dt / 6.0);
            if (r == c) v.x += 1.0;
            out[r + c * D] = v;
        }
}

// One warp per job (four per CTA); sampled states go to Rs (the job's [sstride][4] array).
__global__ void __launch_bounds__(128) k_rk4_chain(const Rk4Job* __restrict__ jobs, int njobs, int D,
                                                   const double2* __restrict__ M, uint64_t mstride,
                                                   double2* __restrict__ Rs, uint64_t sstride) {
    __shared__ __align__(16) double2 ring_all[4][RK_RING * RK_REC];
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= njobs) return;
    double2* ring = ring_all[threadIdx.x >> 5];
    const Rk4Job j = jobs[w];
    const int DD = D * D;
    const int row = lane < D ? lane : 0;
    const uint64_t steps = j.steps, se = j.sample_every;
    const double2* Mj = M + static_cast<size_t>(w) * mstride * RK_REC;
    double2* Rj = Rs + static_cast<size_t>(w) * sstride * 4;
    auto fetch = [&](uint64_t t) {
        if (t < steps && lane < DD) cp_async16(ring + (t % RK_RING) * RK_REC + lane, Mj + t * RK_REC + lane);
    };
    for (uint64_t t = 0; t + 1 < RK_RING; ++t) {
        fetch(t);
        cp_async_commit();
    }
    double2 r = lane < D ? j.r[lane] : make_double2(0.0, 0.0);
    uint64_t s_left = 0, ns = 0;
    for (uint64_t i = 0; i < steps; ++i) {
        fetch(i + RK_RING - 1);
        cp_async_commit();
        cp_async_wait<RK_RING - 2>();
        __syncwarp();
        if (se) {
            if (s_left == 0) {
                if (lane < D) Rj[ns * 4 + lane] = r;
                ++ns;
                s_left = se;
            }
            --s_left;
        }
        const double2* m = ring + (i % RK_RING) * RK_REC;
        double2 mrow[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) mrow[c] = c < D ? m[row + c * D] : make_double2(0.0, 0.0);
        r = warp_matvec<4>(mrow, r, D);
        __syncwarp();
    }
    cp_async_wait<0>();
    if (se && lane < D) Rj[ns * 4 + lane] = r;
    if (lane < D) j.r[lane] = r;
}

// samples[s] and obs_out[s] from the sampled states: one thread per (s, job)
__global__ void k_rk4_samples(const Rk4Job* __restrict__ jobs, int D, const double2* __restrict__ Rs, uint64_t sstride) {
    const Rk4Job& j = jobs[blockIdx.y];
    const uint64_t se = j.sample_every;
    if (!se) return;
    const uint64_t s = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= (j.steps + se - 1) / se + 1) return;
    const double2* r = Rs + (static_cast<size_t>(blockIdx.y) * sstride + s) * 4;
    if (j.samples)
        for (int l = 0; l < D; ++l) j.samples[s * D + l] = r[l];
    if (j.obs_out) {
        double2 v = make_double2(0.0, 0.0);
        for (int l = 0; l < D; ++l) v = cadd(v, cmul(j.obs[l], r[l]));
        j.obs_out[s] = v;
    }
}

// One CTA per instance for larger D: state in shared memory, thread t owns rows
// t, t + blockDim.x, ...; generator entries read from global (L2-resident rows).
template <class S>
__global__ void k_rk4_cta(const Rk4Job* __restrict__ jobs, int D) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* r = reinterpret_cast<double2*>(smem_raw);
    double2* x = r + D;
    double2* k = x + D;  // k1..k4: [4][D]
    const Rk4Job j = jobs[blockIdx.x];
    const S* L = static_cast<const S*>(j.L);
    const S* La = static_cast<const S*>(j.L_add);
    const S* Lh = static_cast<const S*>(j.L_half);
    for (int t = threadIdx.x; t < D; t += blockDim.x) r[t] = j.r[t];
    __syncthreads();
    const double dt = j.dt;
    const size_t DD = static_cast<size_t>(D) * D;
    uint64_t ns = 0;
    auto gen = [&](const S* P, const S* Pa, size_t step, size_t e) {
        double2 v = to_d2(P[step * DD + e]);
        if (Pa) v = cadd(v, to_d2(Pa[step * DD + e]));
        return v;
    };
    for (uint64_t i = 0; i < j.steps; ++i) {
        if (j.sample_every && (i % j.sample_every) == 0) {
            for (int t = threadIdx.x; t < D; t += blockDim.x)
                if (j.samples) j.samples[ns * D + t] = r[t];
            if (j.obs_out && threadIdx.x == 0) {
                double2 acc = make_double2(0.0, 0.0);
                for (int t = 0; t < D; ++t) acc = cadd(acc, cmul(j.obs[t], r[t]));
                j.obs_out[ns] = acc;
            }
            ++ns;
        }
        for (int stage = 0; stage < 4; ++stage) {
            // x = r + c * k_{stage-1}
            const double c = stage == 0 ? 0.0 : (stage == 3 ? dt : 0.5 * dt);
            for (int t = threadIdx.x; t < D; t += blockDim.x)
                x[t] = stage == 0 ? r[t] : cadd(r[t], cscale(k[(stage - 1) * D + t], c));
            __syncthreads();
            for (int row = threadIdx.x; row < D; row += blockDim.x) {
                double2 acc = make_double2(0.0, 0.0);
                for (int col = 0; col < D; ++col) {
                    const size_t e = row + static_cast<size_t>(col) * D;
                    double2 m;
                    if (stage == 0) m = gen(L, La, i, e);
                    else if (stage == 3) m = gen(L, La, i + 1, e);
                    else if (Lh) m = to_d2(Lh[i * DD + e]);
                    else {
                        const double2 a = gen(L, La, i, e), b = gen(L, La, i + 1, e);
                        m = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
                    }
                    acc = cadd(acc, cmul(m, x[col]));
                }
                k[stage * D + row] = acc;
            }
            __syncthreads();
        }
        for (int t = threadIdx.x; t < D; t += blockDim.x) {
            const double2 s = cadd(cadd(k[t], cscale(k[D + t], 2.0)), cadd(cscale(k[2 * D + t], 2.0), k[3 * D + t]));
            r[t] = cadd(r[t], cscale(s, dt / 6.0));
        }
        __syncthreads();
    }
    if (j.sample_every) {
        for (int t = threadIdx.x; t < D; t += blockDim.x)
            if (j.samples) j.samples[ns * D + t] = r[t];
        if (j.obs_out && threadIdx.x == 0) {
            double2 acc = make_double2(0.0, 0.0);
            for (int t = 0; t < D; ++t) acc = cadd(acc, cmul(j.obs[t], r[t]));
            j.obs_out[ns] = acc;
        }
    }
    for (int t = threadIdx.x; t < D; t += blockDim.x) j.r[t] = r[t];
}

}  // namespace taco
