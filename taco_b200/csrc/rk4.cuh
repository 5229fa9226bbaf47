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
