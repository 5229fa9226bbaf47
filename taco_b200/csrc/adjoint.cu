// adjoint.cu -- reverse-mode derivatives of the propagated TCL4 path:
//   RK4 (checkpointed) -> L(t) = L2(t) + L4(t) -> sources F/C/R(t) -> Gamma(t), Bohr frequencies.
//
// Convention: for a real loss l and a complex quantity z, G(z) = dl/dRe z + i dl/dIm z.
// Then y = a z gives G(z) += conj(a) G(y), y = a conj(z) gives G(z) += a conj(G(y)),
// y = M x gives G(x) += M^H G(y) and G(M) += G(y) x^H.
//
// RK4 (cpp/src/core/rk4_dense.cpp:133-160, endpoint overload with Lh = (L_i + L_{i+1})/2):
//   k1 = L0 u1, u1 = r;  k2 = Lh u2, u2 = r + dt/2 k1;  k3 = Lh u3, u3 = r + dt/2 k2;
//   k4 = L1 u4, u4 = r + dt k3;  r' = r + dt/6 (k1 + 2 k2 + 2 k3 + k4).
// The forward sweep stores r every `every` steps (every ~ sqrt(steps)); the reverse sweep
// recomputes one segment of states from its checkpoint into shared memory and walks it
// backwards, so memory is O(sqrt(steps) D) instead of O(steps D).
//
// F/C/R (cpp/src/tcl/tcl4_kernels.cpp:105-281, direct forms): with P[k] = e^{-i w k dt},
// Q = conj(P), w = w_i + w_j + w_k, g1 = Gamma_i and
//   F[k] = dt sum_{m<=k} g2[m] P[k-m] (g1[k] - g1[k-m]),  g2 = Gamma_{mirror(j)}
//   C[k] = same with g2 = conj(Gamma_j)
//   R[k] = dt sum_{m<=k} g2[m] P[m] (g1[k] - g1[m]),      g2 = Gamma_j.
// Their adjoints split into prefix/suffix scans (O(T), k_fcr_adj_scan) and three
// correlations per F/C series, c[m] = sum_{k>=m} a[k-m] Fb[k] with a in {conj(g2),
// conj(P g1), (k-m) conj(P g1)} (O(T^2), k_fcr_adj_corr):
//   G(g1)[n] = conj(dt P[n] A0[n]) Fb[n] - dt Q[n] c1[n],        A0[n] = sum_{m<=n} g2[m] Q[m]
//   G(g2)[m] = dt P[m] sum_{k>=m} Q[k] conj(g1[k]) Fb[k] - dt c2[m]
//   dl/dw   = Re[-i dt^2 sum_k conj(Fb[k]) g1[k] P[k] (k A0[k] - A1[k]) + i dt^2 sum_m g2[m] conj(c3[m])],
//             A1[n] = sum_{m<=n} m g2[m] Q[m]
// and for R, with B0[k] = sum_{m<=k} g2[m] P[m], SR0[m] = sum_{k>=m} conj(g1[k]) Rb[k],
// SR1[m] = sum_{k>=m} Rb[k]:
//   G(g1)[k] = dt conj(B0[k]) Rb[k] - dt conj(g2[k] P[k]) SR1[k]
//   G(g2)[m] = dt Q[m] SR0[m] - dt conj(g1[m] P[m]) SR1[m]
//   dl/dw    = Re sum_m (-i m dt^2) g2[m] P[m] (conj(SR0[m]) - g1[m] conj(SR1[m])).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <thread>
#include <map>
#include <memory>
#include <vector>

#include "common.cuh"
#include "engine.hpp"
#include "gw_coef.hpp"
#include "fused_conv.cuh"

namespace taco {

namespace {

// ------------------------------------------------------------------ scratch --
struct GradScratch {
    void* p = nullptr;
    std::size_t cap = 0;
    char* ensure(std::size_t bytes) {
        if (bytes > cap) {
            if (p) cudaFree(p);
            p = nullptr;
            cap = 0;
            cuda_check(cudaMalloc(&p, bytes), "cudaMalloc(adjoint scratch)");
            cap = bytes;
        }
        return static_cast<char*>(p);
    }
    ~GradScratch() {
        if (p) cudaFree(p);
    }
};

GradScratch& grad_scratch() {
    thread_local std::map<int, GradScratch> per_dev;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    return per_dev[dev];
}

std::size_t up256(std::size_t x) { return (x + 255) / 256 * 256; }

struct Carve {
    char* base;
    std::size_t off = 0;
    template <class T>
    T* take(std::size_t n) {
        off = up256(off);
        T* r = reinterpret_cast<T*>(base ? base + off : nullptr);
        off += n * sizeof(T);
        return r;
    }
};

__device__ __forceinline__ double2 shfl2(double2 v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

__device__ __forceinline__ double2 shfl_up2(double2 v, int d) {
    return make_double2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}

__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

__device__ __forceinline__ double2 cfma2(double2 a, double2 b, double2 c) {  // c + a b
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}

// ---------------------------------------------------------------------- RK4 --
struct Rk4GJob {
    const double2* L;
    const double2* L_add;
    uint64_t steps;
    int D;
    double dt;
    const double2* r0;
    const double2* obs;
    uint64_t sample_every;
    double2* ckpt;
    double2* obs_out;
    double2* r_out;
    const double2* obs_bar;
    const double2* r_final_bar;
    double2* L_bar;
    double2* r0_bar;
    double2* obs_vec_bar;
};

// entry (r, c) of L + L_add at endpoint t
__device__ __forceinline__ double2 gen_at(const Rk4GJob& j, uint64_t t, int r, int c) {
    const size_t e = static_cast<size_t>(t) * j.D * j.D + r + static_cast<size_t>(c) * j.D;
    double2 v = j.L[e];
    if (j.L_add) v = cadd(v, j.L_add[e]);
    return v;
}

template <int DMAX>
__device__ __forceinline__ void load_row(const Rk4GJob& j, uint64_t t, int row, double2* out) {
#pragma unroll
    for (int c = 0; c < DMAX; ++c) out[c] = c < j.D ? gen_at(j, t, row, c) : make_double2(0.0, 0.0);
}

template <int DMAX>
__device__ __forceinline__ void load_col(const Rk4GJob& j, uint64_t t, int col, double2* out) {
#pragma unroll
    for (int r = 0; r < DMAX; ++r) out[r] = r < j.D ? gen_at(j, t, r, col) : make_double2(0.0, 0.0);
}

// (M x)_lane with lane owning row `lane` of M
template <int DMAX>
__device__ __forceinline__ double2 mv_row(const double2* row, double2 x, int D) {
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < DMAX; ++c)
        if (c < D) acc = cfma2(row[c], shfl2(x, c), acc);
    return acc;
}

// (M^H g)_lane with lane owning column `lane` of M
template <int DMAX>
__device__ __forceinline__ double2 mhv_col(const double2* col, double2 g, int D) {
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < DMAX; ++r)
        if (r < D) acc = cfma2(cconj(col[r]), shfl2(g, r), acc);
    return acc;
}

template <int DMAX>
__device__ __forceinline__ double2 rk4_step(double2 r, const double2* l0, const double2* l1, double dt, int D) {
    double2 lh[DMAX];
#pragma unroll
    for (int c = 0; c < DMAX; ++c) lh[c] = make_double2(0.5 * (l0[c].x + l1[c].x), 0.5 * (l0[c].y + l1[c].y));
    const double2 k1 = mv_row<DMAX>(l0, r, D);
    const double2 k2 = mv_row<DMAX>(lh, cadd(r, cscale(k1, 0.5 * dt)), D);
    const double2 k3 = mv_row<DMAX>(lh, cadd(r, cscale(k2, 0.5 * dt)), D);
    const double2 k4 = mv_row<DMAX>(l1, cadd(r, cscale(k3, dt)), D);
    const double2 s = cadd(cadd(k1, cscale(k2, 2.0)), cadd(cscale(k3, 2.0), k4));
    return cadd(r, cscale(s, dt / 6.0));
}

__host__ __device__ __forceinline__ uint64_t n_samples(uint64_t steps, uint64_t se) { return se ? (steps + se - 1) / se + 1 : 0; }

// Forward sweep: one warp per job, lane l < D owns component l of r.
template <int DMAX>
__global__ void __launch_bounds__(128) k_rk4g_fwd(const Rk4GJob* __restrict__ jobs, int njobs, uint64_t every) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= njobs) return;
    const Rk4GJob j = jobs[w];
    const int D = j.D;
    const int row = lane < D ? lane : 0;
    double2 l0[DMAX], l1[DMAX], l2[DMAX];
    load_row<DMAX>(j, 0, row, l0);
    load_row<DMAX>(j, 1, row, l1);
    double2 r = lane < D ? j.r0[lane] : make_double2(0.0, 0.0);
    const uint64_t se = j.sample_every;
    auto sample = [&](uint64_t s) {
        if (!j.obs_out) return;
        const double2 v = warp_sum2(lane < D ? cmul(j.obs[lane], r) : make_double2(0.0, 0.0));
        if (lane == 0) j.obs_out[s] = v;
    };
    for (uint64_t i = 0; i < j.steps; ++i) {
        // the row of L(t_{i+2}) arrives while step i runs
        if (i + 2 <= j.steps) load_row<DMAX>(j, i + 2, row, l2);
        if (j.ckpt && (i % every) == 0 && lane < D) j.ckpt[(i / every) * D + lane] = r;
        if (se && (i % se) == 0) sample(i / se);
        r = rk4_step<DMAX>(r, l0, l1, j.dt, D);
#pragma unroll
        for (int c = 0; c < DMAX; ++c) {
            l0[c] = l1[c];
            l1[c] = l2[c];
        }
    }
    if (se) sample(n_samples(j.steps, se) - 1);
    if (j.r_out && lane < D) j.r_out[lane] = r;
}

// Reverse sweep: one warp per block and job; shared memory holds one segment of states.
template <int DMAX>
__global__ void __launch_bounds__(32) k_rk4g_adj(const Rk4GJob* __restrict__ jobs, uint64_t every) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* seg = reinterpret_cast<double2*>(smem_raw);  // [every][DMAX]
    const Rk4GJob j = jobs[blockIdx.x];
    const int lane = threadIdx.x;
    const int D = j.D;
    const int me = lane < D ? lane : 0;
    const bool own = lane < D;
    const uint64_t steps = j.steps, se = j.sample_every;
    const uint64_t nck = (steps + every - 1) / every;
    const uint64_t nsamp = n_samples(steps, se);
    const double dt = j.dt;
    const size_t DD = static_cast<size_t>(D) * D;
    const double2 ob_l = (j.obs && own) ? j.obs[lane] : make_double2(0.0, 0.0);
    double2 g = (j.r_final_bar && own) ? j.r_final_bar[lane] : make_double2(0.0, 0.0);
    double2 ovb = make_double2(0.0, 0.0);
    double2 pend[DMAX];
#pragma unroll
    for (int c = 0; c < DMAX; ++c) pend[c] = make_double2(0.0, 0.0);
    for (uint64_t sg = nck; sg-- > 0;) {
        const uint64_t s0 = sg * every, s1 = min(s0 + every, steps);
        // recompute the segment's states from its checkpoint
        double2 r = own ? j.ckpt[sg * D + lane] : make_double2(0.0, 0.0);
        {
            double2 l0[DMAX], l1[DMAX];
            load_row<DMAX>(j, s0, me, l0);
            load_row<DMAX>(j, s0 + 1, me, l1);
            for (uint64_t i = s0; i < s1; ++i) {
                if (own) seg[(i - s0) * DMAX + lane] = r;
                r = rk4_step<DMAX>(r, l0, l1, dt, D);
#pragma unroll
                for (int c = 0; c < DMAX; ++c) l0[c] = l1[c];
                if (i + 2 <= s1) load_row<DMAX>(j, i + 2, me, l1);
            }
        }
        if (sg == nck - 1 && se && j.obs_bar) {  // the final sample, taken at r_steps
            const double2 o = j.obs_bar[nsamp - 1];
            g = cadd(g, cmulc(o, ob_l));   // conj(obs_l) o
            ovb = cadd(ovb, cmulc(o, r));  // conj(r_l) o
        }
        __syncwarp();
        double2 r0w[DMAX], r1w[DMAX], c0[DMAX], c1[DMAX];  // rows / columns of L(t_n), L(t_{n+1})
        double2 rp[DMAX], cp[DMAX];                        // L(t_{n-1}), fetched during step n
        load_row<DMAX>(j, s1, me, r1w);
        load_col<DMAX>(j, s1, me, c1);
        load_row<DMAX>(j, s1 - 1, me, rp);
        load_col<DMAX>(j, s1 - 1, me, cp);
        for (uint64_t n = s1; n-- > s0;) {
#pragma unroll
            for (int c = 0; c < DMAX; ++c) {
                r0w[c] = rp[c];
                c0[c] = cp[c];
            }
            if (n > s0) {
                load_row<DMAX>(j, n - 1, me, rp);
                load_col<DMAX>(j, n - 1, me, cp);
            }
            const double2 rn = own ? seg[(n - s0) * DMAX + lane] : make_double2(0.0, 0.0);
            double2 rh[DMAX], ch[DMAX];
#pragma unroll
            for (int c = 0; c < DMAX; ++c) {
                rh[c] = make_double2(0.5 * (r0w[c].x + r1w[c].x), 0.5 * (r0w[c].y + r1w[c].y));
                ch[c] = make_double2(0.5 * (c0[c].x + c1[c].x), 0.5 * (c0[c].y + c1[c].y));
            }
            const double2 u1 = rn;
            const double2 k1 = mv_row<DMAX>(r0w, u1, D);
            const double2 u2 = cadd(rn, cscale(k1, 0.5 * dt));
            const double2 k2 = mv_row<DMAX>(rh, u2, D);
            const double2 u3 = cadd(rn, cscale(k2, 0.5 * dt));
            const double2 k3 = mv_row<DMAX>(rh, u3, D);
            const double2 u4 = cadd(rn, cscale(k3, dt));
            double2 gk1 = cscale(g, dt / 6.0), gk2 = cscale(g, dt / 3.0), gk3 = cscale(g, dt / 3.0);
            const double2 gk4 = cscale(g, dt / 6.0);
            double2 gr = g;
            const double2 gu4 = mhv_col<DMAX>(c1, gk4, D);
            gr = cadd(gr, gu4);
            gk3 = cadd(gk3, cscale(gu4, dt));
            const double2 gu3 = mhv_col<DMAX>(ch, gk3, D);
            gr = cadd(gr, gu3);
            gk2 = cadd(gk2, cscale(gu3, 0.5 * dt));
            const double2 gu2 = mhv_col<DMAX>(ch, gk2, D);
            gr = cadd(gr, gu2);
            gk1 = cadd(gk1, cscale(gu2, 0.5 * dt));
            const double2 gu1 = mhv_col<DMAX>(c0, gk1, D);
            gr = cadd(gr, gu1);
            // row `lane` of G(L(t_n)) and G(L(t_{n+1})) from this step
            double2* Lb1 = j.L_bar + static_cast<size_t>(n + 1) * DD;
#pragma unroll
            for (int c = 0; c < DMAX; ++c) {
                if (c < D) {
                    const double2 x1 = shfl2(u1, c), x2 = shfl2(u2, c), x3 = shfl2(u3, c), x4 = shfl2(u4, c);
                    const double2 h = cscale(cadd(cmulc(gk2, x2), cmulc(gk3, x3)), 0.5);
                    const double2 gl0 = cadd(cmulc(gk1, x1), h);
                    const double2 gl1 = cadd(cmulc(gk4, x4), h);
                    if (own) Lb1[lane + static_cast<size_t>(c) * D] = cadd(pend[c], gl1);
                    pend[c] = gl0;
                }
            }
            if (se && j.obs_bar && (n % se) == 0) {
                const double2 o = j.obs_bar[n / se];
                gr = cadd(gr, cmulc(o, ob_l));
                ovb = cadd(ovb, cmulc(o, rn));
            }
            g = own ? gr : make_double2(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < DMAX; ++c) {
                r1w[c] = r0w[c];
                c1[c] = c0[c];
            }
        }
        __syncwarp();
    }
    if (own) {
#pragma unroll
        for (int c = 0; c < DMAX; ++c)
            if (c < D) j.L_bar[lane + static_cast<size_t>(c) * D] = pend[c];
        if (j.r0_bar) j.r0_bar[lane] = g;
        if (j.obs_vec_bar) j.obs_vec_bar[lane] = ovb;
    }
}

// ------------------------------------------------ asynchronous copies (cp.async) --
// Per-warp rings of GR_RING slots in shared memory, filled GR_RING - 1 steps ahead of
// their use, so that a sequential sweep never waits on a global load.
constexpr int GR_RING = 8;


// ------------------------------------------------ RK4 by step matrices (D <= 4) --
// For the linear system r' = L(t) r, one RK4 step is r_{n+1} = M_n r_n with
//   K1 = L0, K2 = Lh + dt/2 Lh K1, K3 = Lh + dt/2 Lh K2, K4 = L1 + dt L1 K3,
//   M_n = I + dt/6 (K1 + 2 K2 + 2 K3 + K4),  L0 = L(t_n), L1 = L(t_{n+1}), Lh = (L0 + L1)/2,
// which depends on the generator only.  All M_n are built in parallel; the sequential
// sweeps then apply one D x D matrix per step (instead of four dependent products), with
// the matrices streamed through the shared-memory ring.  The reverse sweep applies M_n^H;
// the generator gradients of every step, which need r_n and G(r_{n+1}) only, are formed
// in parallel afterwards.  Matrices are column-major D x D in records of 16 entries.
constexpr int SM_REC = 16;

__device__ __forceinline__ void sm_load(const Rk4GJob& j, uint64_t t, double2* A) {
    const int DD = j.D * j.D;
    for (int e = 0; e < DD; ++e) {
        double2 v = j.L[t * DD + e];
        if (j.L_add) v = cadd(v, j.L_add[t * DD + e]);
        A[e] = v;
    }
}

// C = A (I + a B): C = A + a A B (column-major, D x D)
__device__ __forceinline__ void sm_stage(const double2* A, const double2* B, double a, int D, double2* C) {
    for (int c = 0; c < D; ++c)
        for (int r = 0; r < D; ++r) {
            double2 acc = make_double2(0.0, 0.0);
            for (int k = 0; k < D; ++k) acc = cfma2(A[r + k * D], B[k + c * D], acc);
            C[r + c * D] = cadd(A[r + c * D], cscale(acc, a));
        }
}

__global__ void k_rk4g_stepmat(const Rk4GJob* __restrict__ jobs, uint64_t mstride, double2* __restrict__ M) {
    const Rk4GJob& j = jobs[blockIdx.y];
    const uint64_t n = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n >= j.steps) return;
    const int D = j.D, DD = D * D;
    const double dt = j.dt;
    double2 L0[SM_REC], L1[SM_REC], Lh[SM_REC], Ka[SM_REC], Kb[SM_REC], S[SM_REC];
    sm_load(j, n, L0);
    sm_load(j, n + 1, L1);
    for (int e = 0; e < DD; ++e) {
        Lh[e] = make_double2(0.5 * (L0[e].x + L1[e].x), 0.5 * (L0[e].y + L1[e].y));
        S[e] = L0[e];  // K1
    }
    sm_stage(Lh, L0, 0.5 * dt, D, Ka);  // K2
    for (int e = 0; e < DD; ++e) S[e] = cadd(S[e], cscale(Ka[e], 2.0));
    sm_stage(Lh, Ka, 0.5 * dt, D, Kb);  // K3
    for (int e = 0; e < DD; ++e) S[e] = cadd(S[e], cscale(Kb[e], 2.0));
    sm_stage(L1, Kb, dt, D, Ka);  // K4
    double2* out = M + (static_cast<size_t>(blockIdx.y) * mstride + n) * SM_REC;
    for (int c = 0; c < D; ++c)
        for (int r = 0; r < D; ++r) {
            const int e = r + c * D;
            double2 v = cscale(cadd(S[e], Ka[e]), dt / 6.0);
            if (r == c) v.x += 1.0;
            out[e] = v;
        }
}

// ring of step matrices: lanes < D*D copy 16 bytes each
__device__ __forceinline__ void sm_fetch(const double2* Mj, uint64_t n, int DD, double2* ring, int lane) {
    if (lane < DD) cp_async16(ring + (n % GR_RING) * SM_REC + lane, Mj + n * SM_REC + lane);
}

// Forward sweep: one warp per job (four per CTA), r_{n+1} = M_n r_n.  Every state goes
// to R (the job's [steps + 1][4] array) and the samples are formed afterwards
// (k_rk4g_samples), so that nothing in the loop waits on memory.
__global__ void __launch_bounds__(128) k_rk4g_chain(const Rk4GJob* __restrict__ jobs, int njobs, uint64_t every,
                                                    const double2* __restrict__ M, uint64_t mstride,
                                                    double2* __restrict__ R) {
    __shared__ __align__(16) double2 ring_all[4][GR_RING * SM_REC];
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= njobs) return;
    double2* ring = ring_all[threadIdx.x >> 5];
    const Rk4GJob j = jobs[w];
    const int D = j.D, DD = D * D;
    const int row = lane < D ? lane : 0;
    const uint64_t steps = j.steps;
    const double2* Mj = M + static_cast<size_t>(w) * mstride * SM_REC;
    double2* Rj = R + static_cast<size_t>(w) * (mstride + 1) * 4;
    for (uint64_t t = 0; t + 1 < GR_RING; ++t) {
        if (t < steps) sm_fetch(Mj, t, DD, ring, lane);
        cp_async_commit();
    }
    double2 r = lane < D ? j.r0[lane] : make_double2(0.0, 0.0);
    uint64_t ck_left = 0, ck = 0;
    for (uint64_t i = 0; i < steps; ++i) {
        const uint64_t tn = i + GR_RING - 1;
        if (tn < steps) sm_fetch(Mj, tn, DD, ring, lane);
        cp_async_commit();
        cp_async_wait<GR_RING - 2>();
        __syncwarp();
        if (lane < D) Rj[i * 4 + lane] = r;
        if (ck_left == 0) {
            if (j.ckpt && lane < D) j.ckpt[ck * D + lane] = r;
            ++ck;
            ck_left = every;
        }
        --ck_left;
        const double2* m = ring + (i % GR_RING) * SM_REC;
        double2 mrow[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) mrow[c] = c < D ? m[row + c * D] : make_double2(0.0, 0.0);
        r = mv_row<4>(mrow, r, D);
        __syncwarp();
    }
    cp_async_wait<0>();
    if (lane < D) Rj[steps * 4 + lane] = r;
    if (j.r_out && lane < D) j.r_out[lane] = r;
}

// obs_out[s] = obs . r(t_s), t_s = min(s * sample_every, steps): one thread per (s, job).
__global__ void k_rk4g_samples(const Rk4GJob* __restrict__ jobs, uint64_t mstride, const double2* __restrict__ R) {
    const Rk4GJob& j = jobs[blockIdx.y];
    const uint64_t se = j.sample_every;
    if (!se || !j.obs_out) return;
    const uint64_t s = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (s >= n_samples(j.steps, se)) return;
    const uint64_t t = min(s * se, j.steps);
    const double2* Rt = R + (static_cast<size_t>(blockIdx.y) * (mstride + 1) + t) * 4;
    double2 v = make_double2(0.0, 0.0);
    for (int l = 0; l < j.D; ++l) v = cadd(v, cmul(j.obs[l], Rt[l]));
    j.obs_out[s] = v;
}

// States of every checkpoint segment (one warp per (segment, job)): R[n] for n in [s0, s1],
// R the job's [steps + 1][4] array.
__global__ void __launch_bounds__(32) k_rk4g_states(const Rk4GJob* __restrict__ jobs, uint64_t every,
                                                    const double2* __restrict__ M, uint64_t mstride,
                                                    double2* __restrict__ R) {
    __shared__ __align__(16) double2 ring[GR_RING * SM_REC];
    const Rk4GJob j = jobs[blockIdx.y];
    const uint64_t sg = blockIdx.x;
    const uint64_t steps = j.steps;
    const uint64_t nck = (steps + every - 1) / every;
    if (sg >= nck) return;
    const int lane = threadIdx.x;
    const int D = j.D, DD = D * D;
    const int row = lane < D ? lane : 0;
    const uint64_t s0 = sg * every, s1 = min(s0 + every, steps);
    const double2* Mj = M + static_cast<size_t>(blockIdx.y) * mstride * SM_REC;
    double2* Rj = R + static_cast<size_t>(blockIdx.y) * (mstride + 1) * 4;
    for (uint64_t k = 0; k + 1 < GR_RING; ++k) {
        if (s0 + k < s1) sm_fetch(Mj, s0 + k, DD, ring, lane);
        cp_async_commit();
    }
    double2 r = lane < D ? j.ckpt[sg * D + lane] : make_double2(0.0, 0.0);
    for (uint64_t i = s0; i < s1; ++i) {
        const uint64_t tn = i + GR_RING - 1;
        if (tn < s1) sm_fetch(Mj, tn, DD, ring, lane);
        cp_async_commit();
        cp_async_wait<GR_RING - 2>();
        __syncwarp();
        if (lane < D) Rj[i * 4 + lane] = r;
        const double2* m = ring + (i % GR_RING) * SM_REC;
        double2 mrow[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) mrow[c] = c < D ? m[row + c * D] : make_double2(0.0, 0.0);
        r = mv_row<4>(mrow, r, D);
        __syncwarp();
    }
    cp_async_wait<0>();
    if (s1 == steps && lane < D) Rj[steps * 4 + lane] = r;
}

// Reverse sweep (one warp per job, four per CTA): G[steps] = G(r_steps),
// G[n] = M_n^H G[n+1] + conj(obs) obs_bar[n / se] at sampled n; G(r_0) = G[0].  The sample
// weights travel with the step matrices through the ring (entry SM_REC of a slot), and
// G(obs) = sum over samples of conj(r(t_s)) obs_bar[s] is summed after the loop.
constexpr int SB_SLOT = SM_REC + 2;

__global__ void __launch_bounds__(128) k_rk4g_backchain(const Rk4GJob* __restrict__ jobs, int njobs,
                                                        const double2* __restrict__ M, uint64_t mstride,
                                                        const double2* __restrict__ R, double2* __restrict__ G) {
    __shared__ __align__(16) double2 ring_all[4][GR_RING * SB_SLOT];
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= njobs) return;
    double2* ring = ring_all[threadIdx.x >> 5];
    const Rk4GJob j = jobs[w];
    const int D = j.D, DD = D * D;
    const bool own = lane < D;
    const int col = own ? lane : 0;
    const uint64_t steps = j.steps, se = j.sample_every;
    const bool samples = se && j.obs_bar;
    const uint64_t nsamp = n_samples(steps, se);
    const double2* Mj = M + static_cast<size_t>(w) * mstride * SM_REC;
    const double2* Rj = R + static_cast<size_t>(w) * (mstride + 1) * 4;
    double2* Gj = G + static_cast<size_t>(w) * (mstride + 1) * 4;
    const double2 ob_l = (j.obs && own) ? j.obs[lane] : make_double2(0.0, 0.0);
    double2 g = (j.r_final_bar && own) ? j.r_final_bar[lane] : make_double2(0.0, 0.0);
    if (samples) g = cadd(g, cmulc(j.obs_bar[nsamp - 1], ob_l));  // the final sample, at r_steps
    if (own) Gj[steps * 4 + lane] = g;
    // fetch position f (descending) with f % se and f / se kept incrementally
    uint64_t f = steps, f_mod = 0, f_div = 0;
    if (samples && steps > 0) {
        f_mod = (steps - 1) % se;
        f_div = (steps - 1) / se;
    }
    auto fetch_next = [&]() {  // the slot of step f - 1
        if (f == 0) return;
        --f;
        double2* slot = ring + (f % GR_RING) * SB_SLOT;
        if (lane < DD) cp_async16(slot + lane, Mj + f * SM_REC + lane);
        if (lane == 16) {
            if (samples && f_mod == 0) cp_async16(slot + SM_REC, j.obs_bar + f_div);
            else slot[SM_REC] = make_double2(0.0, 0.0);
        }
        if (samples) {
            if (f_mod == 0) {
                f_mod = se - 1;
                --f_div;
            } else {
                --f_mod;
            }
        }
    };
    for (int k = 0; k + 1 < GR_RING; ++k) {
        fetch_next();
        cp_async_commit();
    }
    for (uint64_t n = steps; n-- > 0;) {
        fetch_next();
        cp_async_commit();
        cp_async_wait<GR_RING - 2>();
        __syncwarp();
        const double2* m = ring + (n % GR_RING) * SB_SLOT;
        double2 mcol[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) mcol[r] = r < D ? m[r + col * D] : make_double2(0.0, 0.0);
        double2 gr = mhv_col<4>(mcol, g, D);
        gr = cadd(gr, cmulc(m[SM_REC], ob_l));  // zero weight at steps without a sample
        g = own ? gr : make_double2(0.0, 0.0);
        if (own) Gj[n * 4 + lane] = g;
        __syncwarp();
    }
    cp_async_wait<0>();
    if (own && j.r0_bar) j.r0_bar[lane] = g;
    // G(obs)_l = sum_s conj(r_l(t_s)) obs_bar[s]: lane = (component lane % 4, slice lane / 4)
    if (j.obs_vec_bar) {
        const int c = lane & 3, sl = lane >> 2;
        double2 acc = make_double2(0.0, 0.0);
        if (samples && c < D)
            for (uint64_t sidx = sl; sidx < nsamp; sidx += 8) {
                const uint64_t t = min(sidx * se, steps);
                acc = cadd(acc, cmulc(j.obs_bar[sidx], Rj[t * 4 + c]));
            }
#pragma unroll
        for (int o = 4; o < 32; o <<= 1) {
            acc.x += __shfl_xor_sync(0xffffffffu, acc.x, o);
            acc.y += __shfl_xor_sync(0xffffffffu, acc.y, o);
        }
        if (lane < D) j.obs_vec_bar[lane] = acc;
    }
}

// Gradient of the RK4 step n with respect to L(t_n) (as L0) and L(t_{n+1}) (as L1),
// from r_n and g = G(r_{n+1}): the reverse-mode rules of the vector recursion
//   u1 = r, k_i = A_i u_i (A = L0, Lh, Lh, L1), u_{i+1} = r + c_i k_i, r' = r + dt/6 (k1 + 2k2 + 2k3 + k4).
__device__ void sm_step_grads(const double2* L0, const double2* L1, int D, double dt, const double2* rn,
                              const double2* g, double2* gl0, double2* gl1) {
    double2 Lh[SM_REC];
    for (int e = 0; e < D * D; ++e) Lh[e] = make_double2(0.5 * (L0[e].x + L1[e].x), 0.5 * (L0[e].y + L1[e].y));
    auto mv = [&](const double2* A, const double2* x, double2* y) {
        for (int r = 0; r < D; ++r) {
            double2 acc = make_double2(0.0, 0.0);
            for (int c = 0; c < D; ++c) acc = cfma2(A[r + c * D], x[c], acc);
            y[r] = acc;
        }
    };
    auto mhv = [&](const double2* A, const double2* x, double2* y) {
        for (int c = 0; c < D; ++c) {
            double2 acc = make_double2(0.0, 0.0);
            for (int r = 0; r < D; ++r) acc = cfma2(cconj(A[r + c * D]), x[r], acc);
            y[c] = acc;
        }
    };
    double2 u1[4], u2[4], u3[4], u4[4], k[4];
    for (int r = 0; r < D; ++r) u1[r] = rn[r];
    mv(L0, u1, k);
    for (int r = 0; r < D; ++r) u2[r] = cadd(rn[r], cscale(k[r], 0.5 * dt));
    mv(Lh, u2, k);
    for (int r = 0; r < D; ++r) u3[r] = cadd(rn[r], cscale(k[r], 0.5 * dt));
    mv(Lh, u3, k);
    for (int r = 0; r < D; ++r) u4[r] = cadd(rn[r], cscale(k[r], dt));
    double2 gk1[4], gk2[4], gk3[4], gk4[4], gu[4];
    for (int r = 0; r < D; ++r) {
        gk1[r] = cscale(g[r], dt / 6.0);
        gk2[r] = cscale(g[r], dt / 3.0);
        gk3[r] = cscale(g[r], dt / 3.0);
        gk4[r] = cscale(g[r], dt / 6.0);
    }
    mhv(L1, gk4, gu);
    for (int r = 0; r < D; ++r) gk3[r] = cadd(gk3[r], cscale(gu[r], dt));
    mhv(Lh, gk3, gu);
    for (int r = 0; r < D; ++r) gk2[r] = cadd(gk2[r], cscale(gu[r], 0.5 * dt));
    mhv(Lh, gk2, gu);
    for (int r = 0; r < D; ++r) gk1[r] = cadd(gk1[r], cscale(gu[r], 0.5 * dt));
    for (int c = 0; c < D; ++c)
        for (int r = 0; r < D; ++r) {
            const double2 h = cscale(cadd(cmulc(gk2[r], u2[c]), cmulc(gk3[r], u3[c])), 0.5);
            gl0[r + c * D] = cadd(cmulc(gk1[r], u1[c]), h);
            gl1[r + c * D] = cadd(cmulc(gk4[r], u4[c]), h);
        }
}

// L_bar[t] = (step t's gradient as L0) + (step t-1's gradient as L1), one thread per (t, job).
__global__ void k_rk4g_lbar(const Rk4GJob* __restrict__ jobs, uint64_t mstride, const double2* __restrict__ R,
                            const double2* __restrict__ G) {
    const Rk4GJob& j = jobs[blockIdx.y];
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t steps = j.steps;
    if (t > steps) return;
    const int D = j.D, DD = D * D;
    const double2* Rj = R + static_cast<size_t>(blockIdx.y) * (mstride + 1) * 4;
    const double2* Gj = G + static_cast<size_t>(blockIdx.y) * (mstride + 1) * 4;
    double2 acc[SM_REC];
    for (int e = 0; e < DD; ++e) acc[e] = make_double2(0.0, 0.0);
    double2 La[SM_REC], Lb[SM_REC], gl0[SM_REC], gl1[SM_REC];
    if (t < steps) {  // step t: L(t) is its L0
        sm_load(j, t, La);
        sm_load(j, t + 1, Lb);
        sm_step_grads(La, Lb, D, j.dt, Rj + t * 4, Gj + (t + 1) * 4, gl0, gl1);
        for (int e = 0; e < DD; ++e) acc[e] = gl0[e];
    }
    if (t >= 1) {  // step t-1: L(t) is its L1
        sm_load(j, t - 1, La);
        sm_load(j, t, Lb);
        sm_step_grads(La, Lb, D, j.dt, Rj + (t - 1) * 4, Gj + t * 4, gl0, gl1);
        for (int e = 0; e < DD; ++e) acc[e] = cadd(acc[e], gl1[e]);
    }
    double2* out = j.L_bar + t * DD;
    for (int e = 0; e < DD; ++e) out[e] = acc[e];
}

// ---------------------------------------------------- L4 -> sources (CSC) --
// src_bar[s][t] = sum over entries (e, w, cj) of column s: cj ? w conj(Lb[t][e]) : conj(w) Lb[t][e]
// The arrays of one instance for k_src_adj and k_coef_z (launched over all instances).
struct SrcAdjJob {
    const double2* Lb;
    const int32_t* colptr;
    const uint32_t* rows;
    const double2* coef;
    double2* src_bar;
    const uint32_t* erow;
    const uint32_t* keys;
    uint32_t nnz;  // 0: no coupling-operator aggregation
    const double2* F;
    const double2* Cc;
    const double2* R;
    double2* Z;
    uint32_t E;  // entries of L4 (N^4)
};

__global__ void k_src_adj(const SrcAdjJob* __restrict__ jobs, uint32_t T) {
    const SrcAdjJob& jb = jobs[blockIdx.z];
    const uint32_t E = jb.E;
    const double2* __restrict__ Lb = jb.Lb;
    const int32_t* __restrict__ colptr = jb.colptr;
    const uint32_t* __restrict__ rows = jb.rows;
    const double2* __restrict__ coef = jb.coef;
    double2* __restrict__ src_bar = jb.src_bar;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t s = blockIdx.y;
    if (t >= T) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int32_t q = colptr[s]; q < colptr[s + 1]; ++q) {
        const uint32_t e = rows[q] & 0x7fffffffu;
        const double2 lb = Lb[static_cast<size_t>(t) * E + e];
        const double2 w = coef[q];
        acc = (rows[q] >> 31) ? cadd(acc, cmulc(w, lb)) : cadd(acc, cmulc(lb, w));
    }
    src_bar[static_cast<size_t>(s) * T + t] = acc;
}

// Z[q] = sum_t conj(Lb[t][e_q]) v~_q(t), one warp per CSR entry.
__global__ void k_coef_z(const SrcAdjJob* __restrict__ jobs, uint32_t T, uint32_t nf3) {
    const SrcAdjJob& jb = jobs[blockIdx.y];
    const uint32_t E = jb.E;
    const double2* __restrict__ Lb = jb.Lb;
    const uint32_t* __restrict__ entry_row = jb.erow;
    const uint32_t* __restrict__ keys = jb.keys;
    const uint32_t nnz = jb.nnz;
    const double2* __restrict__ F = jb.F;
    const double2* __restrict__ Cc = jb.Cc;
    const double2* __restrict__ R = jb.R;
    double2* __restrict__ Z = jb.Z;
    const uint32_t q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (q >= nnz) return;
    const uint32_t e = entry_row[q], key = keys[q];
    const uint32_t s = key & 0x7fffffffu;
    const bool cj = (key >> 31) != 0;
    const uint32_t kind = s / nf3, tri = s % nf3;
    const double2* v = (kind == 0 ? F : (kind == 1 ? Cc : R)) + static_cast<size_t>(tri) * T;
    double2 acc = make_double2(0.0, 0.0);
    for (uint32_t t = lane; t < T; t += 32) {
        double2 x = v[t];
        if (cj) x = cconj(x);
        acc = cadd(acc, cmulc(x, Lb[static_cast<size_t>(t) * E + e]));
    }
    acc = warp_sum2(acc);
    if (lane == 0) Z[q] = acc;
}

// ---------------------------------------------------------- F/C/R adjoint --
struct FcrAdjJob {
    const double2* gamma;  // [nf][T]
    const double2* Fb;     // [nf^3][T]
    const double2* Cb;
    const double2* Rb;
    const double* omegas;  // [nf] (device)
    const int* mirror;     // [nf] (device)
    const uint8_t* fc_used;  // [nf^3]
    double2* G1;   // [nf^3][T] partials: d/d g1
    double2* G2F;  // d/d g2 of F (Gamma_{mirror j})
    double2* G2C;  // d/d g2 of C (conj(Gamma_j))
    double2* G2R;  // d/d g2 of R (Gamma_j)
    double2* A2;   // [nf^3][T] conj(P g1)
    double* wpart;  // [nf^3][1 + ntiles]
    int ntiles;
};

constexpr int SC_THREADS = 256;
constexpr int SC_ITEMS = 4;
constexpr int SC_CHUNK = SC_THREADS * SC_ITEMS;

// Exclusive block scan of NV complex values per thread; returns the block totals.
template <int NV>
__device__ __forceinline__ void block_xscan(double2 (&x)[NV], double2 (&tot)[NV], double2* sm /* [NV][33] */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double2 inc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        inc[v] = x[v];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double2 y = shfl_up2(inc[v], o);
            if (lane >= o) inc[v] = cadd(inc[v], y);
        }
        if (lane == 31) sm[v * 33 + warp] = inc[v];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double2 a = lane < nw ? sm[v * 33 + lane] : make_double2(0.0, 0.0);
            double2 ai = a;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double2 y = shfl_up2(ai, o);
                if (lane >= o) ai = cadd(ai, y);
            }
            if (lane < nw) sm[v * 33 + lane] = csub(ai, a);  // exclusive warp offsets
            if (lane == 31) sm[v * 33 + 32] = ai;            // block total
        }
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        x[v] = cadd(sm[v * 33 + warp], csub(inc[v], x[v]));
        tot[v] = sm[v * 33 + 32];
    }
    __syncthreads();
}

__device__ __forceinline__ double block_sum(double v, double* sm) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += sm[w];
    __syncthreads();
    return t;
}

__device__ __forceinline__ double2 phase_m(double w, double dt, uint32_t k) {  // e^{-i w k dt}
    double s, c;
    sincos(w * (static_cast<double>(k) * dt), &s, &c);
    return make_double2(c, -s);
}

// -i x (multiplication by -i)
__device__ __forceinline__ double2 mul_mi(double2 x) { return make_double2(x.y, -x.x); }

// One CTA per (triple, job): the O(T) parts of the F, C, R adjoints.
__global__ void __launch_bounds__(SC_THREADS) k_fcr_adj_scan(const FcrAdjJob* __restrict__ jobs, int nf, uint32_t T,
                                                             double dt) {
    __shared__ double2 sm[5 * 33];
    __shared__ double red[SC_THREADS / 32];
    const FcrAdjJob jb = jobs[blockIdx.y];
    const uint32_t q = blockIdx.x;
    const int nf2 = nf * nf;
    const int i = static_cast<int>(q / nf2), jj = static_cast<int>((q / nf) % nf), kk = static_cast<int>(q % nf);
    const double w = jb.omegas[i] + jb.omegas[jj] + jb.omegas[kk];
    const double2* g1 = jb.gamma + static_cast<size_t>(i) * T;
    const double2* g2F = jb.gamma + static_cast<size_t>(jb.mirror[jj]) * T;
    const double2* gj = jb.gamma + static_cast<size_t>(jj) * T;  // C uses conj(gj), R uses gj
    const size_t qo = static_cast<size_t>(q) * T;
    const double2* Fb = jb.Fb + qo;
    const double2* Cb = jb.Cb + qo;
    const double2* Rb = jb.Rb + qo;
    const double dt2 = dt * dt;
    double wacc = 0.0;
    // prefix pass: A0F, A1F, A0C, A1C, B0
    double2 carry[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) carry[v] = make_double2(0.0, 0.0);
    for (uint32_t c0 = 0; c0 < T; c0 += SC_CHUNK) {
        double2 x[SC_ITEMS][5];
        double2 tsum[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) tsum[v] = make_double2(0.0, 0.0);
#pragma unroll
        for (int it = 0; it < SC_ITEMS; ++it) {
            const uint32_t t = c0 + threadIdx.x * SC_ITEMS + it;
            if (t < T) {
                const double2 P = phase_m(w, dt, t), Q = cconj(P);
                const double2 a = cmul(g2F[t], Q);
                const double2 b = cmul(cconj(gj[t]), Q);
                x[it][0] = a;
                x[it][1] = cscale(a, static_cast<double>(t));
                x[it][2] = b;
                x[it][3] = cscale(b, static_cast<double>(t));
                x[it][4] = cmul(gj[t], P);
            } else {
#pragma unroll
                for (int v = 0; v < 5; ++v) x[it][v] = make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) tsum[v] = cadd(tsum[v], x[it][v]);
        }
        double2 tot[5];
        block_xscan<5>(tsum, tot, sm);
        double2 run[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) run[v] = cadd(carry[v], tsum[v]);
#pragma unroll
        for (int it = 0; it < SC_ITEMS; ++it) {
            const uint32_t t = c0 + threadIdx.x * SC_ITEMS + it;
#pragma unroll
            for (int v = 0; v < 5; ++v) run[v] = cadd(run[v], x[it][v]);
            if (t < T) {
                const double2 P = phase_m(w, dt, t);
                const double2 g1t = g1[t];
                const double2 fb = Fb[t], cb = Cb[t], rb = Rb[t];
                const double tt = static_cast<double>(t);
                // F: G(g1) += conj(dt P A0) Fb ; dl/dw += Re[-i dt^2 conj(Fb) g1 P (t A0 - A1)]
                const double2 SF = cscale(cmul(P, run[0]), dt);
                const double2 SC = cscale(cmul(P, run[2]), dt);
                double2 G1 = cadd(cmulc(fb, SF), cmulc(cb, SC));
                G1 = cadd(G1, cscale(cmulc(rb, run[4]), dt));
                const double2 TF = cmul(P, csub(cscale(run[0], tt), run[1]));
                const double2 TC = cmul(P, csub(cscale(run[2], tt), run[3]));
                wacc += dt2 * (mul_mi(cmul(cmulc(g1t, fb), TF)).x + mul_mi(cmul(cmulc(g1t, cb), TC)).x);
                jb.G1[qo + t] = G1;
                jb.A2[qo + t] = cconj(cmul(P, g1t));
            }
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) carry[v] = cadd(carry[v], tot[v]);
    }
    __syncthreads();
    // suffix pass over u = T - 1 - t: SufF, SufC, SR0, SR1
    double2 carry2[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) carry2[v] = make_double2(0.0, 0.0);
    for (uint32_t c0 = 0; c0 < T; c0 += SC_CHUNK) {
        double2 x[SC_ITEMS][4];
        double2 tsum[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) tsum[v] = make_double2(0.0, 0.0);
#pragma unroll
        for (int it = 0; it < SC_ITEMS; ++it) {
            const uint32_t u = c0 + threadIdx.x * SC_ITEMS + it;
            if (u < T) {
                const uint32_t t = T - 1 - u;
                const double2 Q = cconj(phase_m(w, dt, t));
                const double2 cg1 = cconj(g1[t]);
                const double2 qg = cmul(Q, cg1);
                x[it][0] = cmul(qg, Fb[t]);
                x[it][1] = cmul(qg, Cb[t]);
                x[it][2] = cmul(cg1, Rb[t]);
                x[it][3] = Rb[t];
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v) x[it][v] = make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) tsum[v] = cadd(tsum[v], x[it][v]);
        }
        double2 tot[4];
        block_xscan<4>(tsum, tot, sm);
        double2 run[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) run[v] = cadd(carry2[v], tsum[v]);
#pragma unroll
        for (int it = 0; it < SC_ITEMS; ++it) {
            const uint32_t u = c0 + threadIdx.x * SC_ITEMS + it;
#pragma unroll
            for (int v = 0; v < 4; ++v) run[v] = cadd(run[v], x[it][v]);
            if (u < T) {
                const uint32_t t = T - 1 - u;
                const double2 P = phase_m(w, dt, t), Q = cconj(P);
                const double2 g1t = g1[t], g2r = gj[t];
                jb.G2F[qo + t] = cscale(cmul(P, run[0]), dt);
                jb.G2C[qo + t] = cscale(cmul(P, run[1]), dt);
                const double2 g2P = cmul(g2r, P), g1P = cmul(g1t, P);
                jb.G1[qo + t] = csub(jb.G1[qo + t], cscale(cmul(cconj(g2P), run[3]), dt));
                jb.G2R[qo + t] = cscale(csub(cmul(Q, run[2]), cmul(cconj(g1P), run[3])), dt);
                const double2 br = csub(cconj(run[2]), cmul(g1t, cconj(run[3])));
                wacc += static_cast<double>(t) * dt2 * mul_mi(cmul(g2P, br)).x;
            }
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) carry2[v] = cadd(carry2[v], tot[v]);
    }
    const double ws = block_sum(wacc, red);
    if (threadIdx.x == 0) jb.wpart[static_cast<size_t>(q) * (1 + jb.ntiles)] = ws;
}

constexpr int CR_TM = 128;  // outputs per CTA (one per thread)
constexpr int CR_TK = 256;  // k per shared-memory tile

// Correlations c1, c2, c3 of the F and C adjoints: one CTA per (m tile, triple, job).
__global__ void __launch_bounds__(CR_TM) k_fcr_adj_corr(const FcrAdjJob* __restrict__ jobs, int nf, uint32_t T,
                                                        double dt) {
    __shared__ double2 fb_s[CR_TK], cb_s[CR_TK];
    __shared__ double2 a1f_s[CR_TM + CR_TK], a1c_s[CR_TM + CR_TK], a2_s[CR_TM + CR_TK];
    __shared__ double red[CR_TM / 32];
    const FcrAdjJob jb = jobs[blockIdx.z];
    const uint32_t q = blockIdx.y;
    if (!jb.fc_used[q]) return;
    const int nf2 = nf * nf;
    const int i = static_cast<int>(q / nf2), jj = static_cast<int>((q / nf) % nf), kk = static_cast<int>(q % nf);
    const double w = jb.omegas[i] + jb.omegas[jj] + jb.omegas[kk];
    const double2* g2F = jb.gamma + static_cast<size_t>(jb.mirror[jj]) * T;
    const double2* gj = jb.gamma + static_cast<size_t>(jj) * T;
    const size_t qo = static_cast<size_t>(q) * T;
    const double2* Fb = jb.Fb + qo;
    const double2* Cb = jb.Cb + qo;
    const double2* A2 = jb.A2 + qo;
    const uint32_t m0 = blockIdx.x * CR_TM;
    const uint32_t m = m0 + threadIdx.x;
    double2 c1f = make_double2(0.0, 0.0), c1c = c1f, c2f = c1f, c2c = c1f, c3f = c1f, c3c = c1f;
    for (uint32_t k0 = m0; k0 < T; k0 += CR_TK) {
        // j = k - m ranges over [k0 - m0 - (TM - 1), k0 - m0 + TK - 1]; stage j >= 0
        const int64_t jbase = static_cast<int64_t>(k0) - m0 - (CR_TM - 1);
        __syncthreads();
        for (int x = threadIdx.x; x < CR_TK; x += CR_TM) {
            const uint32_t k = k0 + x;
            fb_s[x] = k < T ? Fb[k] : make_double2(0.0, 0.0);
            cb_s[x] = k < T ? Cb[k] : make_double2(0.0, 0.0);
        }
        for (int x = threadIdx.x; x < CR_TM + CR_TK - 1; x += CR_TM) {
            const int64_t jv = jbase + x;
            if (jv >= 0 && jv < static_cast<int64_t>(T)) {
                a1f_s[x] = cconj(g2F[jv]);
                a1c_s[x] = gj[jv];  // conj(conj(Gamma_j))
                a2_s[x] = A2[jv];
            } else {
                a1f_s[x] = make_double2(0.0, 0.0);
                a1c_s[x] = a1f_s[x];
                a2_s[x] = a1f_s[x];
            }
        }
        __syncthreads();
        if (m < T) {
            const uint32_t kbeg = max(k0, m), kend = min(k0 + CR_TK, T);
            for (uint32_t k = kbeg; k < kend; ++k) {
                const int xs = static_cast<int>(static_cast<int64_t>(k) - m - jbase);
                const double2 fb = fb_s[k - k0], cb = cb_s[k - k0];
                const double2 a2 = a2_s[xs];
                c1f = cfma2(a1f_s[xs], fb, c1f);
                c1c = cfma2(a1c_s[xs], cb, c1c);
                const double2 tf = cmul(a2, fb), tc = cmul(a2, cb);
                const double jd = static_cast<double>(k - m);
                c2f = cadd(c2f, tf);
                c2c = cadd(c2c, tc);
                c3f = make_double2(fma(jd, tf.x, c3f.x), fma(jd, tf.y, c3f.y));
                c3c = make_double2(fma(jd, tc.x, c3c.x), fma(jd, tc.y, c3c.y));
            }
        }
    }
    double wv = 0.0;
    if (m < T) {
        const double2 Q = cconj(phase_m(w, dt, m));
        jb.G1[qo + m] = csub(jb.G1[qo + m], cscale(cmul(Q, cadd(c1f, c1c)), dt));
        jb.G2F[qo + m] = csub(jb.G2F[qo + m], cscale(c2f, dt));
        jb.G2C[qo + m] = csub(jb.G2C[qo + m], cscale(c2c, dt));
        // Re[i dt^2 (g2F conj(c3F) + g2C conj(c3C))], g2C = conj(Gamma_j)
        const double2 s = cadd(cmulc(g2F[m], c3f), cconj(cmul(gj[m], c3c)));
        wv = -dt * dt * s.y;
    }
    const double ws = block_sum(wv, red);
    if (threadIdx.x == 0) jb.wpart[static_cast<size_t>(q) * (1 + jb.ntiles) + 1 + blockIdx.x] = ws;
}

// ---- FFT form of the correlations (lengths whose working array fits one CTA) ----
// c[m] = sum_{j >= 0} a[j] b[m + j] (m + j < T) is the linear convolution of a with the
// reversed b, read backwards: c[m] = (a * b_rev)[T - 1 - m], b_rev[n] = b[T - 1 - n].  Every
// series is transformed once by the fused path's in-place stages (length N >= 2 T - 1, so the
// circular convolution is the linear one); each of the five outputs (c1 = c1F + c1C summed in
// the frequency domain, c2F, c2C, c3F, c3C) is one product and one inverse transform.
struct AdjSpecJob {
    const double2* src;  // [T]
    double2* out;        // [N] spectrum (digit-reversed order)
    uint32_t T;
    int mode;            // 0: a[n]; 1: conj(a[n]); 2: a[T-1-n]; 3: n a[n]
};

__global__ void __launch_bounds__(FZ_THREADS, 1) k_adj_series_spectrum(const AdjSpecJob* __restrict__ jobs,
                                                                       FzPlan<double2> p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* d = reinterpret_cast<double2*>(smem_raw);
    const AdjSpecJob job = jobs[blockIdx.x];
    for (int n = threadIdx.x; n < p.N; n += blockDim.x) {
        double2 x = make_double2(0.0, 0.0);
        if (static_cast<uint32_t>(n) < job.T) {
            switch (job.mode) {
                case 0: x = job.src[n]; break;
                case 1: x = cconj(job.src[n]); break;
                case 2: x = job.src[job.T - 1 - n]; break;
                default: x = cscale(job.src[n], static_cast<double>(n)); break;
            }
        }
        d[pad_idx<double2>(n)] = x;
    }
    __syncthreads();
    fz_forward(d, p);
    for (int i = threadIdx.x; i < p.N; i += blockDim.x) job.out[i] = d[pad_idx<double2>(i)];
}

struct AdjFftSpectra {
    const double2* gconj;  // [nf][N] spectra of conj(Gamma_b)
    const double2* gplain; // [nf][N] spectra of Gamma_b
    const double2* fb;     // [nf^3][N] spectra of reversed Fb
    const double2* cb;     // [nf^3][N] spectra of reversed Cb
    const double2* a2;     // [nf^3][N] spectra of A2
    const double2* a3;     // [nf^3][N] spectra of n A2[n]
};

// blockIdx = (output kind 0..4, triple, job).  kind 0: G1 -= dt Q c1 (c1 = c1F + c1C);
// 1: G2F -= dt c2F; 2: G2C -= dt c2C; 3, 4: the Bohr-frequency terms of c3F, c3C.
__global__ void __launch_bounds__(FZ_THREADS, 1) k_fcr_adj_corr_fft(const FcrAdjJob* __restrict__ jobs,
                                                                    const AdjFftSpectra* __restrict__ specs, int nf,
                                                                    uint32_t T, double dt, FzPlan<double2> p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* d = reinterpret_cast<double2*>(smem_raw);
    __shared__ double red[FZ_THREADS / 32];
    const int kind = blockIdx.x;
    const uint32_t q = blockIdx.y;
    const FcrAdjJob jb = jobs[blockIdx.z];
    if (!jb.fc_used[q]) return;
    const AdjFftSpectra sp = specs[blockIdx.z];
    const int nf2 = nf * nf;
    const int i = static_cast<int>(q / nf2), jj = static_cast<int>((q / nf) % nf), kk = static_cast<int>(q % nf);
    const int jm = jb.mirror[jj];
    const std::size_t N = static_cast<std::size_t>(p.N), qn = static_cast<std::size_t>(q) * N;
    const double inv = 1.0 / static_cast<double>(p.N);
    for (int n = threadIdx.x; n < p.N; n += blockDim.x) {
        double2 x;
        if (kind == 0) {
            x = cadd(cmul(sp.gconj[static_cast<std::size_t>(jm) * N + n], sp.fb[qn + n]),
                     cmul(sp.gplain[static_cast<std::size_t>(jj) * N + n], sp.cb[qn + n]));
        } else {
            const double2 a = (kind <= 2 ? sp.a2 : sp.a3)[qn + n];
            x = cmul(a, (kind == 1 || kind == 3) ? sp.fb[qn + n] : sp.cb[qn + n]);
        }
        d[pad_idx<double2>(n)] = cscale(x, inv);
    }
    __syncthreads();
    fz_inverse(d, p);
    const double w = jb.omegas[i] + jb.omegas[jj] + jb.omegas[kk];
    const double2* g2F = jb.gamma + static_cast<size_t>(jm) * T;
    const double2* gj = jb.gamma + static_cast<size_t>(jj) * T;
    const size_t qo = static_cast<size_t>(q) * T;
    double wv = 0.0;
    for (uint32_t m = threadIdx.x; m < T; m += blockDim.x) {
        const double2 c = d[pad_idx<double2>(static_cast<int>(T - 1 - m))];
        if (kind == 0) {
            const double2 Q = cconj(phase_m(w, dt, m));
            jb.G1[qo + m] = csub(jb.G1[qo + m], cscale(cmul(Q, c), dt));
        } else if (kind == 1) {
            jb.G2F[qo + m] = csub(jb.G2F[qo + m], cscale(c, dt));
        } else if (kind == 2) {
            jb.G2C[qo + m] = csub(jb.G2C[qo + m], cscale(c, dt));
        } else if (kind == 3) {
            wv += -dt * dt * cmulc(g2F[m], c).y;
        } else {
            wv += -dt * dt * cconj(cmul(gj[m], c)).y;
        }
    }
    if (kind >= 3) {
        const double ws = block_sum(wv, red);
        if (threadIdx.x == 0) atomicAdd(&jb.wpart[static_cast<size_t>(q) * (1 + jb.ntiles) + 1], ws);
    }
}

// FFT length of the correlations for T samples: the smallest 2^k, 3 * 2^k or 5 * 2^k >= 2 T - 1
// whose working array fits one CTA (0: none, the direct kernel runs).
int adj_fft_length(std::size_t T) {
    const std::size_t target = 2 * T - 1;
    std::size_t best = 0;
    for (std::size_t r : {1, 3, 5}) {
        std::size_t n = r;
        while (n < target) n *= 2;
        if (n < 8) continue;
        int rad[FZ_MAX_STAGES], nst = 0;
        if (n > (std::size_t(1) << 16) || !fz_stages(static_cast<int>(n), 8, rad, nst)) continue;
        if (fz_smem<double2>(static_cast<int>(n)) + 256 > 227 * 1024) continue;  // + the static reduction array
        if (!best || n < best) best = n;
    }
    return static_cast<int>(best);
}

// Gamma_bar[b][t] += the partials of every triple that reads column b.
__global__ void k_fcr_adj_reduce(const FcrAdjJob* __restrict__ jobs, int nf, uint32_t T, double2* const* gbar) {
    const FcrAdjJob jb = jobs[blockIdx.z];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    if (t >= T) return;
    const int nf2 = nf * nf;
    double2 acc = make_double2(0.0, 0.0);
    for (int x = 0; x < nf2; ++x) {  // g1 = Gamma_i with i = b
        acc = cadd(acc, jb.G1[(static_cast<size_t>(b) * nf2 + x) * T + t]);
    }
    for (int i = 0; i < nf; ++i)
        for (int jj = 0; jj < nf; ++jj) {
            const bool mir = jb.mirror[jj] == b, dir = jj == b;
            if (!mir && !dir) continue;
            for (int kk = 0; kk < nf; ++kk) {
                const size_t o = (static_cast<size_t>(i) * nf2 + jj * nf + kk) * T + t;
                if (mir) acc = cadd(acc, jb.G2F[o]);
                if (dir) acc = cadd(acc, cadd(cconj(jb.G2C[o]), jb.G2R[o]));
            }
        }
    double2* out = gbar[blockIdx.z] + static_cast<size_t>(b) * T + t;
    *out = cadd(*out, acc);
}

// ------------------------------------------------------------ TCL2 adjoint --
// G(Gamma_b(t)) += 2 Re sum_e conj(Lb_e) D_b,e + i Re sum_e conj(Lb_e) U_b,e
// One instance of the TCL2 adjoint kernels (launched over all instances).
struct Tcl2AdjJob {
    const double2* Lb;     // [T][E]
    const double2* Db;     // [nf][E]
    const double2* Ub;     // [nf][E]
    const double2* gamma;  // [nf][T]
    double2* gbar;         // [nf][T], accumulated
    double2* maps;         // [(1 + 2 nf)][E] or null
    uint32_t T, E;
    int nf;
};

__global__ void k_tcl2_adj_gamma(const Tcl2AdjJob* __restrict__ jobs) {
    const Tcl2AdjJob& jb = jobs[blockIdx.y];
    const double2* __restrict__ Lb = jb.Lb;
    const double2* __restrict__ Db = jb.Db;
    const double2* __restrict__ Ub = jb.Ub;
    double2* __restrict__ gbar = jb.gbar;
    const uint32_t T = jb.T, E = jb.E;
    const int nf = jb.nf;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const double2* l = Lb + static_cast<size_t>(t) * E;
    for (int b = 0; b < nf; ++b) {
        double sd = 0.0, su = 0.0;
        for (uint32_t e = 0; e < E; ++e) {
            const double2 x = l[e];
            const double2 d = Db[static_cast<size_t>(b) * E + e], u = Ub[static_cast<size_t>(b) * E + e];
            sd += x.x * d.x + x.y * d.y;  // Re(conj(x) d)
            su += x.x * u.x + x.y * u.y;
        }
        double2* o = gbar + static_cast<size_t>(b) * T + t;
        *o = cadd(*o, make_double2(2.0 * sd, su));
    }
}

// Per entry e: GL0 = sum_t Lb, GD_b = sum_t 2 Re Gamma_b(t) Lb, GU_b = sum_t Im Gamma_b(t) Lb.
__global__ void k_tcl2_adj_maps(const Tcl2AdjJob* __restrict__ jobs) {
    __shared__ double2 sm[8][32];
    const Tcl2AdjJob& jb = jobs[blockIdx.y];
    const double2* __restrict__ Lb = jb.Lb;
    const double2* __restrict__ gamma = jb.gamma;
    double2* __restrict__ out = jb.maps;  // [(1 + 2 nf)][E]
    const uint32_t T = jb.T, E = jb.E;
    const int nf = jb.nf;
    const uint32_t e = blockIdx.x;
    if (!out || e >= E) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int v = 0; v < 1 + 2 * nf; ++v) {
        double2 acc = make_double2(0.0, 0.0);
        for (uint32_t t = threadIdx.x; t < T; t += blockDim.x) {
            const double2 x = Lb[static_cast<size_t>(t) * E + e];
            double s = 1.0;
            if (v > 0) {
                const int b = (v - 1) >> 1;
                const double2 g = gamma[static_cast<size_t>(b) * T + t];
                s = ((v - 1) & 1) ? g.y : 2.0 * g.x;
            }
            acc = cadd(acc, cscale(x, s));
        }
        acc = warp_sum2(acc);
        if (lane == 0) sm[warp][v & 31] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double2 t2 = make_double2(0.0, 0.0);
            for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t2 = cadd(t2, sm[w][v & 31]);
            out[static_cast<size_t>(v) * E + e] = t2;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------- inner products --
struct InnerJob {
    const double2* a;
    const double2* b;
    uint64_t n;
};

__global__ void k_inner_re(const InnerJob* __restrict__ jobs, double* __restrict__ out) {
    __shared__ double red[8];
    const InnerJob jb = jobs[blockIdx.x];
    double acc = 0.0;
    for (uint64_t k = threadIdx.x; k < jb.n; k += blockDim.x) {
        const double2 x = jb.a[k], y = jb.b[k];
        acc += x.x * y.x + x.y * y.y;
    }
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

template <class T>
T* upload(Carve& cv, const std::vector<T>& v, cudaStream_t st, const char* what) {
    T* d = cv.take<T>(v.size());
    if (!v.empty()) cuda_check(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st), what);
    return d;
}

}  // namespace

// ============================================================== host side ==
std::size_t rk4_num_checkpoints(std::size_t steps, std::size_t every) {
    return every ? (steps + every - 1) / every : 0;
}

namespace {

void validate_rk4g(const std::vector<Rk4GradJob>& jobs, std::size_t every, bool adjoint) {
    if (every == 0) throw Error(kInvalidArgument, "rk4 gradient: checkpoint_every must be > 0");
    for (const auto& j : jobs) {
        if (j.D <= 0 || j.D > 16) throw Error(kInvalidArgument, "rk4 gradient: D = N^2 must be in [1, 16]");
        if (!(j.dt > 0.0)) throw Error(kInvalidArgument, "rk4 gradient: dt must be > 0");
        if (j.steps < 1) throw Error(kInvalidArgument, "rk4 gradient: at least one step");
        if (!j.L || !j.r0) throw Error(kInvalidArgument, "rk4 gradient: null L or r0");
        if (!j.ckpt) throw Error(kInvalidArgument, "rk4 gradient: null checkpoint buffer");
        if ((j.obs_out || j.obs_bar) && (!j.obs || j.sample_every == 0))
            throw Error(kInvalidArgument, "rk4 gradient: samples need obs and sample_every > 0");
        if (adjoint && !j.L_bar) throw Error(kInvalidArgument, "rk4 adjoint: null L_bar");
    }
    if (every * 16 * sizeof(double2) > 160 * 1024) throw Error(kInvalidArgument, "rk4 adjoint: checkpoint_every too large");
}

std::vector<Rk4GJob> to_gjobs(const std::vector<Rk4GradJob>& jobs) {
    std::vector<Rk4GJob> out(jobs.size());
    for (std::size_t k = 0; k < jobs.size(); ++k) {
        const auto& j = jobs[k];
        out[k] = Rk4GJob{j.L,     j.L_add,   j.steps,  j.D,           j.dt,        j.r0,  j.obs,    j.sample_every,
                         j.ckpt,  j.obs_out, j.r_out,  j.obs_bar,     j.r_final_bar, j.L_bar, j.r0_bar, j.obs_vec_bar};
    }
    return out;
}

}  // namespace

void rk4_forward_checkpointed(const std::vector<Rk4GradJob>& jobs, std::size_t every, cudaStream_t st) {
    if (jobs.empty()) return;
    validate_rk4g(jobs, every, false);
    std::vector<Rk4GJob> gj = to_gjobs(jobs);
    int dmax = 0;
    uint64_t mstride = 1;
    for (const auto& j : jobs) {
        dmax = std::max(dmax, j.D);
        mstride = std::max<uint64_t>(mstride, j.steps);
    }
    const int n = static_cast<int>(jobs.size());
    const bool stepmat = dmax <= 4;  // step matrices: [jobs][mstride] records
    Carve probe{nullptr};
    probe.take<Rk4GJob>(gj.size());
    if (stepmat) {
        probe.take<double2>(static_cast<std::size_t>(n) * mstride * SM_REC);
        probe.take<double2>(static_cast<std::size_t>(n) * (mstride + 1) * 4);
    }
    Carve cv{grad_scratch().ensure(probe.off + 256)};
    Rk4GJob* dj = upload(cv, gj, st, "rk4g jobs");
    const unsigned grid = static_cast<unsigned>((n + 3) / 4);
    if (stepmat) {
        double2* M = cv.take<double2>(static_cast<std::size_t>(n) * mstride * SM_REC);
        double2* R = cv.take<double2>(static_cast<std::size_t>(n) * (mstride + 1) * 4);
        k_rk4g_stepmat<<<dim3(static_cast<unsigned>((mstride + 127) / 128), static_cast<unsigned>(n)), 128, 0, st>>>(
            dj, mstride, M);
        launched("k_rk4g_stepmat");
        k_rk4g_chain<<<grid, 128, 0, st>>>(dj, n, every, M, mstride, R);
        launched("k_rk4g_chain");
        uint64_t smax = 1;
        for (const auto& j : jobs)
            if (j.sample_every) smax = std::max<uint64_t>(smax, n_samples(j.steps, j.sample_every));
        k_rk4g_samples<<<dim3(static_cast<unsigned>((smax + 127) / 128), static_cast<unsigned>(n)), 128, 0, st>>>(
            dj, mstride, R);
        launched("k_rk4g_samples");
    } else {
        k_rk4g_fwd<16><<<grid, 128, 0, st>>>(dj, n, every);
        launched("k_rk4g_fwd");
    }
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(rk4 forward)");
}

void rk4_adjoint(const std::vector<Rk4GradJob>& jobs, std::size_t every, cudaStream_t st) {
    if (jobs.empty()) return;
    validate_rk4g(jobs, every, true);
    std::vector<Rk4GJob> gj = to_gjobs(jobs);
    int dmax = 0;
    uint64_t mstride = 1;
    for (const auto& j : jobs) {
        dmax = std::max(dmax, j.D);
        mstride = std::max<uint64_t>(mstride, j.steps);
    }
    const unsigned n = static_cast<unsigned>(jobs.size());
    const bool stepmat = dmax <= 4;  // step matrices, all states R and adjoint states G
    const std::size_t nM = static_cast<std::size_t>(n) * mstride * SM_REC;
    const std::size_t nR = static_cast<std::size_t>(n) * (mstride + 1) * 4;
    Carve probe{nullptr};
    probe.take<Rk4GJob>(gj.size());
    if (stepmat) {
        probe.take<double2>(nM);
        probe.take<double2>(nR);
        probe.take<double2>(nR);
    }
    Carve cv{grad_scratch().ensure(probe.off + 256)};
    Rk4GJob* dj = upload(cv, gj, st, "rk4g jobs");
    if (stepmat) {
        double2* M = cv.take<double2>(nM);
        double2* R = cv.take<double2>(nR);
        double2* G = cv.take<double2>(nR);
        const unsigned nck = static_cast<unsigned>((mstride + every - 1) / every);
        k_rk4g_stepmat<<<dim3(static_cast<unsigned>((mstride + 127) / 128), n), 128, 0, st>>>(dj, mstride, M);
        launched("k_rk4g_stepmat");
        k_rk4g_states<<<dim3(nck, n), 32, 0, st>>>(dj, every, M, mstride, R);
        launched("k_rk4g_states");
        k_rk4g_backchain<<<(n + 3) / 4, 128, 0, st>>>(dj, static_cast<int>(n), M, mstride, R, G);
        launched("k_rk4g_backchain");
        k_rk4g_lbar<<<dim3(static_cast<unsigned>((mstride + 1 + 127) / 128), n), 128, 0, st>>>(dj, mstride, R, G);
        launched("k_rk4g_lbar");
    } else {
        const std::size_t smem = every * 16 * sizeof(double2);
        cuda_check(cudaFuncSetAttribute(k_rk4g_adj<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                   "cudaFuncSetAttribute(k_rk4g_adj)");
        k_rk4g_adj<16><<<n, 32, smem, st>>>(dj, every);
        launched("k_rk4g_adj");
    }
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(rk4 adjoint)");
}

void tcl4_adjoint(const std::vector<Tcl4AdjointJob>& jobs, cudaStream_t st) {
    if (jobs.empty()) return;
    // group by (nf, T): one launch per kernel and group
    std::map<std::pair<int, std::size_t>, std::vector<std::size_t>> groups;
    for (std::size_t k = 0; k < jobs.size(); ++k) {
        const auto& j = jobs[k];
        if (!j.sys || j.T == 0 || !j.gamma || !j.L_bar || !j.gamma_bar)
            throw Error(kInvalidArgument, "tcl4 adjoint: null or empty input");
        if (!(j.dt > 0.0)) throw Error(kInvalidArgument, "tcl4 adjoint: dt must be > 0");
        if (j.T > 0x7fffffffu) throw Error(kOverflow, "tcl4 adjoint: T too large");
        if (j.sys->nf > 27) throw Error(kInvalidArgument, "tcl4 adjoint: at most 27 Bohr frequencies");
        groups[{j.sys->nf, j.T}].push_back(k);
    }
    for (auto& g : groups)
        for (std::size_t k : g.second)
            if (jobs[k].dt != jobs[g.second[0]].dt)
                throw Error(kInvalidArgument, "tcl4 adjoint: jobs with equal (nf, T) must share dt");
    for (auto& g : groups) {
        const int nf = g.first.first;
        const std::size_t T = g.first.second;
        const std::size_t nf3 = static_cast<std::size_t>(nf) * nf * nf;
        const auto& idx = g.second;
        const int ntiles = static_cast<int>((T + CR_TM - 1) / CR_TM);
        // the correlations by FFT when the length fits one CTA and the spectra fit 8 GiB
        int fftN = adj_fft_length(T);
        if (fftN && static_cast<double>(idx.size()) * (2 * nf + 4 * nf3) * fftN * sizeof(double2) > 8.0 * (1ull << 30))
            fftN = 0;
        // per job: coefficient tables (structural), CSC transpose, device metadata
        struct Host {
            CoefTable tab;
            std::vector<int32_t> colptr;
            std::vector<uint32_t> rows;  // e | conj << 31
            std::vector<double2> ccoef;
            std::vector<uint32_t> entry_row;
        };
        std::vector<Host> hs(idx.size());
        std::size_t bytes = 0, packed_bytes = 0;
        {
            Carve probe{nullptr};
            // structural tables and their transposes, one instance per host thread
            auto build_host = [&](std::size_t a) {
                const auto& j = jobs[idx[a]];
                const SystemDesc& s = *j.sys;
                Host& h = hs[a];
                set_coef_table_threads(1);
                build_coef_table(s.N, s.nf, s.p2f.data(), s.ops.data(), s.num_ops, h.tab, true);
                set_coef_table_threads(0);
                const std::size_t E = static_cast<std::size_t>(s.N) * s.N * s.N * s.N;
                const std::size_t nnz = h.tab.src.size();
                h.colptr.assign(3 * nf3 + 1, 0);
                for (std::size_t q = 0; q < nnz; ++q) h.colptr[(h.tab.src[q] & 0x7fffffffu) + 1]++;
                for (std::size_t s2 = 0; s2 < 3 * nf3; ++s2) h.colptr[s2 + 1] += h.colptr[s2];
                h.rows.resize(nnz);
                h.ccoef.resize(nnz);
                h.entry_row.resize(nnz);
                std::vector<int32_t> fill(h.colptr.begin(), h.colptr.end() - 1);
                for (std::size_t e = 0; e < E; ++e)
                    for (int32_t q = h.tab.rowptr[e]; q < h.tab.rowptr[e + 1]; ++q) {
                        const uint32_t key = h.tab.src[q];
                        const int32_t dst = fill[key & 0x7fffffffu]++;
                        h.rows[dst] = static_cast<uint32_t>(e) | (key & 0x80000000u);
                        h.ccoef[dst] = h.tab.coef[q];
                        h.entry_row[q] = static_cast<uint32_t>(e);
                    }
            };
            {
                const std::size_t n = idx.size();
                const unsigned nth = n >= 4 ? std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency())) : 1u;
                if (nth <= 1) {
                    for (std::size_t a = 0; a < n; ++a) build_host(a);
                } else {
                    std::vector<std::thread> pool;
                    for (unsigned k = 0; k < nth; ++k)
                        pool.emplace_back([&, k] {
                            for (std::size_t a = k; a < n; a += nth) build_host(a);
                        });
                    for (auto& th : pool) th.join();
                }
            }
            for (std::size_t a = 0; a < idx.size(); ++a) {
                const Host& h = hs[a];
                const std::size_t nnz = h.tab.src.size();
                probe.take<int32_t>(h.colptr.size());
                probe.take<uint32_t>(nnz);
                probe.take<double2>(nnz);
                probe.take<uint32_t>(nnz);
                probe.take<uint32_t>(nnz);
                probe.take<double>(nf);
                probe.take<int>(nf);
                probe.take<uint8_t>(nf3);
            }
            probe.take<FcrAdjJob>(idx.size());
            probe.take<double2*>(idx.size());
            probe.take<SrcAdjJob>(idx.size());
            packed_bytes = probe.off;  // the uploaded arrays: one host image, one copy
            for (std::size_t a = 0; a < idx.size(); ++a) {
                const std::size_t nnz = hs[a].tab.src.size();
                probe.take<double2>(nnz);             // Z
                probe.take<double2>(3 * nf3 * T);     // src_bar
                probe.take<double2>(5 * nf3 * T);     // G1, G2F, G2C, G2R, A2
                probe.take<double>(nf3 * (1 + ntiles));
            }
            if (fftN) {  // twiddle tables, per-job spectra, their jobs
                FzPlan<double2> fp{};
                fp.N = fftN;
                fz_stages(fftN, 8, fp.rad, fp.nst);
                probe.take<double2>(std::max<std::size_t>(1, fz_table_layout(fp)));
                for (std::size_t a = 0; a < idx.size(); ++a) probe.take<double2>((2 * nf + 4 * nf3) * fftN);
                probe.take<AdjFftSpectra>(idx.size());
                probe.take<AdjSpecJob>(idx.size() * (2 * nf + 4 * nf3));
            }
            bytes = probe.off + 256;
        }
        Carve cv{grad_scratch().ensure(bytes)};
        std::vector<char> image(packed_bytes);
        // carve an array from the packed region and copy its host contents into the image
        auto pack = [&](const auto& v) {
            using T0 = typename std::decay_t<decltype(v)>::value_type;
            T0* d = cv.take<T0>(v.size());
            if (!v.empty()) std::memcpy(image.data() + (reinterpret_cast<char*>(d) - cv.base), v.data(), v.size() * sizeof(T0));
            return d;
        };
        std::vector<FcrAdjJob> fj(idx.size());
        std::vector<double2*> gbar(idx.size());
        struct Dev {
            int32_t* colptr;
            uint32_t* rows;
            double2* ccoef;
            uint32_t* erow;
            uint32_t* keys;
            double2* Z;
            double2* src_bar;
            double* wpart;
        };
        std::vector<Dev> dv(idx.size());
        std::vector<double*> dom_v(idx.size());
        std::vector<int*> dmir_v(idx.size());
        std::vector<uint8_t*> dused_v(idx.size());
        for (std::size_t a = 0; a < idx.size(); ++a) {
            const SystemDesc& s = *jobs[idx[a]].sys;
            Host& h = hs[a];
            Dev& d = dv[a];
            d.colptr = pack(h.colptr);
            d.rows = pack(h.rows);
            d.ccoef = pack(h.ccoef);
            d.erow = pack(h.entry_row);
            d.keys = pack(h.tab.src);
            dom_v[a] = pack(s.omegas);
            dmir_v[a] = pack(s.mirror);
            std::vector<uint8_t> used(nf3);
            for (std::size_t q = 0; q < nf3; ++q) used[q] = h.tab.triple_fc_used[q];
            dused_v[a] = pack(used);
        }
        FcrAdjJob* dfj = cv.take<FcrAdjJob>(idx.size());
        double2** dgbar = cv.take<double2*>(idx.size());
        SrcAdjJob* dsj = cv.take<SrcAdjJob>(idx.size());
        std::vector<SrcAdjJob> sj(idx.size());
        for (std::size_t a = 0; a < idx.size(); ++a) {
            const auto& j = jobs[idx[a]];
            Dev& d = dv[a];
            const std::size_t nnz = hs[a].tab.src.size();
            d.Z = cv.take<double2>(nnz);
            d.src_bar = cv.take<double2>(3 * nf3 * T);
            double2* parts = cv.take<double2>(5 * nf3 * T);
            d.wpart = cv.take<double>(nf3 * (1 + ntiles));
            double* dom = dom_v[a];
            int* dmir = dmir_v[a];
            uint8_t* dused = dused_v[a];
            const bool want_ops = j.ops_bar && j.F && j.C && j.R && nnz;
            sj[a] = SrcAdjJob{j.L_bar, d.colptr, d.rows, d.ccoef, d.src_bar, d.erow, d.keys,
                              static_cast<uint32_t>(want_ops ? nnz : 0), j.F, j.C, j.R, d.Z,
                              static_cast<uint32_t>(j.sys->N * j.sys->N * j.sys->N * j.sys->N)};
            FcrAdjJob& f = fj[a];
            f.gamma = j.gamma;
            f.Fb = d.src_bar;
            f.Cb = d.src_bar + nf3 * T;
            f.Rb = d.src_bar + 2 * nf3 * T;
            f.omegas = dom;
            f.mirror = dmir;
            f.fc_used = dused;
            f.G1 = parts;
            f.G2F = parts + nf3 * T;
            f.G2C = parts + 2 * nf3 * T;
            f.G2R = parts + 3 * nf3 * T;
            f.A2 = parts + 4 * nf3 * T;
            f.wpart = d.wpart;
            f.ntiles = ntiles;
            gbar[a] = j.gamma_bar;
        }
        // FFT correlations: spectra of conj(Gamma_b) and Gamma_b per job, and of the reversed
        // Fb, Cb, A2 and n A2[n] per triple (A2 is written by the scan kernel, which runs first)
        double2* roots = nullptr;
        AdjFftSpectra* dspec = nullptr;
        AdjSpecJob* dsjobs = nullptr;
        std::size_t nspec_jobs = 0;
        FzPlan<double2> fplan{};
        std::size_t ftab = 0;
        if (fftN) {
            fplan.N = fftN;
            fz_stages(fftN, 8, fplan.rad, fplan.nst);
            ftab = std::max<std::size_t>(1, fz_table_layout(fplan));
            roots = cv.take<double2>(ftab);
            std::vector<AdjFftSpectra> spv(idx.size());
            std::vector<AdjSpecJob> sjobs;
            const std::size_t N = static_cast<std::size_t>(fftN);
            for (std::size_t a = 0; a < idx.size(); ++a) {
                double2* base = cv.take<double2>((2 * nf + 4 * nf3) * N);
                AdjFftSpectra& sp = spv[a];
                sp.gconj = base;
                sp.gplain = base + nf * N;
                sp.fb = base + 2 * nf * N;
                sp.cb = sp.fb + nf3 * N;
                sp.a2 = sp.cb + nf3 * N;
                sp.a3 = sp.a2 + nf3 * N;
                const FcrAdjJob& f = fj[a];
                const uint32_t TT = static_cast<uint32_t>(T);
                for (int b = 0; b < nf; ++b) {
                    sjobs.push_back({f.gamma + static_cast<std::size_t>(b) * T, base + b * N, TT, 1});
                    sjobs.push_back({f.gamma + static_cast<std::size_t>(b) * T, base + (nf + b) * N, TT, 0});
                }
                for (std::size_t q = 0; q < nf3; ++q) {
                    sjobs.push_back({f.Fb + q * T, const_cast<double2*>(sp.fb) + q * N, TT, 2});
                    sjobs.push_back({f.Cb + q * T, const_cast<double2*>(sp.cb) + q * N, TT, 2});
                    sjobs.push_back({f.A2 + q * T, const_cast<double2*>(sp.a2) + q * N, TT, 0});
                    sjobs.push_back({f.A2 + q * T, const_cast<double2*>(sp.a3) + q * N, TT, 3});
                }
            }
            nspec_jobs = sjobs.size();
            dspec = cv.take<AdjFftSpectra>(idx.size());
            dsjobs = cv.take<AdjSpecJob>(nspec_jobs);
            cuda_check(cudaMemcpyAsync(dspec, spv.data(), spv.size() * sizeof(AdjFftSpectra), cudaMemcpyHostToDevice, st),
                       "adj fft spectra");
            cuda_check(cudaMemcpyAsync(dsjobs, sjobs.data(), nspec_jobs * sizeof(AdjSpecJob), cudaMemcpyHostToDevice, st),
                       "adj fft jobs");
            // the host vectors above are copy sources: finish before they go out of scope
            cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(adj fft jobs)");
            fplan.tw = roots;
            k_fz_fill_tables<double2><<<static_cast<unsigned>((ftab + 255) / 256), 256, 0, st>>>(
                roots, fplan, static_cast<uint32_t>(ftab));
            launched("k_fz_fill_tables");
        }
        std::memcpy(image.data() + (reinterpret_cast<char*>(dfj) - cv.base), fj.data(), fj.size() * sizeof(FcrAdjJob));
        std::memcpy(image.data() + (reinterpret_cast<char*>(dgbar) - cv.base), gbar.data(), gbar.size() * sizeof(double2*));
        std::memcpy(image.data() + (reinterpret_cast<char*>(dsj) - cv.base), sj.data(), sj.size() * sizeof(SrcAdjJob));
        cuda_check(cudaMemcpyAsync(cv.base, image.data(), packed_bytes, cudaMemcpyHostToDevice, st), "adj arrays");
        // 1. sources and the coupling-operator aggregation, all instances in one launch each
        {
            std::size_t max_nnz = 0;
            for (const auto& x : sj) max_nnz = std::max<std::size_t>(max_nnz, x.nnz);
            k_src_adj<<<dim3(static_cast<unsigned>((T + 127) / 128), static_cast<unsigned>(3 * nf3),
                             static_cast<unsigned>(idx.size())), 128, 0, st>>>(dsj, static_cast<uint32_t>(T));
            launched("k_src_adj");
            if (max_nnz) {
                k_coef_z<<<dim3(static_cast<unsigned>((max_nnz + 7) / 8), static_cast<unsigned>(idx.size())), 256, 0, st>>>(
                    dsj, static_cast<uint32_t>(T), static_cast<uint32_t>(nf3));
                launched("k_coef_z");
            }
        }
        // 2. F/C/R adjoint for every triple of every job
        const unsigned nj = static_cast<unsigned>(idx.size());
        for (std::size_t a = 0; a < idx.size(); ++a)
            cuda_check(cudaMemsetAsync(dv[a].wpart, 0, nf3 * (1 + ntiles) * sizeof(double), st), "adj wpart zero");
        k_fcr_adj_scan<<<dim3(static_cast<unsigned>(nf3), nj), SC_THREADS, 0, st>>>(dfj, nf, static_cast<uint32_t>(T),
                                                                                    jobs[idx[0]].dt);
        launched("k_fcr_adj_scan");
        if (fftN) {
            const FzPlan<double2> fp = fplan;
            const std::size_t fsm = fz_smem<double2>(fftN);
            raise_smem_limit(reinterpret_cast<const void*>(&k_adj_series_spectrum), fsm);
            raise_smem_limit(reinterpret_cast<const void*>(&k_fcr_adj_corr_fft), fsm);
            k_adj_series_spectrum<<<static_cast<unsigned>(nspec_jobs), FZ_THREADS, fsm, st>>>(dsjobs, fp);
            launched("k_adj_series_spectrum");
            k_fcr_adj_corr_fft<<<dim3(5, static_cast<unsigned>(nf3), nj), FZ_THREADS, fsm, st>>>(
                dfj, dspec, nf, static_cast<uint32_t>(T), jobs[idx[0]].dt, fp);
            launched("k_fcr_adj_corr_fft");
        } else {
            k_fcr_adj_corr<<<dim3(static_cast<unsigned>(ntiles), static_cast<unsigned>(nf3), nj), CR_TM, 0, st>>>(
                dfj, nf, static_cast<uint32_t>(T), jobs[idx[0]].dt);
            launched("k_fcr_adj_corr");
        }
        k_fcr_adj_reduce<<<dim3(static_cast<unsigned>((T + 127) / 128), static_cast<unsigned>(nf), nj), 128, 0, st>>>(
            dfj, nf, static_cast<uint32_t>(T), dgbar);
        launched("k_fcr_adj_reduce");
        // 3. host: Bohr-frequency and coupling-operator gradients (all partials copied back,
        // then one synchronisation)
        std::vector<std::vector<double>> wparts(idx.size(), std::vector<double>(nf3 * (1 + ntiles)));
        std::vector<std::vector<double2>> Zs(idx.size());
        for (std::size_t a = 0; a < idx.size(); ++a) {
            const auto& j = jobs[idx[a]];
            cuda_check(cudaMemcpyAsync(wparts[a].data(), dv[a].wpart, wparts[a].size() * sizeof(double),
                                       cudaMemcpyDeviceToHost, st),
                       "adj wpart");
            const std::size_t nnz = hs[a].tab.src.size();
            if (j.ops_bar && j.F && j.C && j.R && nnz) {
                Zs[a].resize(nnz);
                cuda_check(cudaMemcpyAsync(Zs[a].data(), dv[a].Z, nnz * sizeof(double2), cudaMemcpyDeviceToHost, st),
                           "adj Z");
            }
        }
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(tcl4 adjoint)");
        for (std::size_t a = 0; a < idx.size(); ++a) {
            const auto& j = jobs[idx[a]];
            const SystemDesc& s = *j.sys;
            const std::vector<double>& wpart = wparts[a];
            const std::vector<double2>& Z = Zs[a];
            const std::size_t nnz = hs[a].tab.src.size();
            const bool want_ops = j.ops_bar && j.F && j.C && j.R && nnz;
            if (j.omega_bar) {
                for (std::size_t q = 0; q < nf3; ++q) {
                    double wq = 0.0;
                    for (int x = 0; x <= ntiles; ++x) wq += wpart[q * (1 + ntiles) + x];
                    const int i = static_cast<int>(q / (nf * nf)), jj = static_cast<int>((q / nf) % nf),
                              kk = static_cast<int>(q % nf);
                    j.omega_bar[i] += wq;
                    j.omega_bar[jj] += wq;
                    j.omega_bar[kk] += wq;
                }
            }
            if (want_ops) coef_table_ops_grad(s.N, s.nf, s.p2f.data(), s.ops.data(), s.num_ops, hs[a].tab, Z.data(), j.ops_bar);
        }
    }
}

void tcl2_adjoint(const std::vector<Tcl2AdjointJob>& jobs, cudaStream_t st) {
    if (jobs.empty()) return;
    for (const auto& j : jobs)
        if (!j.sys || !j.eps || !j.gamma || !j.L_bar || !j.gamma_bar || j.T == 0)
            throw Error(kInvalidArgument, "tcl2 adjoint: null or empty input");
    const std::size_t n = jobs.size();
    const unsigned nth = n >= 4 ? std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency())) : 1u;
    auto parallel = [&](auto&& fn) {  // fn(k) for every job, on host threads
        if (nth <= 1) {
            for (std::size_t k = 0; k < n; ++k) fn(k);
            return;
        }
        std::vector<std::thread> pool;
        for (unsigned w = 0; w < nth; ++w)
            pool.emplace_back([&, w] {
                for (std::size_t k = w; k < n; k += nth) fn(k);
            });
        for (auto& th : pool) th.join();
    };
    // 1. host maps of every job
    std::vector<std::vector<double2>> Db(n), Ub(n);
    parallel([&](std::size_t k) {
        std::vector<double2> L0;
        tcl2_maps(*jobs[k].sys, jobs[k].eps, L0, Db[k], Ub[k]);
    });
    auto E_of = [&](std::size_t k) {
        const int N = jobs[k].sys->N;
        return static_cast<std::size_t>(N) * N * N * N;
    };
    auto want_maps = [&](std::size_t k) { return jobs[k].ops_bar || jobs[k].eps_bar; };
    // 2. device layout: D and U of every job and the job table (one upload), then the maps
    Carve probe{nullptr};
    for (std::size_t k = 0; k < n; ++k) {
        probe.take<double2>(Db[k].size());
        probe.take<double2>(Ub[k].size());
    }
    probe.take<Tcl2AdjJob>(n);
    const std::size_t packed = probe.off;
    for (std::size_t k = 0; k < n; ++k)
        if (want_maps(k)) probe.take<double2>((1 + 2 * jobs[k].sys->nf) * E_of(k));
    Carve cv{grad_scratch().ensure(probe.off + 256)};
    std::vector<char> image(packed);
    auto pack = [&](const std::vector<double2>& v) {
        double2* d = cv.take<double2>(v.size());
        if (!v.empty()) std::memcpy(image.data() + (reinterpret_cast<char*>(d) - cv.base), v.data(), v.size() * sizeof(double2));
        return d;
    };
    std::vector<Tcl2AdjJob> tj(n);
    for (std::size_t k = 0; k < n; ++k) {
        const auto& j = jobs[k];
        tj[k].Db = pack(Db[k]);
        tj[k].Ub = pack(Ub[k]);
        tj[k].Lb = j.L_bar;
        tj[k].gamma = j.gamma;
        tj[k].gbar = j.gamma_bar;
        tj[k].T = static_cast<uint32_t>(j.T);
        tj[k].E = static_cast<uint32_t>(E_of(k));
        tj[k].nf = j.sys->nf;
    }
    Tcl2AdjJob* dj = cv.take<Tcl2AdjJob>(n);
    std::vector<double2*> maps(n, nullptr);
    for (std::size_t k = 0; k < n; ++k)
        if (want_maps(k)) maps[k] = tj[k].maps = cv.take<double2>((1 + 2 * jobs[k].sys->nf) * E_of(k));
    std::memcpy(image.data() + (reinterpret_cast<char*>(dj) - cv.base), tj.data(), n * sizeof(Tcl2AdjJob));
    cuda_check(cudaMemcpyAsync(cv.base, image.data(), packed, cudaMemcpyHostToDevice, st), "tcl2 adj arrays");
    // 3. G(Gamma) of every job; the aggregated maps where operator or energy gradients are wanted
    std::size_t Tmax = 0, Emax = 0;
    bool any_maps = false;
    for (std::size_t k = 0; k < n; ++k) {
        Tmax = std::max(Tmax, jobs[k].T);
        Emax = std::max(Emax, E_of(k));
        any_maps = any_maps || want_maps(k);
    }
    k_tcl2_adj_gamma<<<dim3(static_cast<unsigned>((Tmax + 127) / 128), static_cast<unsigned>(n)), 128, 0, st>>>(dj);
    launched("k_tcl2_adj_gamma");
    std::vector<std::vector<double2>> h(n);
    if (any_maps) {
        k_tcl2_adj_maps<<<dim3(static_cast<unsigned>(Emax), static_cast<unsigned>(n)), 256, 0, st>>>(dj);
        launched("k_tcl2_adj_maps");
        for (std::size_t k = 0; k < n; ++k)
            if (maps[k]) {
                h[k].resize((1 + 2 * jobs[k].sys->nf) * E_of(k));
                cuda_check(cudaMemcpyAsync(h[k].data(), maps[k], h[k].size() * sizeof(double2), cudaMemcpyDeviceToHost, st),
                           "tcl2 adj maps");
            }
    }
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(tcl2 adjoint)");
    // 4. host: reverse the construction of the maps (on threads unless jobs share a
    // gradient buffer, whose accumulation must then stay sequential)
    bool shared_out = false;
    {
        std::vector<const void*> outs;
        for (const auto& j : jobs) {
            if (j.ops_bar) outs.push_back(j.ops_bar);
            if (j.eps_bar) outs.push_back(j.eps_bar);
        }
        std::sort(outs.begin(), outs.end());
        shared_out = std::adjacent_find(outs.begin(), outs.end()) != outs.end();
    }
    auto host_grad = [&](std::size_t k) {
        if (!maps[k]) return;
        const auto& j = jobs[k];
        const int nf = j.sys->nf;
        const std::size_t E = E_of(k);
        std::vector<double2> GL0(h[k].begin(), h[k].begin() + static_cast<std::ptrdiff_t>(E)), GD(nf * E), GU(nf * E);
        for (int b = 0; b < nf; ++b)
            for (std::size_t e = 0; e < E; ++e) {
                GD[b * E + e] = h[k][(1 + 2 * b) * E + e];
                GU[b * E + e] = h[k][(2 + 2 * b) * E + e];
            }
        tcl2_maps_grad(*j.sys, j.eps, GL0, GD, GU, j.ops_bar, j.eps_bar);
    };
    if (shared_out) {
        for (std::size_t k = 0; k < n; ++k) host_grad(k);
    } else {
        parallel(host_grad);
    }
}

void inner_re_device(const std::vector<InnerRequest>& reqs, double* out, cudaStream_t st) {
    if (reqs.empty()) return;
    std::vector<InnerJob> js(reqs.size());
    for (std::size_t k = 0; k < reqs.size(); ++k) {
        if (!reqs[k].a || !reqs[k].b) throw Error(kInvalidArgument, "inner: null pointer");
        js[k] = InnerJob{reqs[k].a, reqs[k].b, reqs[k].n};
    }
    Carve probe{nullptr};
    probe.take<InnerJob>(js.size());
    probe.take<double>(js.size());
    Carve cv{grad_scratch().ensure(probe.off + 256)};
    InnerJob* dj = upload(cv, js, st, "inner jobs");
    double* dout = cv.take<double>(js.size());
    for (std::size_t k0 = 0; k0 < js.size(); k0 += 65535) {
        const unsigned n = static_cast<unsigned>(std::min<std::size_t>(65535, js.size() - k0));
        k_inner_re<<<n, 256, 0, st>>>(dj + k0, dout + k0);
        launched("k_inner_re");
    }
    cuda_check(cudaMemcpyAsync(out, dout, js.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "inner out");
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(inner)");
}

}  // namespace taco
