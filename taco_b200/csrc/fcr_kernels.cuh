// fcr_kernels.cuh -- device kernels of the F/C/R stage.
//
// The causal convolutions of the F and C kernels are computed with a four-step FFT of
// length Nfft = N1*N2 (both powers of two, at most 2048):
//   B1  column pass: x[t] generated on the fly (gamma column, optional phase
//       exp(-i w t dt), optional conjugate; zero for t >= n_in), N1-point FFTs down the
//       columns, inter-step twiddle w_N^(n2*k1), stored as Z[k1*N2 + n2];
//   B2  row pass: N2-point FFT of each row -> spectrum row in the permuted order
//       S[k1*N2 + k2]; multiplied by the hoisted spectra of the two partner series
//       (F: gamma[:, mirror j]; C: conj gamma[:, j]), both products transformed back
//       along the row and twiddled by w_N^(-n2*k1) (the spectrum of x never leaves
//       shared memory);
//   B3  inverse column pass: N1-point inverse FFTs down the columns, scaled by dt/Nfft,
//       only samples t <= t_max written.
// The spectra of gamma[:, b] and conj(gamma[:, b]) are produced once per instance by
// B1 + a plain forward row pass.
// The scan kernel forms the three prefix integrals per triple (P_F, P_R1, P_R2;
// P_C = conj(P_R1)) with FP64 carries and assembles F, C, R at the requested times.
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace taco {

template <class C>
struct FftPlan {
    int L, L1, L2, s;  // Nfft = 2^L, N1 = 2^L1 (column length), N2 = 2^L2 (row length)
    const C* tw1;      // exp(-2 pi i m / N1), m < N1
    const C* tw2;      // exp(-2 pi i m / N2), m < N2
    const C* twc;      // exp(-2 pi i m 2^s / N), m < N / 2^s
    const C* twf;      // exp(-2 pi i m / N), m < 2^s
};

// w_N^a for 0 <= a < N as the product of a coarse and a fine table entry.
template <class C>
__device__ __forceinline__ C inter_twiddle(const FftPlan<C>& p, uint32_t a) {
    const uint32_t hi = a >> p.s, lo = a & ((1u << p.s) - 1u);
    return cmul(__ldg(&p.twc[hi]), __ldg(&p.twf[lo]));
}

struct ColJob {
    const double2* g;  // gamma column, n_in valid samples
    double omega;      // phase exp(-i omega t dt) applied when has_phase
    double dt;
    int has_phase;
    int conj;
    uint32_t n_in;     // samples t >= n_in are zero (zero padding)
    void* out;         // Z [Nfft] of the working complex type
};

struct RowJob {
    void* data;        // in: Z; out: W_F (or the spectrum when spec_f == nullptr)
    void* wc;          // out: W_C
    const void* spec_f;
    const void* spec_c;
};

struct InvJob {
    const void* w;     // W [Nfft]
    void* out;         // conv [t_count]
    uint32_t t_count;  // number of leading samples kept (t_max + 1)
    double scale;      // dt / Nfft
};

struct ScanJob {
    const double2* gi;
    const double2* gj;
    const double2* gmj;
    double omega;
    double dt;
    uint32_t t_count;  // t_max + 1
    const void* conv_f;
    const void* conv_c;
    const int* tmap;   // [t_count] -> position in the output series, or -1
    void* vf;          // F series at the unique requested times [U]
    void* vc;
    void* vr;
};

__device__ __forceinline__ double2 phase_minus(double omega, double dt, uint32_t t) {
    const double tk = static_cast<double>(t) * dt;  // t_k = k dt, then exp(-i omega t_k)
    double sn, cs;
    sincos(-(omega * tk), &sn, &cs);
    return make_double2(cs, sn);
}

// ---------------------------------------------------------------- B1 -------
template <class R>
__global__ void k_fwd_col(const ColJob* __restrict__ jobs, FftPlan<cplx_t<R>> plan, int C_cols) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    const ColJob job = jobs[blockIdx.y];
    const int N1 = 1 << plan.L1, N2 = 1 << plan.L2;
    const int n2_0 = blockIdx.x * C_cols;
    const int elems = N1 * C_cols;
    for (int idx = threadIdx.x; idx < elems; idx += blockDim.x) {
        const int n1 = idx / C_cols, c = idx - n1 * C_cols;
        const uint32_t t = static_cast<uint32_t>(n1) * N2 + n2_0 + c;
        double2 v = make_double2(0.0, 0.0);
        if (t < job.n_in) {
            v = __ldg(&job.g[t]);
            if (job.conj) v.y = -v.y;
            if (job.has_phase) v = cmul(v, phase_minus(job.omega, job.dt, t));
        }
        s[idx] = from_d2<C>(v);
    }
    __syncthreads();
    tile_fft<C, false>(s, plan.L1, 1, C_cols, plan.tw1);
    C* out = static_cast<C*>(job.out);
    for (int idx = threadIdx.x; idx < elems; idx += blockDim.x) {
        const int k1 = idx / C_cols, c = idx - k1 * C_cols;
        const uint32_t n2 = n2_0 + c;
        out[static_cast<size_t>(k1) * N2 + n2] = cmul(s[idx], inter_twiddle(plan, n2 * static_cast<uint32_t>(k1)));
    }
}

// ---------------------------------------------------------------- B2 -------
// Forward row FFT; with spec_f set: two spectral products, inverse row FFTs and the
// inverse inter-step twiddle.  Shared memory: two tiles of rows*N2 elements.
template <class R>
__global__ void k_row(const RowJob* __restrict__ jobs, FftPlan<cplx_t<R>> plan, int rows) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int N2 = 1 << plan.L2;
    const int elems = rows * N2;
    C* a = reinterpret_cast<C*>(smem_raw);
    C* p = a + elems;
    const RowJob job = jobs[blockIdx.y];
    const size_t off = static_cast<size_t>(blockIdx.x) * elems;
    C* data = static_cast<C*>(job.data) + off;
    for (int idx = threadIdx.x; idx < elems; idx += blockDim.x) a[idx] = data[idx];
    __syncthreads();
    tile_fft<C, false>(a, plan.L2, N2, 1, plan.tw2);
    if (job.spec_f == nullptr) {
        for (int idx = threadIdx.x; idx < elems; idx += blockDim.x) data[idx] = a[idx];
        return;
    }
    const int k1_0 = blockIdx.x * rows;
    for (int which = 0; which < 2; ++which) {
        const C* spec = static_cast<const C*>(which == 0 ? job.spec_f : job.spec_c) + off;
        for (int idx = threadIdx.x; idx < elems; idx += blockDim.x) p[idx] = cmul(a[idx], spec[idx]);
        __syncthreads();
        tile_fft<C, true>(p, plan.L2, N2, 1, plan.tw2);
        C* dst = (which == 0 ? data : static_cast<C*>(job.wc) + off);
        for (int idx = threadIdx.x; idx < elems; idx += blockDim.x) {
            const int r = idx >> plan.L2, n2 = idx & (N2 - 1);
            const uint32_t k1 = static_cast<uint32_t>(k1_0 + r);
            dst[idx] = cmulc(p[idx], inter_twiddle(plan, static_cast<uint32_t>(n2) * k1));
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- B3 -------
template <class R>
__global__ void k_inv_col(const InvJob* __restrict__ jobs, FftPlan<cplx_t<R>> plan, int C_cols) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    const InvJob job = jobs[blockIdx.y];
    const int N1 = 1 << plan.L1, N2 = 1 << plan.L2;
    const int n2_0 = blockIdx.x * C_cols;
    const int elems = N1 * C_cols;
    const C* w = static_cast<const C*>(job.w);
    for (int idx = threadIdx.x; idx < elems; idx += blockDim.x) {
        const int k1 = idx / C_cols, c = idx - k1 * C_cols;
        s[idx] = w[static_cast<size_t>(k1) * N2 + n2_0 + c];
    }
    __syncthreads();
    tile_fft<C, true>(s, plan.L1, 1, C_cols, plan.tw1);
    C* out = static_cast<C*>(job.out);
    const R scale = static_cast<R>(job.scale);
    for (int idx = threadIdx.x; idx < elems; idx += blockDim.x) {
        const int n1 = idx / C_cols, c = idx - n1 * C_cols;
        const uint32_t t = static_cast<uint32_t>(n1) * N2 + n2_0 + c;
        if (t < job.t_count) out[t] = cscale(s[idx], scale);
    }
}

// ---------------------------------------------------------------- scans ----
__device__ __forceinline__ void add6(double* a, const double* b) {
#pragma unroll
    for (int q = 0; q < 6; ++q) a[q] += b[q];
}

// One CTA per triple; SCAN_ITEMS consecutive samples per thread; FP64 carries.
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 4;

template <class R>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_assemble(const ScanJob* __restrict__ jobs) {
    using C = cplx_t<R>;
    __shared__ double warp_tot[SCAN_THREADS / 32][6];
    __shared__ double carry_sh[6];
    const ScanJob job = jobs[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double carry[6] = {0, 0, 0, 0, 0, 0};
    const C* cf = static_cast<const C*>(job.conv_f);
    const C* cc = static_cast<const C*>(job.conv_c);
    C* vf = static_cast<C*>(job.vf);
    C* vc = static_cast<C*>(job.vc);
    C* vr = static_cast<C*>(job.vr);
    const uint32_t tile = SCAN_THREADS * SCAN_ITEMS;
    for (uint32_t t0 = 0; t0 < job.t_count; t0 += tile) {
        // integrands: y0 = g_mj e^{+iwt}, y1 = g_j e^{-iwt}, y2 = g_i g_j e^{-iwt}
        double y[SCAN_ITEMS][6];
        double run[6] = {0, 0, 0, 0, 0, 0};
        const uint32_t tb = t0 + threadIdx.x * SCAN_ITEMS;
#pragma unroll
        for (int q = 0; q < SCAN_ITEMS; ++q) {
            const uint32_t t = tb + q;
            double v[6] = {0, 0, 0, 0, 0, 0};
            if (t < job.t_count) {
                const double2 pm = phase_minus(job.omega, job.dt, t);
                const double2 gmj = __ldg(&job.gmj[t]);
                const double2 gj = __ldg(&job.gj[t]);
                const double2 gi = __ldg(&job.gi[t]);
                const double2 a = cmulc(gmj, pm);  // g_mj * e^{+iwt}
                const double2 b = cmul(gj, pm);
                const double2 c = cmul(cmul(gi, gj), pm);
                v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = c.x; v[5] = c.y;
            }
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                run[k] += v[k];
                y[q][k] = run[k];
            }
        }
        // exclusive scan of the per-thread totals across the block
        double incl[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            double x = run[k];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double nb = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += nb;
            }
            incl[k] = x;
        }
        if (lane == 31) {
#pragma unroll
            for (int k = 0; k < 6; ++k) warp_tot[warp][k] = incl[k];
        }
        __syncthreads();
        double pre[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            double excl = __shfl_up_sync(0xffffffffu, incl[k], 1);
            if (lane == 0) excl = 0.0;
            double w = 0.0;
            for (int q = 0; q < warp; ++q) w += warp_tot[q][k];
            pre[k] = carry[k] + (w + excl);
        }
#pragma unroll
        for (int q = 0; q < SCAN_ITEMS; ++q) {
            const uint32_t t = tb + q;
            if (t >= job.t_count) break;
            const int u = __ldg(&job.tmap[t]);
            if (u < 0) continue;
            const double2 PF = make_double2((pre[0] + y[q][0]) * job.dt, (pre[1] + y[q][1]) * job.dt);
            const double2 PR1 = make_double2((pre[2] + y[q][2]) * job.dt, (pre[3] + y[q][3]) * job.dt);
            const double2 PR2 = make_double2((pre[4] + y[q][4]) * job.dt, (pre[5] + y[q][5]) * job.dt);
            const double2 pm = phase_minus(job.omega, job.dt, t);
            const double2 gi = __ldg(&job.gi[t]);
            const double2 gip = cmul(gi, pm);
            const double2 convf = to_d2(cf[t]);
            const double2 convc = to_d2(cc[t]);
            vf[u] = from_d2<C>(csub(cmul(gip, PF), convf));
            vc[u] = from_d2<C>(csub(cmulc(gip, PR1), convc));  // P_C = conj(P_R1)
            vr[u] = from_d2<C>(csub(cmul(gi, PR1), PR2));
        }
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                double w = 0.0;
                for (int q = 0; q < SCAN_THREADS / 32; ++q) w += warp_tot[q][k];
                carry_sh[k] = carry[k] + w;
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 6; ++k) carry[k] = carry_sh[k];
        __syncthreads();
    }
}

}  // namespace taco
