// cluster_conv.cuh -- whole F/C convolutions of one triple inside a thread-block cluster.
//
// For Nfft = K * M with K <= 8 CTAs in a cluster and M points per CTA in shared memory,
// the length-Nfft transform splits as
//   forward  X[p + K k] = FFT_M( y_p )[k],   y_p[n] = w_N^(p n) sum_q x[n + q M] w_K^(p q)
//   inverse  x[n + q M] = (1/N) sum_p w_N^(-p n) w_K^(-p q) u_p[n],   u_p = IFFT_M(P_p)
// (a radix-K first stage across the cluster, then M-point FFTs local to each CTA).  CTA p
// of the cluster owns the M spectral values X[p + K k].  The radix-K stages read the peer
// CTAs' shared memory through distributed shared memory; the spectrum of the operand, the
// two spectral products and the two inverse transforms never leave the chip.  Only
// the Gamma samples (the operand is generated on the fly), the partner spectra (stored in
// the same [K][M] order by the same kernel in spectrum mode) and the t < t_count outputs
// touch global memory.
//
// Operand: x[t] = (g[t] - g[n_in-1]) (conj when job.conj) (* exp(-i w t dt) when
// has_phase) for t < n_in, zero beyond (the shifted form of fcr_kernels.cuh).
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"
#include "fcr_kernels.cuh"
#include "fft.cuh"

namespace taco {

struct ClusterPlanBase {
    int LN, LM, s;  // Nfft = 2^LN, M = 2^LM points per CTA, fine-table bits s
};

template <class C>
struct ClusterPlan : ClusterPlanBase {
    const C* twM;  // exp(-2 pi i m / M), m < M
    const C* twc;  // exp(-2 pi i m 2^s / N), m < N / 2^s
    const C* twf;  // exp(-2 pi i m / N), m < 2^s
};

struct ClusterJob {
    const double2* g;    // gamma column (n_in valid samples)
    double omega;
    double dt;
    int has_phase;
    int conj;
    uint32_t n_in;
    uint32_t t_count;    // outputs kept (conv mode)
    double scale;        // dt / Nfft (conv mode)
    const void* spec_f;  // [K][M] partner spectra (conv mode)
    const void* spec_c;
    void* out_f;         // conv mode: conv_F [t_count]; spectrum mode: spectrum [K][M]
    void* out_c;         // conv mode: conv_C [t_count]; spectrum mode: unused
};

template <class C>
__device__ __forceinline__ C wN(const ClusterPlan<C>& p, uint32_t a) {  // exp(-2 pi i a / N), a < N
    const uint32_t hi = a >> p.s, lo = a & ((1u << p.s) - 1u);
    return cmul(__ldg(&p.twc[hi]), __ldg(&p.twf[lo]));
}

// spectrum mode (spec_f == nullptr): write X_p to out_f + p*M; conv mode: F and C outputs.
template <class R, int KLOG>
__global__ void __launch_bounds__(sizeof(R) == 8 ? 512 : 1024) k_conv_cluster(const ClusterJob* __restrict__ jobs, ClusterPlan<cplx_t<R>> plan) {
    using C = cplx_t<R>;
    namespace cg = cooperative_groups;
    constexpr int K = 1 << KLOG;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    const int p = static_cast<int>(cluster.block_rank());
    const ClusterJob job = jobs[blockIdx.x >> KLOG];
    const int M = 1 << plan.LM;
    C* A = reinterpret_cast<C*>(smem_raw);
    C* B = A + padded_size<C>(M);
    const int nth = blockDim.x;  // == M / 8

    // 1. own segment of the operand: A[n] = x[p M + n]
    {
        const double2 shift = __ldg(&job.g[job.n_in - 1]);
        double2 v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const uint32_t t = static_cast<uint32_t>(p) * M + threadIdx.x + q * nth;
            v[q] = t < job.n_in ? __ldg(&job.g[t]) : shift;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int n = threadIdx.x + q * nth;
            const uint32_t t = static_cast<uint32_t>(p) * M + n;
            double2 x = csub(v[q], shift);
            if (job.conj) x.y = -x.y;
            if (job.has_phase && t < job.n_in) x = cmul(x, phase_minus(job.omega, job.dt, t));
            A[pad_idx<C>(n)] = from_d2<C>(x);
        }
    }
    cluster.sync();
    // 2. y_p[n] = w_N^(p n) sum_q A_q[n] w_K^(p q) over the segments that hold samples
    const int nseg = min(K, static_cast<int>((job.n_in + M - 1) / M));
#pragma unroll 2
    for (int e = 0; e < 8; ++e) {
        const int n = threadIdx.x + e * nth;
        C acc = C{0, 0};
#pragma unroll 1
        for (int q = 0; q < K; ++q) {
            if (q < nseg) {
                const C* Aq = cluster.map_shared_rank(A, q);
                const C x = Aq[pad_idx<C>(n)];
                const uint32_t kq = static_cast<uint32_t>((p * q) & (K - 1)) << plan.LM;  // w_K^(pq) = w_N^(pq M)
                acc = cadd(acc, q == 0 ? x : cmul(x, wN(plan, kq)));
            }
        }
        B[pad_idx<C>(n)] = p == 0 ? acc : cmul(acc, wN(plan, static_cast<uint32_t>(p) * n));
    }
    cluster.sync();  // every peer has read this CTA's A
    // 3. local forward transform: B = X_p
    tile_fft<C, false, false>(B, plan.LM, 0, 0, 1, plan.twM);
    if (job.spec_f == nullptr) {
        C* out = static_cast<C*>(job.out_f) + static_cast<size_t>(p) * M;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int n = threadIdx.x + q * nth;
            out[n] = B[pad_idx<C>(n)];
        }
        return;
    }
    const R scale = static_cast<R>(job.scale);
    const int nout = min(K, static_cast<int>((job.t_count + M - 1) / M));
    for (int which = 0; which < 2; ++which) {
        // 4. product with the partner spectrum and local inverse transform (into A)
        const C* spec = static_cast<const C*>(which == 0 ? job.spec_f : job.spec_c) + static_cast<size_t>(p) * M;
        C sv[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) sv[q] = __ldg(&spec[threadIdx.x + q * nth]);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int n = threadIdx.x + q * nth;
            A[pad_idx<C>(n)] = cmul(B[pad_idx<C>(n)], sv[q]);
        }
        __syncthreads();
        tile_fft<C, true, false>(A, plan.LM, 0, 0, 1, plan.twM);
        cluster.sync();
        // 5. segment q = p of the output: x[n + p M] = sum_r w_N^(-r n) w_K^(-r p) u_r[n]
        if (p < nout) {
            C* out = static_cast<C*>(which == 0 ? job.out_f : job.out_c);
#pragma unroll 2
            for (int e = 0; e < 8; ++e) {
                const int n = threadIdx.x + e * nth;
                const uint32_t t = static_cast<uint32_t>(p) * M + n;
                if (t >= job.t_count) continue;
                C acc = C{0, 0};
#pragma unroll 1
                for (int rr = 0; rr < K; ++rr) {
                    const C* Ar = cluster.map_shared_rank(A, rr);
                    C x = Ar[pad_idx<C>(n)];
                    if (rr > 0) {
                        const uint32_t a = (static_cast<uint32_t>(rr) * n +
                                            ((static_cast<uint32_t>((rr * p) & (K - 1))) << plan.LM)) &
                                           ((1u << plan.LN) - 1u);
                        x = cmulc(x, wN(plan, a));  // * w_N^(-(r n + r p M))
                    }
                    acc = cadd(acc, x);
                }
                out[t] = cscale(acc, scale);
            }
        }
        cluster.sync();  // every peer has read this CTA's A before it is rewritten
    }
}

}  // namespace taco
