// fused_conv.cuh -- one CTA per (triple, half): the F or C convolution of a triple held
// entirely in shared memory, followed by the prefix scans and the F/C/R assembly.
//
// For FFT lengths whose working array fits one CTA's shared memory (FP32 up to 24576
// points, FP64 up to 12288), the three global passes of the four-step path (column pass,
// row pass with the spectral products, inverse column pass, each a round trip through
// HBM) and the separate scan kernel become one kernel per (triple, half):
//   1. x[t] = (g_i[t] - g_i[n_in-1]) e^{-i w t dt} for t < n_in, 0 beyond (FP64 phases);
//   2. in-place decimation-in-frequency FFT: natural order in, digit-reversed spectrum out;
//   3. product with the partner spectrum (half F: d of gamma[:, mirror j]; half C: conj d
//      of gamma[:, j]), produced by the same forward transform and so in the same order,
//      and the scale dt / N;
//   4. in-place decimation-in-time inverse FFT with the stages in reverse order:
//      digit-reversed in, natural order out -- the causal convolution at t <= t_max;
//   5. the prefix integrals (FP64 sums and carries) and the assembly of F and R (half F) or
//      C (half C) at the requested times, the convolution read from shared memory.
// Stage s of the forward transform splits blocks of length M into RAD strided sub-blocks
// of length m = M / RAD: y_p = sum_q x[j + q m] w_RAD^{pq}, times w_M^{pj}, written back
// to j + p m (every butterfly reads and writes the same slots, so a stage needs no second
// buffer).  The odd radix (3 or 5) comes first, so every later m is a power of two.
// Twiddles come from per-stage tables laid out [p - 1][j], so that for one p consecutive
// butterflies read consecutive entries (coalesced), each entry evaluated directly in FP64.  The two halves of a triple repeat the forward
// transform (one more transform per triple than the four-step path) so that one
// 20480-point FP32 array is all a CTA holds.
#pragma once

#include "common.cuh"
#include "fcr_kernels.cuh"
#include "fft.cuh"

namespace taco {

constexpr int FZ_THREADS = 512;
constexpr int FZ_MAX_STAGES = 8;
constexpr int FZ_ITEMS = 2;  // samples per thread per scan tile

template <class C>
struct FzPlan {
    int N;
    int nst;                    // stages of the forward transform
    int rad[FZ_MAX_STAGES];     // radix of each stage (odd radix first)
    int twoff[FZ_MAX_STAGES];   // offset of each stage's twiddles in tw
    const C* tw;                // per stage s (block length M, sub-block m): w_M^(p j) at
                                // twoff[s] + (p - 1) m + j, p = 1..rad-1, j < m
};

// Shared memory of the fused kernels: the padded working array and the scan scratch.
template <class C>
constexpr std::size_t fz_scan_scratch() {
    return sizeof(double) * (2 * (FZ_THREADS / 32) * 8 + 2 * 8) + 2 * sizeof(double2);
}
// Byte offset of the scan scratch: after the working array, 16-byte aligned (it holds
// double2 values; the FP32 array's size is only a multiple of 8 bytes).
template <class C>
__host__ __device__ __forceinline__ std::size_t fz_scratch_off(int N) {
    return (static_cast<std::size_t>(padded_size<C>(N)) * sizeof(C) + 15) / 16 * 16;
}
template <class C>
inline std::size_t fz_smem(int N) {
    return fz_scratch_off<C>(N) + fz_scan_scratch<C>() + 64;
}

// Stage list for N = R * 2^L, R in {1, 3, 5}: the odd radix, stages of max_radix (16 for
// FP32, 8 for FP64: register budget), then the remaining power of two.
inline bool fz_stages(int N, int max_radix, int* rad, int& nst) {
    int R = 1;
    if (N % 5 == 0) R = 5;
    else if (N % 3 == 0) R = 3;
    int p = N / R;
    if (p <= 0 || (p & (p - 1))) return false;
    nst = 0;
    if (R > 1) rad[nst++] = R;
    while (p >= max_radix) {
        rad[nst++] = max_radix;
        p /= max_radix;
    }
    if (p > 1) rad[nst++] = p;
    return nst <= FZ_MAX_STAGES;
}

// Offsets of the per-stage twiddle tables; returns the number of entries.  A stage's table
// is [p - 1][j]: for one p, consecutive butterflies j read consecutive entries.
template <class C>
inline std::size_t fz_table_layout(FzPlan<C>& p) {
    std::size_t off = 0;
    int M = p.N;
    for (int s = 0; s < p.nst; ++s) {
        const int m = M / p.rad[s];
        p.twoff[s] = static_cast<int>(off);
        off += static_cast<std::size_t>(p.rad[s] - 1) * m;
        M = m;
    }
    return off;
}

// (stage block length M, p, j) of table entry e, for filling the tables.
template <class C>
__host__ __device__ inline void fz_table_entry(const FzPlan<C>& p, std::size_t e, int& M, int& pp, int& j) {
    M = p.N;
    for (int s = 0; s < p.nst; ++s) {
        const int m = M / p.rad[s];
        const std::size_t end = (s + 1 < p.nst) ? static_cast<std::size_t>(p.twoff[s + 1])
                                                : static_cast<std::size_t>(p.twoff[s]) + static_cast<std::size_t>(p.rad[s] - 1) * m;
        if (e < end) {
            const std::size_t k = e - p.twoff[s];
            pp = static_cast<int>(k / m) + 1;
            j = static_cast<int>(k % m);
            return;
        }
        M = m;
    }
    M = 1;
    pp = 0;
    j = 0;
}

// w16^e constants (forward sign), e = n2 * k1 in {0, 1, 2, 3, 4, 6, 9}
template <class C, bool INV>
__host__ __device__ __forceinline__ C w16(int e, C a) {
    using R = decltype(a.x);
    const R c1 = static_cast<R>(0.92387953251128675613), s1 = static_cast<R>(0.38268343236508977173);
    const R h = static_cast<R>(0.70710678118654752440);
    C w;
    switch (e) {
        case 1: w = C{c1, -s1}; break;
        case 2: w = C{h, -h}; break;
        case 3: w = C{s1, -c1}; break;
        case 4: w = C{0, -1}; break;
        case 6: w = C{-h, -h}; break;
        case 9: w = C{-c1, s1}; break;
        default: return a;
    }
    return INV ? cmulc(a, w) : cmul(a, w);
}

template <class C, bool INV>
__host__ __device__ __forceinline__ void dft16(C* x) {
    // n = n2 + 4 n1, k = k1 + 4 k2: 4-point DFTs over n1, twiddles w16^(n2 k1), 4-point
    // DFTs over n2
    C a[16];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
        C c0 = x[n2], c1 = x[n2 + 4], c2 = x[n2 + 8], c3 = x[n2 + 12];
        dft4<C, INV>(c0, c1, c2, c3);
        a[n2 * 4 + 0] = c0;
        a[n2 * 4 + 1] = w16<C, INV>(n2, c1);
        a[n2 * 4 + 2] = w16<C, INV>(2 * n2, c2);
        a[n2 * 4 + 3] = w16<C, INV>(3 * n2, c3);
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        C d0 = a[k1], d1 = a[4 + k1], d2 = a[8 + k1], d3 = a[12 + k1];
        dft4<C, INV>(d0, d1, d2, d3);
        x[k1] = d0;
        x[k1 + 4] = d1;
        x[k1 + 8] = d2;
        x[k1 + 12] = d3;
    }
}

template <class C, int RAD, bool INV>
__host__ __device__ __forceinline__ void fz_dft(C* x) {
    if constexpr (RAD == 2) dft2<C, INV>(x[0], x[1]);
    else if constexpr (RAD == 3) dft3<C, INV>(x[0], x[1], x[2]);
    else if constexpr (RAD == 4) dft4<C, INV>(x[0], x[1], x[2], x[3]);
    else if constexpr (RAD == 5) dft5<C, INV>(x);
    else if constexpr (RAD == 8) dft8<C, INV>(x);
    else dft16<C, INV>(x);
}

// The RAD - 1 twiddles w_M^(p j), p = 1..RAD-1, of one butterfly, from its stage's table
// ([p - 1][j], m entries per p).
template <class C, int RAD>
__host__ __device__ __forceinline__ void fz_twiddles(const C* __restrict__ tw, int j, int m, C* w) {
#pragma unroll
    for (int p = 1; p < RAD; ++p) w[p] = tw[(p - 1) * m + j];
}

// One stage on blocks of length M (m = M / RAD a power of two, log2 lm), butterflies
// tid, tid + nthr, ...; tw is the stage's table.  Forward: DFT then twiddles; inverse:
// conjugate twiddles then DFT.
template <class C, int RAD, bool INV>
__host__ __device__ __forceinline__ void fz_stage(C* d, int N, int M, int lm, const C* __restrict__ tw, int tid,
                                                  int nthr) {
    const int m = 1 << lm;
    const int nbf = N / RAD;
    (void)M;
    for (int bf = tid; bf < nbf; bf += nthr) {
        const int blk = bf >> lm, j = bf & (m - 1);
        const int base = blk * (RAD << lm) + j;
        C x[RAD];
#pragma unroll
        for (int q = 0; q < RAD; ++q) x[q] = d[pad_idx<C>(base + q * m)];
        C w[RAD];
        if (j) fz_twiddles<C, RAD>(tw, j, m, w);
        if (INV && j) {
#pragma unroll
            for (int q = 1; q < RAD; ++q) x[q] = cmulc(x[q], w[q]);
        }
        fz_dft<C, RAD, INV>(x);
        if (!INV && j) {
#pragma unroll
            for (int p = 1; p < RAD; ++p) x[p] = cmul(x[p], w[p]);
        }
#pragma unroll
        for (int p = 0; p < RAD; ++p) d[pad_idx<C>(base + p * m)] = x[p];
    }
}

template <class C, bool INV>
__host__ __device__ __forceinline__ void fz_stage_any(C* d, int N, int M, int r, int lm, const C* tw, int tid, int nthr) {
    switch (r) {
        case 2: fz_stage<C, 2, INV>(d, N, M, lm, tw, tid, nthr); break;
        case 3: fz_stage<C, 3, INV>(d, N, M, lm, tw, tid, nthr); break;
        case 4: fz_stage<C, 4, INV>(d, N, M, lm, tw, tid, nthr); break;
        case 5: fz_stage<C, 5, INV>(d, N, M, lm, tw, tid, nthr); break;
        case 8: fz_stage<C, 8, INV>(d, N, M, lm, tw, tid, nthr); break;
        default:
            // radix 16 for FP32 only: FP64 plans stop at 8 (register budget), and leaving the
            // FP64 radix-16 body out keeps it from setting the kernels' register allocation
            if constexpr (sizeof(C) == 8) fz_stage<C, 16, INV>(d, N, M, lm, tw, tid, nthr);
            break;
    }
}

// Block length and log2 sub-block length of every forward stage.
template <class C>
__host__ __device__ __forceinline__ void fz_shape(const FzPlan<C>& p, int s, int& M, int& lm) {
    M = p.N;
    for (int k = 0; k < s; ++k) M /= p.rad[k];
    const int m = M / p.rad[s];
    lm = 0;
    while ((1 << lm) < m) ++lm;
}

#ifdef __CUDACC__
// Fills the per-stage twiddle tables of p (n entries): w_M^(p j) evaluated in FP64.
template <class C>
__global__ void k_fz_fill_tables(C* out, FzPlan<C> p, uint32_t n) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    int M, pp, j;
    fz_table_entry(p, e, M, pp, j);
    double sn, cs;
    sincospi(-2.0 * static_cast<double>(pp) * static_cast<double>(j) / static_cast<double>(M), &sn, &cs);
    out[e] = from_d2<C>(make_double2(cs, sn));
}

template <class C>
__device__ __forceinline__ void fz_forward(C* d, const FzPlan<C>& p) {
    for (int s = 0; s < p.nst; ++s) {
        int M, lm;
        fz_shape(p, s, M, lm);
        fz_stage_any<C, false>(d, p.N, M, p.rad[s], lm, p.tw + p.twoff[s], threadIdx.x, blockDim.x);
        __syncthreads();
    }
}

template <class C>
__device__ __forceinline__ void fz_inverse(C* d, const FzPlan<C>& p) {
    for (int s = p.nst - 1; s >= 0; --s) {
        int M, lm;
        fz_shape(p, s, M, lm);
        fz_stage_any<C, true>(d, p.N, M, p.rad[s], lm, p.tw + p.twoff[s], threadIdx.x, blockDim.x);
        __syncthreads();
    }
}

// Spectra of the partner series: x = gamma_b - gamma_b[n_in-1] (conjugated for half 1),
// zero beyond n_in, forward transform, stored in the digit-reversed order.
template <class R>
__global__ void __launch_bounds__(FZ_THREADS, 1) k_fz_spectrum(const ColJob* __restrict__ jobs, FzPlan<cplx_t<R>> p) {
    using C = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* d = reinterpret_cast<C*>(smem_raw);
    const ColJob job = jobs[blockIdx.x];
    const double2 shift = __ldg(&job.g[job.n_in - 1]);
    for (int t = threadIdx.x; t < p.N; t += blockDim.x) {
        double2 x = make_double2(0.0, 0.0);
        if (static_cast<uint32_t>(t) < job.n_in) {
            x = csub(__ldg(&job.g[t]), shift);
            if (job.conj) x.y = -x.y;
        }
        d[pad_idx<C>(t)] = from_d2<C>(x);
    }
    __syncthreads();
    fz_forward(d, p);
    C* out = static_cast<C*>(job.out);
    for (int i = threadIdx.x; i < p.N; i += blockDim.x) out[i] = d[pad_idx<C>(i)];
}

// The fused convolution, scans and assembly of one (triple, half): blockIdx.x = 2 triple + half.
template <class R>
__global__ void __launch_bounds__(FZ_THREADS, 1) k_fz_conv_scan(const ScanJob* __restrict__ jobs, FzPlan<cplx_t<R>> p) {
    using C = cplx_t<R>;
    constexpr int NW = FZ_THREADS / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* d = reinterpret_cast<C*>(smem_raw);
    double* warp_tot = reinterpret_cast<double*>(smem_raw + fz_scratch_off<C>(p.N));
    double* carry = warp_tot + 2 * NW * 8;  // [2][8]
    double2* steps = reinterpret_cast<double2*>(carry + 2 * 8);
    const ScanJob job = jobs[blockIdx.x >> 1];
    const int half = blockIdx.x & 1;  // 0: F (and R), 1: C
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double dt = job.dt;
    // 1. x[t] = (g_i[t] - c_i) e^{-i w t dt}; phases by recurrence over the thread's samples
    const double2 ci = __ldg(&job.gi[job.n_in - 1]);
    {
        // eight samples per thread per round: their loads are issued before any is used
        const double2 step = phase_minus(job.omega, dt, blockDim.x);
        double2 ph = phase_minus(job.omega, dt, threadIdx.x);
        for (int t0 = threadIdx.x; t0 < p.N; t0 += 8 * blockDim.x) {
            double2 g[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int t = t0 + k * static_cast<int>(blockDim.x);
                g[k] = static_cast<uint32_t>(t) < job.n_in ? __ldg(&job.gi[t]) : ci;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int t = t0 + k * static_cast<int>(blockDim.x);
                if (t < p.N) d[pad_idx<C>(t)] = from_d2<C>(cmul(csub(g[k], ci), ph));  // zero beyond n_in
                ph = cmul(ph, step);
            }
        }
    }
    __syncthreads();
    // 2.-4. forward transform, partner spectrum, inverse transform
    fz_forward(d, p);
    {
        const C* spec = static_cast<const C*>(half ? job.spec_c : job.spec_f);
        const R scale = static_cast<R>(dt / static_cast<double>(p.N));
        for (int i0 = threadIdx.x; i0 < p.N; i0 += 8 * blockDim.x) {
            C sv[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int i = i0 + k * static_cast<int>(blockDim.x);
                sv[k] = i < p.N ? __ldg(&spec[i]) : C{0, 0};
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int i = i0 + k * static_cast<int>(blockDim.x);
                if (i < p.N) {
                    const int q = pad_idx<C>(i);
                    d[q] = cscale(cmul(d[q], sv[k]), scale);
                }
            }
        }
    }
    __syncthreads();
    fz_inverse(d, p);
    // 5. prefix integrals (FP64) and assembly at the requested times.  Components:
    //    half 0: P_F <- g_mj e^{+iwt}, P_R1 <- g_j e^{-iwt}, P_R2 <- g_i g_j e^{-iwt},
    //            S <- (g_i - c_i) e^{-iwt};  half 1: P_R1, S.
    const double2 cmj = __ldg(&job.gmj[job.n_in - 1]);
    const double2 cj = __ldg(&job.gj[job.n_in - 1]);
    const uint32_t tile = FZ_THREADS * FZ_ITEMS;
    if (threadIdx.x < 8) carry[threadIdx.x] = 0.0;
    if (threadIdx.x == 0) steps[0] = phase_minus(job.omega, dt, 1);
    if (threadIdx.x == 32) steps[1] = phase_minus(job.omega, dt, tile);
    double2 pm_next = phase_minus(job.omega, dt, threadIdx.x * FZ_ITEMS);
    __syncthreads();
    const double2 step = steps[0], tile_step = steps[1];
    C* vf = static_cast<C*>(job.vf);
    C* vc = static_cast<C*>(job.vc);
    C* vr = static_cast<C*>(job.vr);
    constexpr int K = 8;
    for (uint32_t t0 = 0, par = 0; t0 < job.t_count; t0 += tile, par ^= 1u) {
        const uint32_t tb = t0 + threadIdx.x * FZ_ITEMS;
        double run[K];
#pragma unroll
        for (int k = 0; k < K; ++k) run[k] = 0.0;
        const double2 pm0 = pm_next;
        pm_next = cmul(pm_next, tile_step);
        double2 gi_s[FZ_ITEMS], gj_s[FZ_ITEMS], gmj_s[FZ_ITEMS];
        {
            double2 pm = pm0;
#pragma unroll
            for (int q = 0; q < FZ_ITEMS; ++q, pm = cmul(pm, step)) {
                const uint32_t t = tb + q;
                gi_s[q] = gj_s[q] = gmj_s[q] = make_double2(0.0, 0.0);
                if (t < job.t_count) {
                    gi_s[q] = __ldg(&job.gi[t]);
                    gj_s[q] = __ldg(&job.gj[t]);
                    const double2 b = cmul(gj_s[q], pm);
                    const double2 dd = cmul(csub(gi_s[q], ci), pm);
                    run[2] += b.x;
                    run[3] += b.y;
                    run[6] += dd.x;
                    run[7] += dd.y;
                    if (half == 0) {
                        gmj_s[q] = __ldg(&job.gmj[t]);
                        const double2 a = cmulc(gmj_s[q], pm);
                        const double2 c = cmul(cmul(gi_s[q], gj_s[q]), pm);
                        run[0] += a.x;
                        run[1] += a.y;
                        run[4] += c.x;
                        run[5] += c.y;
                    }
                }
            }
        }
        // block-exclusive prefix of the per-thread sums (warp scans, warp totals by parity)
        double pre[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double x = run[k];
            if (half == 1 && (k == 0 || k == 1 || k == 4 || k == 5)) {
                pre[k] = 0.0;
                continue;
            }
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double nb = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += nb;
            }
            if (lane == 31) warp_tot[(par * NW + warp) * K + k] = x;
            const double excl = __shfl_up_sync(0xffffffffu, x, 1);
            pre[k] = lane == 0 ? 0.0 : excl;
        }
        __syncthreads();
        {
            double wk = 0.0;
            if (lane < K) {
                wk = carry[par * 8 + lane];
                for (int q = 0; q < warp; ++q) wk += warp_tot[(par * NW + q) * K + lane];
                if (warp == NW - 1) carry[(par ^ 1u) * 8 + lane] = wk + warp_tot[(par * NW + warp) * K + lane];
            }
#pragma unroll
            for (int k = 0; k < K; ++k) pre[k] += __shfl_sync(0xffffffffu, wk, k);
        }
        double2 pm = pm0;
#pragma unroll
        for (int q = 0; q < FZ_ITEMS; ++q, pm = cmul(pm, step)) {
            const uint32_t t = tb + q;
            if (t >= job.t_count) break;
            const double2 gi = gi_s[q], gj = gj_s[q];
            const double2 b = cmul(gj, pm);
            const double2 dd = cmul(csub(gi, ci), pm);
            pre[2] += b.x;
            pre[3] += b.y;
            pre[6] += dd.x;
            pre[7] += dd.y;
            if (half == 0) {
                const double2 a = cmulc(gmj_s[q], pm);
                const double2 c = cmul(cmul(gi, gj), pm);
                pre[0] += a.x;
                pre[1] += a.y;
                pre[4] += c.x;
                pre[5] += c.y;
            }
            const int u = __ldg(&job.tmap[t]);
            if (u < 0) continue;
            const double2 PR1 = make_double2(pre[2] * dt, pre[3] * dt);
            const double2 S = make_double2(pre[6] * dt, pre[7] * dt);
            const double2 conv = to_d2(d[pad_idx<C>(static_cast<int>(t))]);
            if (half == 0) {
                const double2 PF = make_double2(pre[0] * dt, pre[1] * dt);
                const double2 PR2 = make_double2(pre[4] * dt, pre[5] * dt);
                vf[u] = from_d2<C>(csub(cmul(dd, PF), cadd(conv, cmul(cmj, S))));
                vr[u] = from_d2<C>(csub(cmul(gi, PR1), PR2));
            } else {
                vc[u] = from_d2<C>(csub(cmulc(dd, PR1), cadd(conv, cmulc(S, cj))));
            }
        }
    }
}
#endif

}  // namespace taco
