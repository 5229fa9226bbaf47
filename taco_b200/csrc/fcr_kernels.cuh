// fcr_kernels.cuh -- device kernels of the F/C/R stage.
//
// F and C (cpp/src/tcl/tcl4_kernels.cpp:105-152) are
//   F[t] = g1[t] e_t P_F(t) - dt sum_{m<=t} g1[t-m] e_{t-m} g2[m],   e_t = exp(-i w t dt),
// a prefix integral minus a causal convolution that nearly cancel (term ratios above
// 100 occur).  The kernels evaluate the algebraically identical form with both series
// shifted by their last sample (c1 = g1[n_in-1], c2 = g2[n_in-1], d = g - c):
//   F[t] = d1[t] e_t P_F(t) - dt sum_m d1[t-m] e_{t-m} d2[m] - c2 S(t),
//   S(t) = dt sum_{k<=t} d1[k] e_k,
// which leaves only the transient in the FFT operands: the FFT round-off, proportional
// to the operand norms, drops by about three orders of magnitude (what makes the FP32
// form meet 1e-6), and the FP64 path gains accuracy as well.
//
// The convolutions use a four-step FFT of length Nfft = N1*N2 (powers of two <= 2048):
//   B1  column pass: x[t] generated on the fly (gamma column minus its last sample,
//       optional conjugate, optional phase exp(-i w t dt); zero for t >= n_in),
//       N1-point FFTs down the columns, inter-step twiddle w_N^(n2*k1), stored as
//       Z[k1*N2 + n2];
//   B2  row pass: N2-point FFT of each row -> spectrum row in the permuted order
//       S[k1*N2 + k2]; multiplied by the hoisted spectra of the two partner series
//       (F: d of gamma[:, mirror j]; C: conj d of gamma[:, j]), both products transformed
//       back along the row and twiddled by w_N^(-n2*k1) (the spectrum of x never leaves
//       shared memory);
//   B3  inverse column pass: N1-point inverse FFTs down the columns, scaled by dt/Nfft,
//       only samples t <= t_max written.
// The spectra of d_b and conj(d_b) are produced once per instance by B1 + a plain
// forward row pass.  The scan kernel forms the prefix integrals per triple (P_F, P_R1,
// P_R2, S; P_C = conj(P_R1)) with FP64 carries and assembles F, C, R at the requested
// times.
#pragma once

#include <algorithm>
#include <cstddef>

#include "common.cuh"
#include "fft.cuh"

namespace taco {

template <class C>
struct FftPlan {
    int L, L1, L2, s;  // Nfft = R*2^L = N1*N2, N1 = R*2^L1 (column length), N2 = 2^L2 (row length)
    int R;             // odd factor of the length: 1, 3 or 5
    const C* tw1;      // exp(-2 pi i m / N1), m < N1
    const C* tw2;      // exp(-2 pi i m / N2), m < N2
    const C* twc;      // exp(-2 pi i m 2^s / N), m < N / 2^s
    const C* twf;      // exp(-2 pi i m / N), m < 2^s
};

// Launch geometry of the four-step passes (host side).
struct Geometry {
    int log2c, col_threads, log2r, row_threads;
    std::size_t col_smem, row_smem;
    unsigned col_grid, row_grid;
};

// Tile shapes: column tiles of col_tile elements (N1 rows x 2^log2c columns), row tiles
// of row_tile elements (2^log2r rows of N2), both padded in shared memory.
template <class C>
Geometry geometry(const FftPlan<C>& p, int col_tile, int row_tile) {
    Geometry g;
    const int N1 = p.R << p.L1, N2 = 1 << p.L2;
    auto floor_log2 = [](int x) {
        int l = 0;
        while ((2 << l) <= x) ++l;
        return l;
    };
    const int cc = std::max(1, std::min(N2, col_tile / N1));
    g.log2c = floor_log2(cc);
    g.col_threads = (N1 << g.log2c) / 8;
    g.col_smem = static_cast<std::size_t>(padded_size<C>(N1 << g.log2c)) * sizeof(C);
    g.col_grid = static_cast<unsigned>(N2 >> g.log2c);
    const int rr = std::max(1, std::min(1 << p.L1, row_tile / N2));  // rows of a tile divide N1
    g.log2r = floor_log2(rr);
    g.row_threads = (N2 << g.log2r) / 8;
    g.row_smem = 2 * static_cast<std::size_t>(padded_size<C>(N2 << g.log2r)) * sizeof(C);
    g.row_grid = static_cast<unsigned>(N1 >> g.log2r);
    constexpr std::size_t kSmemMax = 227 * 1024;
    while (g.row_smem > kSmemMax && g.log2r > 0) {  // explicit schedules too large for one CTA
        --g.log2r;
        g.row_threads = (N2 << g.log2r) / 8;
        g.row_smem = 2 * static_cast<std::size_t>(padded_size<C>(N2 << g.log2r)) * sizeof(C);
    }
    while (g.col_smem > kSmemMax && g.log2c > 0) {
        --g.log2c;
        g.col_threads = (N1 << g.log2c) / 8;
        g.col_smem = static_cast<std::size_t>(padded_size<C>(N1 << g.log2c)) * sizeof(C);
    }
    g.col_grid = static_cast<unsigned>(N2 >> g.log2c);
    g.row_grid = static_cast<unsigned>(N1 >> g.log2r);
    return g;
}

// w_N^a for 0 <= a < N as the product of a coarse and a fine table entry.
template <class C>
__device__ __forceinline__ C inter_twiddle(const FftPlan<C>& p, uint32_t a) {
    const uint32_t hi = a >> p.s, lo = a & ((1u << p.s) - 1u);
    return cmul(__ldg(&p.twc[hi]), __ldg(&p.twf[lo]));
}

struct ColJob {
    const double2* g;  // gamma column, n_in valid samples; g[n_in-1] is subtracted
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
    uint32_t n_in;     // samples used by the convolution operands (shift = g[n_in-1])
    uint32_t t_count;  // t_max + 1
    const void* conv_f;
    const void* conv_c;
    const int* tmap;   // [t_count] -> position in the output series, or -1
    void* vf;          // F series at the unique requested times [U]
    void* vc;
    void* vr;
    const void* spec_f;  // fused path: partner spectra in the fused transform's order
    const void* spec_c;
};

// Threads of a compile-time-size FFT tile (8 elements per thread).
constexpr int ct_threads(int kl, int kc) { return kl >= 0 ? (1 << (kl + kc)) / 8 : 1024; }

__device__ __forceinline__ double2 phase_minus(double omega, double dt, uint32_t t) {
    const double tk = static_cast<double>(t) * dt;  // t_k = k dt, then exp(-i omega t_k)
    double sn, cs;
    sincos(-(omega * tk), &sn, &cs);
    return make_double2(cs, sn);
}

// ---------------------------------------------------------------- B1 -------
// Column tile: 2^log2c columns n2_0 .. n2_0 + 2^log2c - 1, all N1 rows; element
// (column c, row n1) at pad(n1 * 2^log2c + c).
// KL, KC >= 0: N1 = 2^KL and the tile width 2^KC fixed at compile time (-1: runtime).
template <class R, int KL, int KC, int RADIX = 1>
__device__ __forceinline__ void fwd_col_body(const ColJob* __restrict__ jobs, const FftPlan<cplx_t<R>>& plan, int log2c_rt) {
    using C = cplx_t<R>;
    constexpr bool CT = KL >= 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    const ColJob job = jobs[blockIdx.y];
    const int L1 = CT ? KL : plan.L1;
    const int log2c = CT ? KC : log2c_rt;
    const int nthr = CT ? ((RADIX << (KL + KC)) / 8) : static_cast<int>(blockDim.x);
    const int N2 = 1 << plan.L2;
    const int ccols = 1 << log2c;
    const int n2_0 = blockIdx.x << log2c;
    const double2 shift = __ldg(&job.g[job.n_in - 1]);
    // (N1 << log2c) == 8 * threads: issue the 8 loads of a thread before using any of them
    double2 v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int idx = threadIdx.x + q * nthr;
        const int n1 = idx >> log2c, c = idx & (ccols - 1);
        const uint32_t t = static_cast<uint32_t>(n1) * N2 + n2_0 + c;
        v[q] = t < job.n_in ? __ldg(&job.g[t]) : shift;
    }
    // when the tile is at most nthr columns wide, a thread's 8 samples are equally spaced
    // in t (stride nthr / ccols rows): phases by recurrence from the first
    const bool spaced = nthr >= ccols;
    const uint32_t t_first = static_cast<uint32_t>(threadIdx.x >> log2c) * N2 + n2_0 + (threadIdx.x & (ccols - 1));
    const uint32_t t_step = static_cast<uint32_t>(nthr >> log2c) * N2;
    double2 ph = make_double2(1.0, 0.0), ph_step = ph;
    if (job.has_phase && spaced) {
        ph = phase_minus(job.omega, job.dt, t_first);
        ph_step = phase_minus(job.omega, job.dt, t_step);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int idx = threadIdx.x + q * nthr;
        double2 x = csub(v[q], shift);  // zero beyond n_in
        if (job.conj) x.y = -x.y;
        if (job.has_phase) {
            if (spaced) {
                x = cmul(x, ph);
                ph = cmul(ph, ph_step);
            } else {
                const uint32_t t = static_cast<uint32_t>(idx >> log2c) * N2 + n2_0 + (idx & (ccols - 1));
                x = cmul(x, phase_minus(job.omega, job.dt, t));
            }
        }
        s[pad_idx<C>(idx)] = from_d2<C>(x);
    }
    __syncthreads();
    if constexpr (CT && RADIX > 1) tile_fft_mx<C, false, true, RADIX, KL, KC>(s, plan.tw1);
    else if constexpr (CT) tile_fft_ct<C, false, true, KL, KC>(s, plan.tw1);
    else tile_fft<C, false, true>(s, L1, log2c, 1, ccols, plan.tw1);
    C* out = static_cast<C*>(job.out);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int idx = threadIdx.x + q * nthr;
        const int k1 = idx >> log2c, c = idx & (ccols - 1);
        const uint32_t n2 = n2_0 + c;
        out[static_cast<size_t>(k1) * N2 + n2] =
            cmul(s[pad_idx<C>(idx)], inter_twiddle(plan, n2 * static_cast<uint32_t>(k1)));
    }
}

// ---------------------------------------------------------------- B2 -------
// Row tile: 2^log2r rows of N2 elements, element (row r, i) at pad(r * N2 + i).
// Forward row FFT; with spec_f set: two spectral products, inverse row FFTs and the
// inverse inter-step twiddle.  Shared memory: two padded tiles.
// KL, KC >= 0: N2 = 2^KL and 2^KC rows per tile fixed at compile time (-1: runtime).
template <class R, int KL, int KC>
__device__ __forceinline__ void row_body(const RowJob* __restrict__ jobs, const FftPlan<cplx_t<R>>& plan, int log2r_rt) {
    using C = cplx_t<R>;
    constexpr bool CT = KL >= 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L2 = CT ? KL : plan.L2;
    const int log2r = CT ? KC : log2r_rt;
    const int nthr = CT ? ((1 << (KL + KC)) / 8) : static_cast<int>(blockDim.x);
    const int N2 = 1 << L2;
    const int elems = N2 << log2r;
    C* a = reinterpret_cast<C*>(smem_raw);
    C* p = a + padded_size<C>(elems);
    const RowJob job = jobs[blockIdx.y];
    const size_t off = static_cast<size_t>(blockIdx.x) * elems;
    C* data = static_cast<C*>(job.data) + off;
    // elems == 8 * threads: 8 loads per thread in flight at once
    C x[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) x[q] = data[threadIdx.x + q * nthr];
    const bool conv = job.spec_f != nullptr;
    // the partner spectra arrive while the forward transform runs
    C sf[8], sc[8];
    if (conv) {
        const C* spf = static_cast<const C*>(job.spec_f) + off;
        const C* spc = static_cast<const C*>(job.spec_c) + off;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            sf[q] = __ldg(&spf[threadIdx.x + q * nthr]);
            sc[q] = __ldg(&spc[threadIdx.x + q * nthr]);
        }
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) a[pad_idx<C>(threadIdx.x + q * nthr)] = x[q];
    __syncthreads();
    if constexpr (CT) tile_fft_ct<C, false, false, KL, KC>(a, plan.tw2);
    else tile_fft<C, false, false>(a, L2, log2r, N2, 1, plan.tw2);
    if (!conv) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = threadIdx.x + q * nthr;
            data[idx] = a[pad_idx<C>(idx)];
        }
        return;
    }
    const int k1_0 = blockIdx.x << log2r;
    for (int which = 0; which < 2; ++which) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = threadIdx.x + q * nthr;
            p[pad_idx<C>(idx)] = cmul(a[pad_idx<C>(idx)], which == 0 ? sf[q] : sc[q]);
        }
        __syncthreads();
        if constexpr (CT) tile_fft_ct<C, true, false, KL, KC>(p, plan.tw2);
        else tile_fft<C, true, false>(p, L2, log2r, N2, 1, plan.tw2);
        C* dst = (which == 0 ? data : static_cast<C*>(job.wc) + off);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int idx = threadIdx.x + q * nthr;
            const int r = idx >> L2, n2 = idx & (N2 - 1);
            const uint32_t k1 = static_cast<uint32_t>(k1_0 + r);
            dst[idx] = cmulc(p[pad_idx<C>(idx)], inter_twiddle(plan, static_cast<uint32_t>(n2) * k1));
        }
        __syncthreads();
    }
}

// ------------------------------------------------------ B2, one warp per row ----
// 256-point row transforms held in registers, 8 elements per lane, as 256 = 8 * 8 * 4:
//   x[l + 32 r] (lane l, r < 8) --DFT8 over r--> k1; twiddle w256^(l k1);
//   transpose 1: lane (q, a) = (lane / 4, lane % 4) takes z_b = y_{a + 4 b}[q], b < 8;
//   --DFT8 over b--> c; twiddle w256^(8 a c) (= w32^(a c));
//   transpose 2: lane takes the pairs P = 2 lane + h (h < 2), each with its 4 values of a;
//   --DFT4 over a--> d:  element 4 h + d holds X[k] with k = P / 8 + 8 (P % 8) + 64 d.
// The inverse runs the same steps backwards with conjugate twiddles (unnormalised), so
// a forward transform, an elementwise product in that register order and an inverse
// give the cyclic convolution in natural order.  Both transposes go through a
// warp-private shared buffer with padding that keeps every access conflict-free
// (rows of 36 for the first, P * 4 + a + P / 2 for the second); the warp never waits
// on other warps.
constexpr int WROW_WARPS = 4;
constexpr int WROW_THREADS = 32 * WROW_WARPS;
constexpr int WROW_BUF = 288;

__device__ __forceinline__ int wrow_k(int lane, int j) {
    const int P = 2 * lane + (j >> 2), d = j & 3;
    return (P >> 3) + 8 * (P & 7) + 64 * d;
}

template <class C, bool INV>
__device__ __forceinline__ void warp_fft256(C (&x)[8], C* buf, const C* __restrict__ tw, int lane) {
    const int q = lane >> 2, a = lane & 3;
    if (!INV) {
        dft8<C, false>(x);
#pragma unroll
        for (int k = 1; k < 8; ++k) x[k] = cmul(x[k], __ldg(&tw[(lane * k) & 255]));
#pragma unroll
        for (int k = 0; k < 8; ++k) buf[k * 36 + lane] = x[k];
        __syncwarp();
#pragma unroll
        for (int b = 0; b < 8; ++b) x[b] = buf[q * 36 + a + 4 * b];
        __syncwarp();
        dft8<C, false>(x);
#pragma unroll
        for (int c = 1; c < 8; ++c) x[c] = cmul(x[c], __ldg(&tw[(8 * a * c) & 255]));
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int P = q * 8 + c;
            buf[P * 4 + a + (P >> 1)] = x[c];
        }
        __syncwarp();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int P = 2 * lane + h;
#pragma unroll
            for (int e = 0; e < 4; ++e) x[4 * h + e] = buf[P * 4 + e + (P >> 1)];
        }
        __syncwarp();
        dft4<C, false>(x[0], x[1], x[2], x[3]);
        dft4<C, false>(x[4], x[5], x[6], x[7]);
    } else {
        dft4<C, true>(x[0], x[1], x[2], x[3]);
        dft4<C, true>(x[4], x[5], x[6], x[7]);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int P = 2 * lane + h;
#pragma unroll
            for (int e = 0; e < 4; ++e) buf[P * 4 + e + (P >> 1)] = x[4 * h + e];
        }
        __syncwarp();
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int P = q * 8 + c;
            x[c] = buf[P * 4 + a + (P >> 1)];
        }
        __syncwarp();
#pragma unroll
        for (int c = 1; c < 8; ++c) x[c] = cmulc(x[c], __ldg(&tw[(8 * a * c) & 255]));
        dft8<C, true>(x);
#pragma unroll
        for (int b = 0; b < 8; ++b) buf[q * 36 + a + 4 * b] = x[b];
        __syncwarp();
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = buf[k * 36 + lane];
        __syncwarp();
#pragma unroll
        for (int k = 1; k < 8; ++k) x[k] = cmulc(x[k], __ldg(&tw[(lane * k) & 255]));
        dft8<C, true>(x);
    }
}

// B2 for N2 = 256: one warp per row (row k1 of the job's N1 rows).  Spectra jobs
// (spec_f == nullptr) write the forward row transform; triple jobs multiply it by both
// partner spectra (loaded while the forward transform runs), invert each product, apply
// the inverse inter-step twiddle and write W_F (in place) and W_C.
template <class R>
__global__ void __launch_bounds__(WROW_THREADS) k_row_warp256(const RowJob* __restrict__ jobs, FftPlan<cplx_t<R>> plan,
                                                               int n_rows) {
    using C = cplx_t<R>;
    __shared__ C bufs[WROW_WARPS][WROW_BUF];
    const RowJob job = jobs[blockIdx.y];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int row = blockIdx.x * WROW_WARPS + warp;
    if (row >= n_rows) return;
    const size_t off = static_cast<size_t>(row) * 256;
    C* data = static_cast<C*>(job.data) + off;
    C* buf = bufs[warp];
    C x[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) x[r] = data[lane + 32 * r];
    const bool conv = job.spec_f != nullptr;
    C sf[8], sc[8];
    if (conv) {
        const C* spf = static_cast<const C*>(job.spec_f) + off;
        const C* spc = static_cast<const C*>(job.spec_c) + off;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            sf[j] = __ldg(&spf[wrow_k(lane, j)]);
            sc[j] = __ldg(&spc[wrow_k(lane, j)]);
        }
    }
    warp_fft256<C, false>(x, buf, plan.tw2, lane);
    if (!conv) {
#pragma unroll
        for (int j = 0; j < 8; ++j) data[wrow_k(lane, j)] = x[j];
        return;
    }
#pragma unroll
    for (int which = 0; which < 2; ++which) {
        C y[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) y[j] = cmul(x[j], which == 0 ? sf[j] : sc[j]);
        warp_fft256<C, true>(y, buf, plan.tw2, lane);
        C* dst = which == 0 ? data : static_cast<C*>(job.wc) + off;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const uint32_t n2 = static_cast<uint32_t>(lane + 32 * r);
            dst[n2] = cmulc(y[r], inter_twiddle(plan, n2 * static_cast<uint32_t>(row)));
        }
    }
}

// ---------------------------------------------------------------- B3 -------
template <class R, int KL, int KC, int RADIX = 1>
__device__ __forceinline__ void inv_col_body(const InvJob* __restrict__ jobs, const FftPlan<cplx_t<R>>& plan, int log2c_rt) {
    using C = cplx_t<R>;
    constexpr bool CT = KL >= 0;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    const InvJob job = jobs[blockIdx.y];
    const int L1 = CT ? KL : plan.L1;
    const int log2c = CT ? KC : log2c_rt;
    const int nthr = CT ? ((RADIX << (KL + KC)) / 8) : static_cast<int>(blockDim.x);
    const int N2 = 1 << plan.L2;
    const int ccols = 1 << log2c;
    const int n2_0 = blockIdx.x << log2c;
    const C* w = static_cast<const C*>(job.w);
    C x[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int idx = threadIdx.x + q * nthr;
        const int k1 = idx >> log2c, c = idx & (ccols - 1);
        x[q] = w[static_cast<size_t>(k1) * N2 + n2_0 + c];
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) s[pad_idx<C>(threadIdx.x + q * nthr)] = x[q];
    __syncthreads();
    if constexpr (CT && RADIX > 1) tile_fft_mx<C, true, true, RADIX, KL, KC>(s, plan.tw1);
    else if constexpr (CT) tile_fft_ct<C, true, true, KL, KC>(s, plan.tw1);
    else tile_fft<C, true, true>(s, L1, log2c, 1, ccols, plan.tw1);
    C* out = static_cast<C*>(job.out);
    const R scale = static_cast<R>(job.scale);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int idx = threadIdx.x + q * nthr;
        const int n1 = idx >> log2c, c = idx & (ccols - 1);
        const uint32_t t = static_cast<uint32_t>(n1) * N2 + n2_0 + c;
        if (t < job.t_count) out[t] = cscale(s[pad_idx<C>(idx)], scale);
    }
}

// Kernels: runtime sizes (k_fwd_col, k_row, k_inv_col) and compile-time sizes (the _ct
// variants, bounded to two CTAs per SM).
template <class R>
__global__ void k_fwd_col(const ColJob* __restrict__ jobs, FftPlan<cplx_t<R>> plan, int log2c) {
    fwd_col_body<R, -1, -1>(jobs, plan, log2c);
}
template <class R>
__global__ void k_row(const RowJob* __restrict__ jobs, FftPlan<cplx_t<R>> plan, int log2r) {
    row_body<R, -1, -1>(jobs, plan, log2r);
}
template <class R>
__global__ void k_inv_col(const InvJob* __restrict__ jobs, FftPlan<cplx_t<R>> plan, int log2c) {
    inv_col_body<R, -1, -1>(jobs, plan, log2c);
}
template <class R, int KL, int KC>
__global__ void __launch_bounds__(ct_threads(KL, KC), ct_threads(KL, KC) > 256 ? 1 : 3) k_fwd_col_ct(const ColJob* __restrict__ jobs,
                                                                       FftPlan<cplx_t<R>> plan, int log2c) {
    fwd_col_body<R, KL, KC>(jobs, plan, log2c);
}
// Column passes of the mixed lengths N1 = RADIX * 2^KL (RADIX 3 or 5).
template <class R, int RADIX, int KL, int KC>
__global__ void __launch_bounds__((RADIX << (KL + KC)) / 8) k_fwd_col_mx(const ColJob* __restrict__ jobs,
                                                                         FftPlan<cplx_t<R>> plan, int log2c) {
    fwd_col_body<R, KL, KC, RADIX>(jobs, plan, log2c);
}
template <class R, int RADIX, int KL, int KC>
__global__ void __launch_bounds__((RADIX << (KL + KC)) / 8) k_inv_col_mx(const InvJob* __restrict__ jobs,
                                                                         FftPlan<cplx_t<R>> plan, int log2c) {
    inv_col_body<R, KL, KC, RADIX>(jobs, plan, log2c);
}
template <class R, int KL, int KC>
__global__ void __launch_bounds__(ct_threads(KL, KC), ct_threads(KL, KC) > 256 ? 1 : 2) k_row_ct(const RowJob* __restrict__ jobs,
                                                                   FftPlan<cplx_t<R>> plan, int log2r) {
    row_body<R, KL, KC>(jobs, plan, log2r);
}
template <class R, int KL, int KC>
__global__ void __launch_bounds__(ct_threads(KL, KC), ct_threads(KL, KC) > 256 ? 1 : 3) k_inv_col_ct(const InvJob* __restrict__ jobs,
                                                                       FftPlan<cplx_t<R>> plan, int log2c) {
    inv_col_body<R, KL, KC>(jobs, plan, log2c);
}

// Pruned inverse column pass for t_count <= MAXR * N2: only rows n1 < nrows of the
// output are needed, so each thread owns one column and evaluates those rows as a
// direct inverse DFT over k1 (one streaming read of W, no shared-memory stages).
constexpr int INV_DFT_MAXR = 16;
constexpr int INV_DFT_THREADS = 128;

template <class R>
__global__ void __launch_bounds__(INV_DFT_THREADS) k_inv_col_dft(const InvJob* __restrict__ jobs,
                                                                  FftPlan<cplx_t<R>> plan, int nrows) {
    using C = cplx_t<R>;
    const InvJob job = jobs[blockIdx.y];
    const int N1 = plan.R << plan.L1, N2 = 1 << plan.L2;
    const int n2 = blockIdx.x * INV_DFT_THREADS + threadIdx.x;
    if (n2 >= N2) return;
    const C* w = static_cast<const C*>(job.w) + n2;
    C acc[INV_DFT_MAXR];
    int e[INV_DFT_MAXR];  // (r * k1) mod N1, advanced by r per k1
#pragma unroll
    for (int r = 0; r < INV_DFT_MAXR; ++r) {
        acc[r] = C{0, 0};
        e[r] = 0;
    }
#pragma unroll 4
    for (int k1 = 0; k1 < N1; ++k1) {
        const C x = w[static_cast<size_t>(k1) * N2];
#pragma unroll
        for (int r = 0; r < INV_DFT_MAXR; ++r) {
            if (r < nrows) acc[r] = cadd(acc[r], cmulc(x, __ldg(&plan.tw1[e[r]])));
            e[r] += r;
            if (e[r] >= N1) e[r] -= N1;
        }
    }
    C* out = static_cast<C*>(job.out);
    const R scale = static_cast<R>(job.scale);
#pragma unroll
    for (int r = 0; r < INV_DFT_MAXR; ++r) {
        const uint32_t t = static_cast<uint32_t>(r) * N2 + n2;
        if (r < nrows && t < job.t_count) out[t] = cscale(acc[r], scale);
    }
}

// ---------------------------------------------------------------- scans ----
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_W = 8;  // four complex prefix sums

// The four integrands at sample t (times dt later):
// P_F <- g_mj e^{+iwt}, P_R1 <- g_j e^{-iwt}, P_R2 <- g_i g_j e^{-iwt}, S <- (g_i - c_i) e^{-iwt}.
__device__ __forceinline__ void scan_integrands(const ScanJob& job, uint32_t t, double2 ci, double2 pm,
                                                double2 gi, double* v) {
    const double2 gmj = __ldg(&job.gmj[t]);
    const double2 gj = __ldg(&job.gj[t]);
    const double2 a = cmulc(gmj, pm);
    const double2 b = cmul(gj, pm);
    const double2 c = cmul(cmul(gi, gj), pm);
    const double2 d = cmul(csub(gi, ci), pm);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    v[4] = c.x; v[5] = c.y; v[6] = d.x; v[7] = d.y;
}

// One CTA per triple, ITEMS consecutive samples per thread, FP64 sums and carries.
// Pass 1 of a tile sums each thread's samples; after the block scan, pass 2 recomputes
// the integrands (cheaper than keeping them live: it doubles the occupancy) and
// assembles F, C, R at the requested times.
template <class R, int ITEMS, int MIN_BLOCKS>
__global__ void __launch_bounds__(SCAN_THREADS, MIN_BLOCKS) k_scan_assemble(const ScanJob* __restrict__ jobs) {
    using C = cplx_t<R>;
    // warp totals and carries double-buffered by tile parity: one block barrier per tile
    __shared__ double warp_tot[2][SCAN_THREADS / 32][SCAN_W];
    __shared__ double carry[2][SCAN_W];
    const ScanJob job = jobs[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < SCAN_W) carry[0][threadIdx.x] = 0.0;
    const C* cf = static_cast<const C*>(job.conv_f);
    const C* cc = static_cast<const C*>(job.conv_c);
    C* vf = static_cast<C*>(job.vf);
    C* vc = static_cast<C*>(job.vc);
    C* vr = static_cast<C*>(job.vr);
    const double2 ci = __ldg(&job.gi[job.n_in - 1]);
    const double2 cmj = __ldg(&job.gmj[job.n_in - 1]);
    const double2 cj = __ldg(&job.gj[job.n_in - 1]);
    const double dt = job.dt;
    // e^{-i w dt} and e^{-i w tile dt}: phases by recurrence over a thread's samples and
    // from one tile to the next (computed once per CTA)
    __shared__ double2 steps[2];
    const uint32_t tile = SCAN_THREADS * ITEMS;
    if (threadIdx.x == 0) steps[0] = phase_minus(job.omega, dt, 1);
    if (threadIdx.x == 32) steps[1] = phase_minus(job.omega, dt, tile);
    double2 pm_next = phase_minus(job.omega, dt, threadIdx.x * ITEMS);
    __syncthreads();
    const double2 step = steps[0], tile_step = steps[1];
    for (uint32_t t0 = 0, par = 0; t0 < job.t_count; t0 += tile, par ^= 1u) {
        const uint32_t tb = t0 + threadIdx.x * ITEMS;
        double run[SCAN_W];
#pragma unroll
        for (int k = 0; k < SCAN_W; ++k) run[k] = 0.0;
        const double2 pm0 = pm_next;
        pm_next = cmul(pm_next, tile_step);
        {
            double2 pm = pm0;
#pragma unroll
            for (int q = 0; q < ITEMS; ++q) {
                const uint32_t t = tb + q;
                if (t < job.t_count) {
                    double v[SCAN_W];
                    scan_integrands(job, t, ci, pm, __ldg(&job.gi[t]), v);
#pragma unroll
                    for (int k = 0; k < SCAN_W; ++k) run[k] += v[k];
                }
                pm = cmul(pm, step);
            }
        }
        // block-exclusive prefix of the per-thread sums
        double pre[SCAN_W];
#pragma unroll
        for (int k = 0; k < SCAN_W; ++k) {
            double x = run[k];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double nb = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += nb;
            }
            if (lane == 31) warp_tot[par][warp][k] = x;
            double excl = __shfl_up_sync(0xffffffffu, x, 1);
            pre[k] = lane == 0 ? 0.0 : excl;
        }
        __syncthreads();
        {
            // lane k < SCAN_W adds the carry and the preceding warps' totals of component k
            // (the last warp also leaves the next tile's carry in the other buffer)
            double wk = 0.0;
            if (lane < SCAN_W) {
                wk = carry[par][lane];
                for (int q = 0; q < warp; ++q) wk += warp_tot[par][q][lane];
                if (warp == SCAN_THREADS / 32 - 1) carry[par ^ 1u][lane] = wk + warp_tot[par][warp][lane];
            }
#pragma unroll
            for (int k = 0; k < SCAN_W; ++k) pre[k] += __shfl_sync(0xffffffffu, wk, k);
        }
        double2 pm = pm0;
#pragma unroll
        for (int q = 0; q < ITEMS; ++q, pm = cmul(pm, step)) {
            const uint32_t t = tb + q;
            if (t >= job.t_count) break;
            const double2 gi = __ldg(&job.gi[t]);
            double v[SCAN_W];
            scan_integrands(job, t, ci, pm, gi, v);
#pragma unroll
            for (int k = 0; k < SCAN_W; ++k) pre[k] += v[k];
            const int u = __ldg(&job.tmap[t]);
            if (u < 0) continue;
            const double2 PF = make_double2(pre[0] * dt, pre[1] * dt);
            const double2 PR1 = make_double2(pre[2] * dt, pre[3] * dt);
            const double2 PR2 = make_double2(pre[4] * dt, pre[5] * dt);
            const double2 S = make_double2(pre[6] * dt, pre[7] * dt);
            const double2 dip = cmul(csub(gi, ci), pm);
            const double2 convf = cadd(to_d2(cf[t]), cmul(cmj, S));
            const double2 convc = cadd(to_d2(cc[t]), cmulc(S, cj));  // conj(c_j) S
            vf[u] = from_d2<C>(csub(cmul(dip, PF), convf));
            vc[u] = from_d2<C>(csub(cmulc(dip, PR1), convc));  // P_C = conj(P_R1)
            vr[u] = from_d2<C>(csub(cmul(gi, PR1), PR2));
        }
    }
}

// ------------------------------------------------------- chunked scans ----
// Reduce-then-scan over chunks of SCAN_THREADS*SCAN_ITEMS samples, so that one triple's
// time axis spreads over many CTAs: k_scan_reduce writes the FP64 integrand sums of each
// chunk; k_scan_chunks adds the sums of the preceding chunks of its triple (its carry),
// rescans its chunk and assembles F, C, R.  No CTA waits on another.
constexpr int SCAN_CHUNK = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ void block_sum8(double* v, double (*warp_tot)[SCAN_W]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < SCAN_W; ++k) {
        double x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) warp_tot[warp][k] = x;
    }
    __syncthreads();
}

template <class R>  // R unused: a template keeps the header-defined kernel out of every TU's link
__global__ void __launch_bounds__(SCAN_THREADS, 2) k_scan_reduce(const ScanJob* __restrict__ jobs,
                                                                  double* __restrict__ partial, int max_chunks) {
    __shared__ double warp_tot[SCAN_THREADS / 32][SCAN_W];
    const ScanJob job = jobs[blockIdx.y];
    const uint32_t t0 = blockIdx.x * SCAN_CHUNK;
    if (t0 >= job.t_count) return;
    const double2 ci = __ldg(&job.gi[job.n_in - 1]);
    double run[SCAN_W];
#pragma unroll
    for (int k = 0; k < SCAN_W; ++k) run[k] = 0.0;
    const uint32_t tb = t0 + threadIdx.x * SCAN_ITEMS;
    const double2 step = phase_minus(job.omega, job.dt, 1);
    double2 pm = phase_minus(job.omega, job.dt, tb);
#pragma unroll
    for (int q = 0; q < SCAN_ITEMS; ++q, pm = cmul(pm, step)) {
        const uint32_t t = tb + q;
        if (t < job.t_count) {
            double v[SCAN_W];
            scan_integrands(job, t, ci, pm, __ldg(&job.gi[t]), v);
#pragma unroll
            for (int k = 0; k < SCAN_W; ++k) run[k] += v[k];
        }
    }
    block_sum8(run, warp_tot);
    if (threadIdx.x < SCAN_W) {
        double w = 0.0;
        for (int q = 0; q < SCAN_THREADS / 32; ++q) w += warp_tot[q][threadIdx.x];
        partial[(static_cast<size_t>(blockIdx.y) * max_chunks + blockIdx.x) * SCAN_W + threadIdx.x] = w;
    }
}

template <class R>
__global__ void __launch_bounds__(SCAN_THREADS, 2) k_scan_chunks(const ScanJob* __restrict__ jobs,
                                                                  const double* __restrict__ partial,
                                                                  int max_chunks) {
    using C = cplx_t<R>;
    __shared__ double warp_tot[SCAN_THREADS / 32][SCAN_W];
    __shared__ double carry[SCAN_W];
    const ScanJob job = jobs[blockIdx.y];
    const uint32_t t0 = blockIdx.x * SCAN_CHUNK;
    if (t0 >= job.t_count) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < SCAN_W) {
        double w = 0.0;
        const double* pp = partial + static_cast<size_t>(blockIdx.y) * max_chunks * SCAN_W + threadIdx.x;
        for (uint32_t c = 0; c < blockIdx.x; ++c) w += pp[c * SCAN_W];
        carry[threadIdx.x] = w;
    }
    const C* cf = static_cast<const C*>(job.conv_f);
    const C* cc = static_cast<const C*>(job.conv_c);
    C* vf = static_cast<C*>(job.vf);
    C* vc = static_cast<C*>(job.vc);
    C* vr = static_cast<C*>(job.vr);
    const double2 ci = __ldg(&job.gi[job.n_in - 1]);
    const double2 cmj = __ldg(&job.gmj[job.n_in - 1]);
    const double2 cj = __ldg(&job.gj[job.n_in - 1]);
    const double dt = job.dt;
    const uint32_t tb = t0 + threadIdx.x * SCAN_ITEMS;
    const double2 step = phase_minus(job.omega, dt, 1);  // e^{-i w dt}: phases by recurrence over a thread's samples
    const double2 pm0 = phase_minus(job.omega, dt, tb);
    double run[SCAN_W];
#pragma unroll
    for (int k = 0; k < SCAN_W; ++k) run[k] = 0.0;
    {
        double2 pm = pm0;
#pragma unroll
        for (int q = 0; q < SCAN_ITEMS; ++q, pm = cmul(pm, step)) {
            const uint32_t t = tb + q;
            if (t < job.t_count) {
                double v[SCAN_W];
                scan_integrands(job, t, ci, pm, __ldg(&job.gi[t]), v);
#pragma unroll
                for (int k = 0; k < SCAN_W; ++k) run[k] += v[k];
            }
        }
    }
    double pre[SCAN_W];
#pragma unroll
    for (int k = 0; k < SCAN_W; ++k) {
        double x = run[k];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double nb = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += nb;
        }
        if (lane == 31) warp_tot[warp][k] = x;
        const double excl = __shfl_up_sync(0xffffffffu, x, 1);
        pre[k] = lane == 0 ? 0.0 : excl;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < SCAN_W; ++k) {
        double w = 0.0;
        for (int q = 0; q < warp; ++q) w += warp_tot[q][k];
        pre[k] = carry[k] + (w + pre[k]);
    }
    double2 pm = pm0;
#pragma unroll
    for (int q = 0; q < SCAN_ITEMS; ++q, pm = cmul(pm, step)) {
        const uint32_t t = tb + q;
        if (t >= job.t_count) break;
        const double2 gi = __ldg(&job.gi[t]);
        double v[SCAN_W];
        scan_integrands(job, t, ci, pm, gi, v);
#pragma unroll
        for (int k = 0; k < SCAN_W; ++k) pre[k] += v[k];
        const int u = __ldg(&job.tmap[t]);
        if (u < 0) continue;
        const double2 PF = make_double2(pre[0] * dt, pre[1] * dt);
        const double2 PR1 = make_double2(pre[2] * dt, pre[3] * dt);
        const double2 PR2 = make_double2(pre[4] * dt, pre[5] * dt);
        const double2 S = make_double2(pre[6] * dt, pre[7] * dt);
        const double2 dip = cmul(csub(gi, ci), pm);
        const double2 convf = cadd(to_d2(cf[t]), cmul(cmj, S));
        const double2 convc = cadd(to_d2(cc[t]), cmulc(S, cj));
        vf[u] = from_d2<C>(csub(cmul(dip, PF), convf));
        vc[u] = from_d2<C>(csub(cmulc(dip, PR1), convc));
        vr[u] = from_d2<C>(csub(cmul(gi, PR1), PR2));
    }
}

}  // namespace taco
