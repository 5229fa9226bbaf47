// fft.cuh -- shared-memory Stockham FFT engine for power-of-two lengths.
//
// A tile in shared memory holds `nfft` independent transforms of length n.  Element i
// of transform f lives at pad(f*fs + i*es), where pad(x) = x + (x >> PAD) inserts one
// spare slot every 2^PAD elements (128 bytes) so that the strided Stockham writes of
// the first stages do not pile onto one bank.  Every thread owns 8 elements per stage
// (blockDim.x == nfft*n/8), so each radix-2^r stage reads 8 values into registers,
// twiddles them, runs 8/2^r small DFTs and writes them back (Stockham autosort: natural
// order in, natural order out; in place with a barrier between the read and the write
// phase).  F_FAST selects the thread -> (transform, element) mapping: transforms
// fastest for column tiles (fs == 1: consecutive threads touch consecutive addresses),
// elements fastest for row tiles (es == 1).  The twiddle table tw[m] =
// exp(-2*pi*i*m/n), m in [0, n), is read through the read-only path; inverse transforms
// conjugate it and are unnormalised.
#pragma once

#include "common.cuh"

namespace taco {

// one pad slot per 128 bytes: every 8 complex doubles or 16 complex floats
template <class C> struct PadShift;
template <> struct PadShift<double2> { static constexpr int value = 3; };
template <> struct PadShift<float2> { static constexpr int value = 4; };

template <class C>
__host__ __device__ __forceinline__ int pad_idx(int x) { return x + (x >> PadShift<C>::value); }

template <class C>
__host__ __device__ __forceinline__ int padded_size(int n) { return n + (n >> PadShift<C>::value) + 1; }

template <class C, bool INV>
__host__ __device__ __forceinline__ C mul_w(C a, C w) {
    return INV ? cmulc(a, w) : cmul(a, w);  // INV: a * conj(w)
}

// multiply by -i (forward) or +i (inverse)
template <class C, bool INV>
__host__ __device__ __forceinline__ C rot90(C a) {
    return INV ? C{-a.y, a.x} : C{a.y, -a.x};
}

template <class C, bool INV>
__host__ __device__ __forceinline__ void dft2(C& a, C& b) {
    const C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <class C, bool INV>
__host__ __device__ __forceinline__ void dft4(C& x0, C& x1, C& x2, C& x3) {
    const C a = cadd(x0, x2), b = csub(x0, x2);
    const C c = cadd(x1, x3), d = rot90<C, INV>(csub(x1, x3));
    x0 = cadd(a, c);
    x2 = csub(a, c);
    x1 = cadd(b, d);
    x3 = csub(b, d);
}

template <class C, bool INV>
__host__ __device__ __forceinline__ void dft8(C* x) {
    using R = decltype(x[0].x);
    const R h = static_cast<R>(0.70710678118654752440084436210484903928);
    C e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6];
    C o0 = x[1], o1 = x[3], o2 = x[5], o3 = x[7];
    dft4<C, INV>(e0, e1, e2, e3);
    dft4<C, INV>(o0, o1, o2, o3);
    // twiddles w8^k, k = 0..3 (w8 = exp(-+ 2 pi i / 8))
    const C t1 = INV ? C{h * (o1.x - o1.y), h * (o1.x + o1.y)} : C{h * (o1.x + o1.y), h * (o1.y - o1.x)};
    const C t2 = rot90<C, INV>(o2);
    const C t3 = INV ? C{-h * (o3.x + o3.y), h * (o3.x - o3.y)} : C{h * (o3.y - o3.x), -h * (o3.x + o3.y)};
    x[0] = cadd(e0, o0);
    x[4] = csub(e0, o0);
    x[1] = cadd(e1, t1);
    x[5] = csub(e1, t1);
    x[2] = cadd(e2, t2);
    x[6] = csub(e2, t2);
    x[3] = cadd(e3, t3);
    x[7] = csub(e3, t3);
}

// 3- and 5-point DFTs (radix factors of the mixed lengths 3*2^k and 5*2^k).
// y_k = sum_r x_r w^{r k}, w = exp(-+ 2 pi i / R); rot90 supplies the -+i.
template <class C, bool INV>
__host__ __device__ __forceinline__ void dft3(C& x0, C& x1, C& x2) {
    using R = decltype(x0.x);
    const R h = static_cast<R>(0.86602540378443864676);  // sin(2 pi / 3)
    const C t = cadd(x1, x2);
    const C m = C{x0.x - static_cast<R>(0.5) * t.x, x0.y - static_cast<R>(0.5) * t.y};
    const C d = rot90<C, INV>(cscale(csub(x1, x2), h));
    x0 = cadd(x0, t);
    x1 = cadd(m, d);
    x2 = csub(m, d);
}

template <class C, bool INV>
__host__ __device__ __forceinline__ void dft5(C* x) {
    using R = decltype(x[0].x);
    const R c1 = static_cast<R>(0.30901699437494742410);   // cos(2 pi / 5)
    const R c2 = static_cast<R>(-0.80901699437494742410);  // cos(4 pi / 5)
    const R s1 = static_cast<R>(0.95105651629515357212);   // sin(2 pi / 5)
    const R s2 = static_cast<R>(0.58778525229247312917);   // sin(4 pi / 5)
    const C t1 = cadd(x[1], x[4]), t2 = cadd(x[2], x[3]);
    const C t3 = csub(x[1], x[4]), t4 = csub(x[2], x[3]);
    const C a1 = C{x[0].x + c1 * t1.x + c2 * t2.x, x[0].y + c1 * t1.y + c2 * t2.y};
    const C a2 = C{x[0].x + c2 * t1.x + c1 * t2.x, x[0].y + c2 * t1.y + c1 * t2.y};
    const C b1 = rot90<C, INV>(C{s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y});
    const C b2 = rot90<C, INV>(C{s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y});
    x[0] = cadd(x[0], cadd(t1, t2));
    x[1] = cadd(a1, b1);
    x[4] = csub(a1, b1);
    x[2] = cadd(a2, b2);
    x[3] = csub(a2, b2);
}

// One Stockham stage of radix 2^LR on a shared-memory tile.
template <class C, int LR, bool INV, bool F_FAST>
__device__ __forceinline__ void stockham_stage(C* s, int log2n, int log2nfft, int p, int fs, int es,
                                               const C* __restrict__ tw) {
    constexpr int RAD = 1 << LR;
    constexpr int ITEMS = 8 / RAD;
    const int n = 1 << log2n;
    const int lq = log2n - LR;  // log2(n / RAD): items per transform
    C x[8];
    int base[ITEMS], jout[ITEMS];
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
        const int g = threadIdx.x * ITEMS + q;
        int f, i;
        if (F_FAST) {
            f = g & ((1 << log2nfft) - 1);
            i = g >> log2nfft;
        } else {
            f = g >> lq;
            i = g & ((1 << lq) - 1);
        }
        const int k = i & (p - 1);
        base[q] = f * fs;
        jout[q] = ((i - k) << LR) + k;
#pragma unroll
        for (int r = 0; r < RAD; ++r) x[q * RAD + r] = s[pad_idx<C>(base[q] + (i + (r << lq)) * es)];
        if (p > 1) {
            // w_{p*RAD}^{r*k} = tw[r * k * n / (p * RAD)]
            const int stride = (n / (p * RAD)) * k;
#pragma unroll
            for (int r = 1; r < RAD; ++r) x[q * RAD + r] = mul_w<C, INV>(x[q * RAD + r], __ldg(&tw[r * stride]));
        }
        if (RAD == 8) dft8<C, INV>(&x[q * RAD]);
        else if (RAD == 4) dft4<C, INV>(x[q * RAD], x[q * RAD + 1], x[q * RAD + 2], x[q * RAD + 3]);
        else dft2<C, INV>(x[q * RAD], x[q * RAD + 1]);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
#pragma unroll
        for (int r = 0; r < RAD; ++r) s[pad_idx<C>(base[q] + (jout[q] + r * p) * es)] = x[q * RAD + r];
    }
    __syncthreads();
}

// Full transform of every length-n sequence in the tile (2^log2nfft sequences).
// Requires blockDim.x * 8 == 2^log2nfft * n and n >= 2.  The tile must be visible to all
// threads (a __syncthreads() after filling it) on entry; it is complete and visible on
// exit.
template <class C, bool INV, bool F_FAST>
__device__ void tile_fft(C* s, int log2n, int log2nfft, int fs, int es, const C* __restrict__ tw) {
    int p = 1;
    int rem = log2n;
    // radix-4 first when log2n % 3 == 2, radix-2 first when log2n % 3 == 1, then radix-8
    if (rem % 3 == 2) {
        stockham_stage<C, 2, INV, F_FAST>(s, log2n, log2nfft, p, fs, es, tw);
        p <<= 2;
        rem -= 2;
    } else if (rem % 3 == 1) {
        stockham_stage<C, 1, INV, F_FAST>(s, log2n, log2nfft, p, fs, es, tw);
        p <<= 1;
        rem -= 1;
    }
    while (rem > 0) {
        stockham_stage<C, 3, INV, F_FAST>(s, log2n, log2nfft, p, fs, es, tw);
        p <<= 3;
        rem -= 3;
    }
}

// ---- compile-time sizes -------------------------------------------------------
// The same Stockham stages with the transform length, the tile count and the strides
// known at compile time (fs = 1, es = 2^LOG2NFFT for column tiles; fs = 2^LOG2N, es = 1
// for row tiles), so that the index arithmetic folds into constants and the stage loop
// unrolls.  Used for the FFT lengths of the measured configurations.
template <class C, int LR, bool INV, bool F_FAST, int LOG2N, int LOG2NFFT, int P, int EPT>
__device__ __forceinline__ void stockham_stage_ct(C* s, const C* __restrict__ tw) {
    constexpr int RAD = 1 << LR;
    constexpr int ITEMS = EPT / RAD;
    constexpr int n = 1 << LOG2N;
    constexpr int lq = LOG2N - LR;
    constexpr int fs = F_FAST ? 1 : n;
    constexpr int es = F_FAST ? (1 << LOG2NFFT) : 1;
    C x[EPT];
    int base[ITEMS], jout[ITEMS];
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
        const int g = threadIdx.x * ITEMS + q;
        int f, i;
        if (F_FAST) {
            f = g & ((1 << LOG2NFFT) - 1);
            i = g >> LOG2NFFT;
        } else {
            f = g >> lq;
            i = g & ((1 << lq) - 1);
        }
        const int k = i & (P - 1);
        base[q] = f * fs;
        jout[q] = ((i - k) << LR) + k;
#pragma unroll
        for (int r = 0; r < RAD; ++r) x[q * RAD + r] = s[pad_idx<C>(base[q] + (i + (r << lq)) * es)];
        if (P > 1) {
            constexpr int st = n / (P * RAD);
            const int stride = st * k;
#pragma unroll
            for (int r = 1; r < RAD; ++r) x[q * RAD + r] = mul_w<C, INV>(x[q * RAD + r], __ldg(&tw[r * stride]));
        }
        if (RAD == 8) dft8<C, INV>(&x[q * RAD]);
        else if (RAD == 4) dft4<C, INV>(x[q * RAD], x[q * RAD + 1], x[q * RAD + 2], x[q * RAD + 3]);
        else dft2<C, INV>(x[q * RAD], x[q * RAD + 1]);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
#pragma unroll
        for (int r = 0; r < RAD; ++r) s[pad_idx<C>(base[q] + (jout[q] + r * P) * es)] = x[q * RAD + r];
    }
    __syncthreads();
}

template <class C, bool INV, bool F_FAST, int LOG2N, int LOG2NFFT, int P, int REM, int EPT>
__device__ __forceinline__ void stages_ct(C* s, const C* __restrict__ tw) {
    if constexpr (REM > 0) {
        constexpr int LR = (P == 1 && REM % 3 == 2) ? 2 : ((P == 1 && REM % 3 == 1) ? 1 : 3);
        stockham_stage_ct<C, LR, INV, F_FAST, LOG2N, LOG2NFFT, P, EPT>(s, tw);
        stages_ct<C, INV, F_FAST, LOG2N, LOG2NFFT, (P << LR), REM - LR, EPT>(s, tw);
    }
}

// tile_fft with compile-time sizes: the same stage sequence (radix 4 or 2 first, then 8).
// EPT elements per thread (8, or 16 for a tile of twice the transforms on the same threads).
template <class C, bool INV, bool F_FAST, int LOG2N, int LOG2NFFT, int EPT = 8>
__device__ __forceinline__ void tile_fft_ct(C* s, const C* __restrict__ tw) {
    stages_ct<C, INV, F_FAST, LOG2N, LOG2NFFT, 1, LOG2N, EPT>(s, tw);
}

// ---- mixed lengths N = R * 2^a (R = 3 or 5), compile-time sizes ------------------
// The general Stockham stage: butterfly i of a transform reads x[i + r N/RAD], applies
// w_{P RAD}^{r k} (k = i mod P) and writes x[(i - k) RAD + k + r P].  Radix 3 and 5 stages
// stride their butterflies over the threads (EPT / RAD is not an integer); the others
// keep EPT / RAD consecutive butterflies per thread.
template <class C, int RAD, bool INV, bool F_FAST, int N, int LOG2NFFT, int P, int EPT>
__device__ __forceinline__ void stockham_stage_mx(C* s, const C* __restrict__ tw) {
    constexpr int NB = N / RAD;
    constexpr int NT = 1 << LOG2NFFT;
    constexpr int TOTAL = NT * NB;
    constexpr int NTHR = NT * N / EPT;
    constexpr bool STRIDED = (EPT % RAD) != 0;
    constexpr int ITEMS = STRIDED ? (TOTAL + NTHR - 1) / NTHR : EPT / RAD;
    constexpr int fs = F_FAST ? 1 : N;
    constexpr int es = F_FAST ? NT : 1;
    C x[ITEMS * RAD];
    int base[ITEMS], jout[ITEMS];
    bool ok[ITEMS];
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
        const int g = STRIDED ? static_cast<int>(threadIdx.x) + q * NTHR : static_cast<int>(threadIdx.x) * ITEMS + q;
        ok[q] = g < TOTAL;
        const int gg = ok[q] ? g : 0;
        int f, i;
        if (F_FAST) {
            f = gg % NT;
            i = gg / NT;
        } else {
            f = gg / NB;
            i = gg % NB;
        }
        const int k = i % P;
        base[q] = f * fs;
        jout[q] = (i - k) * RAD + k;
#pragma unroll
        for (int r = 0; r < RAD; ++r) x[q * RAD + r] = s[pad_idx<C>(base[q] + (i + r * NB) * es)];
        if (P > 1) {
            const int stride = (N / (P * RAD)) * k;
#pragma unroll
            for (int r = 1; r < RAD; ++r) x[q * RAD + r] = mul_w<C, INV>(x[q * RAD + r], __ldg(&tw[r * stride]));
        }
        if (RAD == 8) dft8<C, INV>(&x[q * RAD]);
        else if (RAD == 5) dft5<C, INV>(&x[q * RAD]);
        else if (RAD == 4) dft4<C, INV>(x[q * RAD], x[q * RAD + 1], x[q * RAD + 2], x[q * RAD + 3]);
        else if (RAD == 3) dft3<C, INV>(x[q * RAD], x[q * RAD + 1], x[q * RAD + 2]);
        else dft2<C, INV>(x[q * RAD], x[q * RAD + 1]);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < ITEMS; ++q) {
        if (!ok[q]) continue;
#pragma unroll
        for (int r = 0; r < RAD; ++r) s[pad_idx<C>(base[q] + (jout[q] + r * P) * es)] = x[q * RAD + r];
    }
    __syncthreads();
}

template <class C, bool INV, bool F_FAST, int N, int LOG2NFFT, int P, int REM, int EPT>
__device__ __forceinline__ void stages_mx_pow2(C* s, const C* __restrict__ tw) {
    if constexpr (REM > 0) {
        constexpr int LR2 = (REM % 3 == 2) ? 2 : ((REM % 3 == 1) ? 1 : 3);
        stockham_stage_mx<C, (1 << LR2), INV, F_FAST, N, LOG2NFFT, P, EPT>(s, tw);
        stages_mx_pow2<C, INV, F_FAST, N, LOG2NFFT, P * (1 << LR2), REM - LR2, EPT>(s, tw);
    }
}

// Transform of length N = RADIX * 2^LOG2A (RADIX 3 or 5): the radix stage first, then the
// power-of-two stages (radix 4 or 2 first when needed, then 8).  The tile holds 2^LOG2NFFT
// transforms; EPT * threads == 2^LOG2NFFT * N.  tw[m] = exp(-2 pi i m / N), m < N.
template <class C, bool INV, bool F_FAST, int RADIX, int LOG2A, int LOG2NFFT, int EPT = 8>
__device__ __forceinline__ void tile_fft_mx(C* s, const C* __restrict__ tw) {
    constexpr int N = RADIX << LOG2A;
    stockham_stage_mx<C, RADIX, INV, F_FAST, N, LOG2NFFT, 1, EPT>(s, tw);
    stages_mx_pow2<C, INV, F_FAST, N, LOG2NFFT, RADIX, LOG2A, EPT>(s, tw);
}

}  // namespace taco
