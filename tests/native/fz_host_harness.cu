// Host build of the fused path's transform stages (taco_b200/csrc/fused_conv.cuh) for the
// CPU tests: the stages run with one "thread" looping over all butterflies, stage after
// stage, which is what the barriers between stages guarantee on the device.
#include <cmath>
#include <vector>

#include "fused_conv.cuh"

using namespace taco;

template <class C>
static int convolve(int N, int max_radix, const double* a, const double* b, double* out) {
    using R = decltype(C{}.x);
    FzPlan<C> p{};
    p.N = N;
    if (!fz_stages(N, max_radix, p.rad, p.nst)) return 1;
    std::vector<C> tw(std::max<std::size_t>(1, fz_table_layout(p)));
    for (std::size_t e = 0; e < tw.size(); ++e) {
        int M, pp, j;
        fz_table_entry(p, e, M, pp, j);
        const double ang = -2.0 * M_PI * static_cast<double>(pp) * static_cast<double>(j) / M;
        tw[e] = C{static_cast<R>(std::cos(ang)), static_cast<R>(std::sin(ang))};
    }
    p.tw = tw.data();
    std::vector<C> x(padded_size<C>(N)), y(padded_size<C>(N));
    for (int t = 0; t < N; ++t) {
        x[pad_idx<C>(t)] = C{static_cast<R>(a[2 * t]), static_cast<R>(a[2 * t + 1])};
        y[pad_idx<C>(t)] = C{static_cast<R>(b[2 * t]), static_cast<R>(b[2 * t + 1])};
    }
    for (auto* d : {&x, &y})
        for (int s = 0; s < p.nst; ++s) {
            int M, lm;
            fz_shape(p, s, M, lm);
            fz_stage_any<C, false>(d->data(), N, M, p.rad[s], lm, p.tw + p.twoff[s], 0, 1);
        }
    for (int i = 0; i < N; ++i) x[pad_idx<C>(i)] = cmul(x[pad_idx<C>(i)], y[pad_idx<C>(i)]);
    for (int s = p.nst - 1; s >= 0; --s) {
        int M, lm;
        fz_shape(p, s, M, lm);
        fz_stage_any<C, true>(x.data(), N, M, p.rad[s], lm, p.tw + p.twoff[s], 0, 1);
    }
    for (int t = 0; t < N; ++t) {
        out[2 * t] = static_cast<double>(x[pad_idx<C>(t)].x) / N;
        out[2 * t + 1] = static_cast<double>(x[pad_idx<C>(t)].y) / N;
    }
    return 0;
}

// Circular convolution of a and b (interleaved complex, length N) by the fused path's
// forward stages, pointwise product and inverse stages; fp32 selects float2 arithmetic.
extern "C" int fz_host_convolve(int N, int fp32, int max_radix, const double* a, const double* b, double* out) {
    return fp32 ? convolve<float2>(N, max_radix, a, b, out) : convolve<double2>(N, max_radix, a, b, out);
}
