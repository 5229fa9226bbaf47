// bcf.cu -- bath correlation function C(t) from J(w) and beta on the device, and its
// derivatives with respect to the bath parameters.
//
// bcf_fft_fun (cpp/include/taco/correlation_fft.hpp:153-214): with Nt = N + 1 samples,
// nfft = next_pow2(2 Nt), dw = 2 pi / (dt nfft) and w_ny = pi / dt, the KMS spectrum
//   S[k]        = (pi/2) J(k dw) / (1 - e^{-beta k dw})               0 < k < nfft/2
//   S[nfft - k] = (pi/2) J(k dw) e^{-beta k dw} / (1 - e^{-beta k dw})
//   S[0]        = (pi/4) J(dw) (1 + r) / (1 - r),  r = e^{-beta dw}
//   S[nfft/2]   = (pi/4) J(w_ny) coth(beta w_ny / 2)
// (beta = inf: the positive half (pi/2) J, S[0] = 0, S[nfft/2] = (pi/4) J(w_ny)) is
// transformed forward and C(t_k) = (dw / pi) FFT(S)[k], k < Nt.  The reference builds
// e^{-beta k dw} by a running product; here each factor is evaluated directly (expm1
// for 1 - e^{-x}), which removes the O(k eps) drift of the product.
//
// J is the Ohmic alpha w e^{-w/wc}, optionally plus the Drude-Lorentz term
// 2 lam gam w / (w^2 + gam^2).  Derivative modes transform dS/dtheta instead of S, for
// theta in {alpha, wc, beta} (the Drude-Lorentz parameters are held fixed): the tangent
// correlation functions dC/dtheta used by the adjoint.
//
// The transform is a two-pass four-step FFT, nfft = N1 N2:
//   pass 1 (one CTA per 8 columns n2): the spectrum is generated in shared memory, the
//     N1-point transforms run along n1, and y[k1][n2] = W_nfft^{n2 k1} (...) is stored;
//   pass 2 (one CTA per 8 rows k1): N2-point transforms along n2 give
//     X[k1 + N1 k2]; only the requested k < n_out are written (scaled by dw / pi).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <vector>

#include "common.cuh"
#include "engine.hpp"
#include "fft.cuh"

namespace taco {

namespace {

constexpr double kPi = 3.14159265358979323846;

struct BcfJob {
    int model, which;
    double alpha, wc, lam, gam, beta;
    double dw, wny;
    double scale;  // dw / pi
    double2* out;
    uint32_t n_out;
};

__device__ __forceinline__ double bcf_J(const BcfJob& j, double w, int which) {
    if (!(w > 0.0)) return 0.0;
    const double e = exp(-w / j.wc);
    if (which == 1) return w * e;                               // dJ/dalpha
    if (which == 2) return j.alpha * w * e * w / (j.wc * j.wc);  // dJ/dwc
    double v = j.alpha * w * e;
    if (j.model == 1) v += 2.0 * j.lam * j.gam * w / (w * w + j.gam * j.gam);
    return v;
}

// Spectrum sample n of an nfft-point grid (or its beta derivative when which == 3).
__device__ double bcf_S(const BcfJob& j, uint32_t n, uint32_t nfft) {
    const uint32_t half = nfft >> 1;
    const bool dbeta = j.which == 3;
    const int jw = dbeta ? 0 : j.which;
    const bool inf = isinf(j.beta);
    if (n == 0) {
        if (inf) return 0.0;
        const double x = j.beta * j.dw;
        const double em = -expm1(-x), r = exp(-x);  // 1 - r, r
        const double Jv = bcf_J(j, j.dw, jw);
        return dbeta ? 0.25 * kPi * Jv * (-2.0 * j.dw * r / (em * em)) : 0.25 * kPi * Jv * (1.0 + r) / em;
    }
    if (n == half) {
        const double Jv = bcf_J(j, j.wny, jw);
        if (inf) return dbeta ? 0.0 : 0.25 * kPi * Jv;
        const double x = j.beta * j.wny;
        const double em = -expm1(-x), ex = exp(-x);
        return dbeta ? 0.25 * kPi * Jv * (-2.0 * j.wny * ex / (em * em)) : 0.25 * kPi * Jv * (1.0 + 2.0 * ex / em);
    }
    const bool pos = n < half;
    const uint32_t k = pos ? n : nfft - n;
    const double w = j.dw * static_cast<double>(k);
    const double Jv = bcf_J(j, w, jw);
    if (inf) return (pos && !dbeta) ? 0.5 * kPi * Jv : 0.0;
    const double x = j.beta * w;
    const double em = -expm1(-x), ex = exp(-x);
    if (dbeta) return -0.5 * kPi * Jv * w * ex / (em * em);  // same on both halves
    return pos ? 0.5 * kPi * Jv / em : 0.5 * kPi * Jv * ex / em;
}

__global__ void k_bcf_twiddle(double2* tw, uint32_t n) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double s, c;
    sincospi(-2.0 * static_cast<double>(m) / static_cast<double>(n), &s, &c);
    tw[m] = make_double2(c, s);
}

// Pass 1: columns n2 in [c0, c0 + CT) of job blockIdx.y; blockDim.x = CT * N1 / 8.
__global__ void __launch_bounds__(1024) k_bcf_cols(const BcfJob* __restrict__ jobs, int L1, int L2, int lct,
                                                   const double2* __restrict__ tw1, double2* __restrict__ y) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* s = reinterpret_cast<double2*>(smem_raw);
    const BcfJob j = jobs[blockIdx.y];
    const uint32_t N1 = 1u << L1, N2 = 1u << L2, CT = 1u << lct, nfft = N1 << L2;
    const uint32_t c0 = blockIdx.x * CT;
    const uint32_t total = CT * N1;
    for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const uint32_t f = idx & (CT - 1), n1 = idx >> lct;
        s[pad_idx<double2>(f + n1 * CT)] = make_double2(bcf_S(j, n1 * N2 + c0 + f, nfft), 0.0);
    }
    __syncthreads();
    tile_fft<double2, false, true>(s, L1, lct, 1, CT, tw1);
    double2* yj = y + static_cast<size_t>(blockIdx.y) * nfft;
    for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const uint32_t f = idx & (CT - 1), k1 = idx >> lct;
        const uint32_t n2 = c0 + f;
        const uint64_t e = (static_cast<uint64_t>(n2) * k1) & (nfft - 1);
        double sn, cs;
        sincospi(-2.0 * static_cast<double>(e) / static_cast<double>(nfft), &sn, &cs);
        yj[static_cast<size_t>(k1) * N2 + n2] = cmul(s[pad_idx<double2>(f + k1 * CT)], make_double2(cs, sn));
    }
}

// Pass 2: rows k1 in [r0, r0 + RT) of job blockIdx.y; blockDim.x = RT * N2 / 8.
__global__ void __launch_bounds__(1024) k_bcf_rows(const BcfJob* __restrict__ jobs, int L1, int L2, int lrt,
                                                   const double2* __restrict__ tw2, const double2* __restrict__ y) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* s = reinterpret_cast<double2*>(smem_raw);
    const BcfJob j = jobs[blockIdx.y];
    const uint32_t N1 = 1u << L1, N2 = 1u << L2, RT = 1u << lrt, nfft = N1 << L2;
    const uint32_t r0 = blockIdx.x * RT;
    const uint32_t total = RT * N2;
    const double2* yj = y + static_cast<size_t>(blockIdx.y) * nfft + static_cast<size_t>(r0) * N2;
    for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) s[pad_idx<double2>(idx)] = yj[idx];
    __syncthreads();
    tile_fft<double2, false, false>(s, L2, lrt, N2, 1, tw2);
    for (uint32_t idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const uint32_t f = idx & (RT - 1), k2 = idx >> lrt;
        const uint64_t k = static_cast<uint64_t>(r0 + f) + static_cast<uint64_t>(N1) * k2;
        if (k < j.n_out) j.out[k] = cscale(s[pad_idx<double2>(f * N2 + k2)], j.scale);
    }
}

struct BcfScratch {
    void* p = nullptr;
    std::size_t cap = 0;
    double2* ensure(std::size_t bytes) {
        if (bytes > cap) {
            if (p) cudaFree(p);
            p = nullptr;
            cap = 0;
            cuda_check(cudaMalloc(&p, bytes), "cudaMalloc(bcf scratch)");
            cap = bytes;
        }
        return static_cast<double2*>(p);
    }
    ~BcfScratch() {
        if (p) cudaFree(p);
    }
};

BcfScratch& bcf_scratch() {
    thread_local std::map<int, BcfScratch> per_dev;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    return per_dev[dev];
}

}  // namespace

std::size_t bcf_nfft(std::size_t N) {
    const std::size_t nfft = 2 * (N + 1);
    return (nfft & (nfft - 1)) ? next_pow2(nfft) : nfft;
}

void bcf_device(const std::vector<BcfRequest>& reqs, cudaStream_t st) {
    // group by FFT length; one pass-1 and one pass-2 launch per group
    std::map<std::size_t, std::vector<const BcfRequest*>> groups;
    for (const auto& r : reqs) {
        if (r.model != 0 && r.model != 1) throw Error(kInvalidArgument, "bcf: unknown spectral density model");
        if (r.which < 0 || r.which > 3) throw Error(kInvalidArgument, "bcf: derivative mode must be 0..3");
        if (!(r.dt > 0.0)) throw Error(kInvalidArgument, "bcf: dt must be > 0");
        if (!(r.omega_c > 0.0)) throw Error(kInvalidArgument, "bcf: omega_c must be > 0");
        if (!(r.beta > 0.0)) throw Error(kInvalidArgument, "bcf: beta must be > 0");
        if (r.which == 3 && std::isinf(r.beta)) throw Error(kInvalidArgument, "bcf: d/dbeta needs a finite beta");
        if (r.n_out == 0 || r.n_out > r.N + 1) throw Error(kOutOfRange, "bcf: n_out must be in [1, N + 1]");
        if (r.out == nullptr) throw Error(kInvalidArgument, "bcf: null output");
        const std::size_t nfft = bcf_nfft(r.N);
        if (nfft > (std::size_t(1) << 20) || nfft < 8) throw Error(kOverflow, "bcf: FFT length outside [8, 2^20]");
        groups[nfft].push_back(&r);
    }
    for (auto& g : groups) {
        const std::size_t nfft = g.first;
        const auto& rs = g.second;
        const int L = ilog2(nfft), L2 = L / 2, L1 = L - L2;
        const uint32_t N1 = 1u << L1, N2 = 1u << L2;
        const int lct = std::min(3, L2), lrt = std::min(3, L1);
        std::vector<BcfJob> jobs(rs.size());
        uint32_t max_out = 0;
        for (std::size_t q = 0; q < rs.size(); ++q) {
            const BcfRequest& r = *rs[q];
            BcfJob& j = jobs[q];
            j.model = r.model;
            j.which = r.which;
            j.alpha = r.alpha;
            j.wc = r.omega_c;
            j.lam = r.lambda;
            j.gam = r.gamma;
            j.beta = r.beta;
            j.dw = 2.0 * kPi / (r.dt * static_cast<double>(nfft));
            j.wny = kPi / r.dt;
            j.scale = j.dw / kPi;
            j.out = r.out;
            j.n_out = static_cast<uint32_t>(r.n_out);
            max_out = std::max(max_out, j.n_out);
        }
        for (std::size_t q0 = 0; q0 < jobs.size(); q0 += 65535) {
            const std::size_t nj = std::min<std::size_t>(65535, jobs.size() - q0);
            const std::size_t bytes_y = nj * nfft * sizeof(double2);
            const std::size_t bytes_meta = nj * sizeof(BcfJob) + (N1 + N2) * sizeof(double2) + 512;
            char* base = reinterpret_cast<char*>(bcf_scratch().ensure(bytes_y + bytes_meta));
            double2* y = reinterpret_cast<double2*>(base);
            double2* tw1 = reinterpret_cast<double2*>(base + bytes_y);
            double2* tw2 = tw1 + N1;
            BcfJob* dj = reinterpret_cast<BcfJob*>(reinterpret_cast<char*>(tw2 + N2) + 256 - (reinterpret_cast<uintptr_t>(tw2 + N2) & 255));
            cuda_check(cudaMemcpyAsync(dj, jobs.data() + q0, nj * sizeof(BcfJob), cudaMemcpyHostToDevice, st), "bcf jobs");
            k_bcf_twiddle<<<(N1 + 255) / 256, 256, 0, st>>>(tw1, N1);
            launched("k_bcf_twiddle");
            k_bcf_twiddle<<<(N2 + 255) / 256, 256, 0, st>>>(tw2, N2);
            launched("k_bcf_twiddle");
            const uint32_t CT = 1u << lct, RT = 1u << lrt;
            const std::size_t smem1 = padded_size<double2>(static_cast<int>(CT * N1)) * sizeof(double2);
            const std::size_t smem2 = padded_size<double2>(static_cast<int>(RT * N2)) * sizeof(double2);
            cuda_check(cudaFuncSetAttribute(k_bcf_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem1)),
                       "cudaFuncSetAttribute(k_bcf_cols)");
            cuda_check(cudaFuncSetAttribute(k_bcf_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem2)),
                       "cudaFuncSetAttribute(k_bcf_rows)");
            k_bcf_cols<<<dim3(N2 / CT, static_cast<unsigned>(nj)), CT * N1 / 8, smem1, st>>>(dj, L1, L2, lct, tw1, y);
            launched("k_bcf_cols");
            const uint32_t rows = std::min<uint32_t>(N1, max_out);
            k_bcf_rows<<<dim3((rows + RT - 1) / RT, static_cast<unsigned>(nj)), RT * N2 / 8, smem2, st>>>(dj, L1, L2, lrt,
                                                                                                       tw2, y);
            launched("k_bcf_rows");
            // the scratch is reused by the next chunk: order it after this one
            if (q0 + nj < jobs.size()) cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(bcf)");
        }
    }
}

}  // namespace taco
