// tcl2.cu -- second-order generator series L2(t) and the trapezoid Gamma(w, t) on the device.
//
// L2(t) is the TCL2 generator total() of cpp/src/tcl/generator.cpp:164-177 with the
// spin-boson example's kernel fill (examples/TCL4_spin_boson_example.cpp:303-315:
// Gamma_b(alpha, alpha) = Gamma_b(t) for every channel, zero across channels):
//   L2(t) = -i[diag(eps) + H_LS(t), .] + sum_{b,alpha} gamma_b(t) [conj(A_ab) (x) A_ab
//           - 1/2 I (x) A_ab^+ A_ab - 1/2 (A_ab^+ A_ab)^T (x) I],
//   H_LS(t) = hermitize(sum_{b,alpha} S_b(t) A_ab^+ A_ab),  gamma_b = 2 Re Gamma_b, S_b = Im Gamma_b,
// with A_ab the entries of the eigenbasis coupling operator alpha on the pairs of bucket b
// (system.hpp:163-182).  It is affine in (gamma_b, S_b):
//   L2(t) = L0 + sum_b gamma_b(t) D_b + sum_b S_b(t) U_b,
// so the host forms L0, D_b, U_b once (N^2 x N^2 each) and one kernel writes L2 at every
// requested time.  Terms the reference skips (zero gamma, zero S, zero A_ab^+ A_ab) add
// exact zeros here.
//
// gamma_trapz: Gamma_b(t_k) = sum_{m<k} dt/2 (phi_m C_m + phi_{m+1} C_{m+1}),
// phi_m = exp(i w_b m dt) (cpp/include/taco/gamma.hpp:166-213), as a reduce-then-scan over
// chunks of 1024 samples with FP64 sums (phases from sincos rather than the reference's
// running product, which drifts by O(k eps)).
#include <cuda_runtime.h>

#include <algorithm>
#include <complex>
#include <map>
#include <vector>

#include "common.cuh"
#include "engine.hpp"

namespace taco {

namespace {

using cd = std::complex<double>;

// --------------------------------------------------------------- TCL2 series
__global__ void k_tcl2_series(const double2* __restrict__ gamma, std::size_t Nt, int nf, const uint32_t* __restrict__ tidx,
                              uint32_t T, const double2* __restrict__ L0, const double2* __restrict__ Db,
                              const double2* __restrict__ Ub, uint32_t E, double2* __restrict__ out) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t o = blockIdx.y;
    if (e >= E || o >= T) return;
    const uint32_t t = tidx[o];
    double2 acc = L0[e];
    for (int b = 0; b < nf; ++b) {
        const double2 g = gamma[static_cast<std::size_t>(b) * Nt + t];
        const double gam = 2.0 * g.x, S = g.y;
        const double2 d = Db[static_cast<std::size_t>(b) * E + e];
        const double2 u = Ub[static_cast<std::size_t>(b) * E + e];
        acc.x += gam * d.x + S * u.x;
        acc.y += gam * d.y + S * u.y;
    }
    out[static_cast<std::size_t>(o) * E + e] = acc;
}

// kron(A, B) entry (r1 n + r2, c1 n + c2) = A(r1, c1) B(r2, c2); column-major N^2 x N^2.
void kron_add(std::vector<cd>& L, int n, const std::vector<cd>& A, const std::vector<cd>& B, cd s) {
    const std::size_t D = static_cast<std::size_t>(n) * n;
    for (int r1 = 0; r1 < n; ++r1)
        for (int c1 = 0; c1 < n; ++c1) {
            const cd a = A[r1 + n * c1];
            if (a == cd(0.0, 0.0)) continue;
            for (int r2 = 0; r2 < n; ++r2)
                for (int c2 = 0; c2 < n; ++c2)
                    L[(static_cast<std::size_t>(r1) * n + r2) + D * (static_cast<std::size_t>(c1) * n + c2)] +=
                        s * a * B[r2 + n * c2];
        }
}

// -i (kron(I, H) - kron(H^T, I)) (generator.cpp:81-90)
void unitary_add(std::vector<cd>& L, int n, const std::vector<cd>& H, cd s) {
    std::vector<cd> I(static_cast<std::size_t>(n) * n, cd(0.0, 0.0)), HT(I.size());
    for (int i = 0; i < n; ++i) I[i + n * i] = 1.0;
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) HT[r + n * c] = H[c + n * r];
    kron_add(L, n, I, H, s * cd(0.0, -1.0));
    kron_add(L, n, HT, I, s * cd(0.0, 1.0));
}

// ------------------------------------------------------------- Gamma (trapz)
constexpr int GT_THREADS = 256;
constexpr int GT_ITEMS = 4;
constexpr int GT_CHUNK = GT_THREADS * GT_ITEMS;

// trapezoid increment of step k (k >= 1): dt/2 (phi_{k-1} C_{k-1} + phi_k C_k)
__device__ __forceinline__ double2 trapz_inc(const double2* C, double w, double dt, std::size_t k) {
    double s0, c0, s1, c1;
    sincos(w * (static_cast<double>(k - 1) * dt), &s0, &c0);
    sincos(w * (static_cast<double>(k) * dt), &s1, &c1);
    const double2 a = cmul(make_double2(c0, s0), C[k - 1]);
    const double2 b = cmul(make_double2(c1, s1), C[k]);
    return make_double2(0.5 * dt * (a.x + b.x), 0.5 * dt * (a.y + b.y));
}

// One Gamma job: C [N] (device), omegas [nb] (device), G [nb][N] (device), and its
// per-(bucket, chunk) partial sums.
struct GammaJob {
    const double2* C;
    std::size_t N;
    double dt;
    const double* omegas;
    int nb, nchunks;
    double2* G;
    double2* partial;  // [nb][nchunks]
};

// grid (chunk, bucket, job)
__global__ void k_gamma_reduce(const GammaJob* __restrict__ jobs) {
    __shared__ double2 wsum[GT_THREADS / 32];
    const GammaJob j = jobs[blockIdx.z];
    const int b = blockIdx.y;
    if (b >= j.nb || static_cast<int>(blockIdx.x) >= j.nchunks) return;
    const std::size_t k0 = static_cast<std::size_t>(blockIdx.x) * GT_CHUNK + threadIdx.x * GT_ITEMS;
    const double w = j.omegas[b];
    double2 s = make_double2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < GT_ITEMS; ++q) {
        const std::size_t k = k0 + q;
        if (k >= 1 && k < j.N) s = cadd(s, trapz_inc(j.C, w, j.dt, k));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
        s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
    }
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int q = 0; q < GT_THREADS / 32; ++q) t = cadd(t, wsum[q]);
        j.partial[static_cast<std::size_t>(b) * j.nchunks + blockIdx.x] = t;
    }
}

__global__ void k_gamma_scan(const GammaJob* __restrict__ jobs) {
    __shared__ double2 wsum[GT_THREADS / 32];
    __shared__ double2 carry;
    const GammaJob j = jobs[blockIdx.z];
    const int b = blockIdx.y;
    if (b >= j.nb || static_cast<int>(blockIdx.x) >= j.nchunks) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        double2 t = make_double2(0.0, 0.0);
        for (int c = 0; c < static_cast<int>(blockIdx.x); ++c) t = cadd(t, j.partial[static_cast<std::size_t>(b) * j.nchunks + c]);
        carry = t;
    }
    const std::size_t k0 = static_cast<std::size_t>(blockIdx.x) * GT_CHUNK + threadIdx.x * GT_ITEMS;
    const double w = j.omegas[b];
    double2 v[GT_ITEMS];
    double2 run = make_double2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < GT_ITEMS; ++q) {
        const std::size_t k = k0 + q;
        v[q] = (k >= 1 && k < j.N) ? trapz_inc(j.C, w, j.dt, k) : make_double2(0.0, 0.0);
        run = cadd(run, v[q]);
    }
    double2 x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double nx = __shfl_up_sync(0xffffffffu, x.x, o);
        const double ny = __shfl_up_sync(0xffffffffu, x.y, o);
        if (lane >= o) {
            x.x += nx;
            x.y += ny;
        }
    }
    if (lane == 31) wsum[warp] = x;
    double2 excl = make_double2(__shfl_up_sync(0xffffffffu, x.x, 1), __shfl_up_sync(0xffffffffu, x.y, 1));
    if (lane == 0) excl = make_double2(0.0, 0.0);
    __syncthreads();
    double2 pre = carry;
    for (int q = 0; q < warp; ++q) pre = cadd(pre, wsum[q]);
    pre = cadd(pre, excl);
    double2* Gb = j.G + static_cast<std::size_t>(b) * j.N;
#pragma unroll
    for (int q = 0; q < GT_ITEMS; ++q) {
        const std::size_t k = k0 + q;
        pre = cadd(pre, v[q]);
        if (k < j.N) Gb[k] = pre;  // G(0) = 0: the k = 0 increment is zero
    }
}

__global__ void k_add_c64(const float2* __restrict__ src, double2* __restrict__ dst, std::size_t n) {
    for (std::size_t k = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<std::size_t>(gridDim.x) * blockDim.x)
        dst[k] = cadd(dst[k], to_d2(src[k]));
}

// Grow-only device scratch per host thread and device (the small maps and partial sums).
struct Tcl2Scratch {
    void* p = nullptr;
    std::size_t cap = 0;
    char* ensure(std::size_t bytes) {
        if (bytes > cap) {
            if (p) cudaFree(p);
            p = nullptr;
            cap = 0;
            cuda_check(cudaMalloc(&p, bytes), "cudaMalloc(tcl2 scratch)");
            cap = bytes;
        }
        return static_cast<char*>(p);
    }
    ~Tcl2Scratch() {
        if (p) cudaFree(p);
    }
};

char* tcl2_scratch(std::size_t bytes) {
    thread_local std::map<int, Tcl2Scratch> per_dev;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    return per_dev[dev].ensure(bytes);
}

}  // namespace

void add_c64_into_c128(const float2* src, double2* dst, std::size_t n, cudaStream_t st) {
    const unsigned grid = static_cast<unsigned>(std::min<std::size_t>((n + 255) / 256, 148 * 16));
    k_add_c64<<<grid, 256, 0, st>>>(src, dst, n);
    launched("k_add_c64");
}

namespace {

// reverse of kron_add(L, n, A, B, s): G(A) and G(B) from G(L) (either may be null)
void kron_add_grad(const std::vector<cd>& GL, int n, const std::vector<cd>& A, const std::vector<cd>& B, cd s,
                   std::vector<cd>* GA, std::vector<cd>* GB) {
    const std::size_t D = static_cast<std::size_t>(n) * n;
    const cd sc = std::conj(s);
    for (int r1 = 0; r1 < n; ++r1)
        for (int c1 = 0; c1 < n; ++c1)
            for (int r2 = 0; r2 < n; ++r2)
                for (int c2 = 0; c2 < n; ++c2) {
                    const cd g = GL[(static_cast<std::size_t>(r1) * n + r2) + D * (static_cast<std::size_t>(c1) * n + c2)];
                    if (GA) (*GA)[r1 + n * c1] += sc * std::conj(B[r2 + n * c2]) * g;
                    if (GB) (*GB)[r2 + n * c2] += sc * std::conj(A[r1 + n * c1]) * g;
                }
}

// G(H) of unitary_add(L, n, H, 1) = -i kron(I, H) + i kron(H^T, I)
std::vector<cd> unitary_grad(const std::vector<cd>& GL, int n, const std::vector<cd>& H) {
    std::vector<cd> I(static_cast<std::size_t>(n) * n, cd(0.0, 0.0)), HT(I.size()), GH(I.size(), cd(0.0, 0.0)),
        GHT(I.size(), cd(0.0, 0.0));
    for (int i = 0; i < n; ++i) I[i + n * i] = 1.0;
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) HT[r + n * c] = H[c + n * r];
    kron_add_grad(GL, n, I, H, cd(0.0, -1.0), nullptr, &GH);
    kron_add_grad(GL, n, HT, I, cd(0.0, 1.0), &GHT, nullptr);
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) GH[c + n * r] += GHT[r + n * c];
    return GH;
}

// Coupling operator alpha restricted to the pairs of bucket b, its A^+ A, and whether the
// reference includes the term (non-zero A_ab and non-zero A^+ A).
bool bucket_op(const SystemDesc& s, int b, int al, std::vector<cd>& Aw, std::vector<cd>& AdA) {
    const int n = s.N;
    const std::size_t D = static_cast<std::size_t>(n) * n;
    const cd* ops = reinterpret_cast<const cd*>(s.ops.data());
    Aw.assign(D, cd(0.0, 0.0));
    AdA.assign(D, cd(0.0, 0.0));
    double nrm = 0.0;
    for (std::size_t k = 0; k < D; ++k)
        if (s.p2f[k] == b) {
            Aw[k] = ops[static_cast<std::size_t>(al) * D + k];
            nrm += std::norm(Aw[k]);
        }
    if (nrm == 0.0) return false;
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            cd acc(0.0, 0.0);
            for (int k = 0; k < n; ++k) acc += std::conj(Aw[k + n * r]) * Aw[k + n * c];
            AdA[r + n * c] = acc;
        }
    double an = 0.0;
    for (auto& x : AdA) an += std::norm(x);
    return an != 0.0;
}

}  // namespace

void tcl2_maps(const SystemDesc& sys, const double* eps, std::vector<double2>& L0out, std::vector<double2>& Dbout,
               std::vector<double2>& Ubout) {
    const int n = sys.N, nf = sys.nf;
    const std::size_t D = static_cast<std::size_t>(n) * n, E = D * D;
    std::vector<cd> L0(E, cd(0.0, 0.0)), Db(nf * E, cd(0.0, 0.0)), Ub(nf * E, cd(0.0, 0.0));
    std::vector<cd> Hd(D, cd(0.0, 0.0)), I(D, cd(0.0, 0.0));
    for (int i = 0; i < n; ++i) {
        Hd[i + n * i] = eps[i];
        I[i + n * i] = 1.0;
    }
    unitary_add(L0, n, Hd, 1.0);
    for (int b = 0; b < nf; ++b) {
        std::vector<cd> D_b(E, cd(0.0, 0.0)), AdA_sum(D, cd(0.0, 0.0));
        for (int al = 0; al < sys.num_ops; ++al) {
            std::vector<cd> Aw, AdA;
            if (!bucket_op(sys, b, al, Aw, AdA)) continue;
            std::vector<cd> Ac(D), AdAT(D);
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < n; ++c) {
                    Ac[r + n * c] = std::conj(Aw[r + n * c]);
                    AdAT[r + n * c] = AdA[c + n * r];
                }
            kron_add(D_b, n, Ac, Aw, 1.0);
            kron_add(D_b, n, I, AdA, -0.5);
            kron_add(D_b, n, AdAT, I, -0.5);
            for (std::size_t k = 0; k < D; ++k) AdA_sum[k] += AdA[k];
        }
        std::vector<cd> Hh(D);  // hermitize (ops.hpp:234)
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) Hh[r + n * c] = 0.5 * (AdA_sum[r + n * c] + std::conj(AdA_sum[c + n * r]));
        std::vector<cd> U_b(E, cd(0.0, 0.0));
        unitary_add(U_b, n, Hh, 1.0);
        std::copy(D_b.begin(), D_b.end(), Db.begin() + static_cast<std::ptrdiff_t>(b * E));
        std::copy(U_b.begin(), U_b.end(), Ub.begin() + static_cast<std::ptrdiff_t>(b * E));
    }
    auto out = [](const std::vector<cd>& v, std::vector<double2>& o) {
        o.resize(v.size());
        for (std::size_t k = 0; k < v.size(); ++k) o[k] = make_double2(v[k].real(), v[k].imag());
    };
    out(L0, L0out);
    out(Db, Dbout);
    out(Ub, Ubout);
}

void tcl2_maps_grad(const SystemDesc& sys, const double* eps, const std::vector<double2>& GL0v,
                    const std::vector<double2>& GDv, const std::vector<double2>& GUv, double2* ops_bar, double* eps_bar) {
    const int n = sys.N, nf = sys.nf;
    const std::size_t D = static_cast<std::size_t>(n) * n, E = D * D;
    auto in = [](const double2* p, std::size_t cnt) {
        std::vector<cd> v(cnt);
        for (std::size_t k = 0; k < cnt; ++k) v[k] = cd(p[k].x, p[k].y);
        return v;
    };
    if (eps_bar) {
        std::vector<cd> Hd(D, cd(0.0, 0.0));
        for (int i = 0; i < n; ++i) Hd[i + n * i] = eps[i];
        const std::vector<cd> GH = unitary_grad(in(GL0v.data(), E), n, Hd);
        for (int i = 0; i < n; ++i) eps_bar[i] += GH[i + n * i].real();
    }
    if (!ops_bar) return;
    cd* G = reinterpret_cast<cd*>(ops_bar);
    std::vector<cd> I(D, cd(0.0, 0.0));
    for (int i = 0; i < n; ++i) I[i + n * i] = 1.0;
    for (int b = 0; b < nf; ++b) {
        const std::vector<cd> GD = in(GDv.data() + b * E, E), GU = in(GUv.data() + b * E, E);
        // U_b = unitary(Hh), Hh = (S + S^H) / 2, S = sum_alpha A^+ A over the included terms
        std::vector<cd> S(D, cd(0.0, 0.0));
        std::vector<std::vector<cd>> Aws, AdAs;
        std::vector<int> als;
        for (int al = 0; al < sys.num_ops; ++al) {
            std::vector<cd> Aw, AdA;
            if (!bucket_op(sys, b, al, Aw, AdA)) continue;
            for (std::size_t k = 0; k < D; ++k) S[k] += AdA[k];
            Aws.push_back(Aw);
            AdAs.push_back(AdA);
            als.push_back(al);
        }
        if (als.empty()) continue;
        std::vector<cd> Hh(D);
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) Hh[r + n * c] = 0.5 * (S[r + n * c] + std::conj(S[c + n * r]));
        const std::vector<cd> GHh = unitary_grad(GU, n, Hh);
        std::vector<cd> GS(D);
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) GS[r + n * c] = 0.5 * (GHh[r + n * c] + std::conj(GHh[c + n * r]));
        for (std::size_t a = 0; a < als.size(); ++a) {
            const std::vector<cd>& Aw = Aws[a];
            const std::vector<cd>& AdA = AdAs[a];
            std::vector<cd> Ac(D), AdAT(D);
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < n; ++c) {
                    Ac[r + n * c] = std::conj(Aw[r + n * c]);
                    AdAT[r + n * c] = AdA[c + n * r];
                }
            std::vector<cd> GAc(D, cd(0.0, 0.0)), GAw(D, cd(0.0, 0.0)), GAdA(GS), GAdAT(D, cd(0.0, 0.0));
            kron_add_grad(GD, n, Ac, Aw, 1.0, &GAc, &GAw);
            kron_add_grad(GD, n, I, AdA, -0.5, nullptr, &GAdA);
            kron_add_grad(GD, n, AdAT, I, -0.5, &GAdAT, nullptr);
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < n; ++c) GAdA[c + n * r] += GAdAT[r + n * c];
            // AdA = Aw^H Aw: G(Aw) += Aw (G + G^H)
            for (int r = 0; r < n; ++r)
                for (int c = 0; c < n; ++c) {
                    cd acc(0.0, 0.0);
                    for (int k = 0; k < n; ++k) acc += Aw[r + n * k] * (GAdA[k + n * c] + std::conj(GAdA[c + n * k]));
                    GAw[r + n * c] += acc + std::conj(GAc[r + n * c]);
                }
            for (std::size_t k = 0; k < D; ++k)
                if (sys.p2f[k] == b) G[static_cast<std::size_t>(als[a]) * D + k] += GAw[k];
        }
    }
}

void tcl2_series_device(const SystemDesc& sys, const double* eps, const double2* gamma, std::size_t Nt,
                        const std::vector<uint32_t>& tidx, double2* out, cudaStream_t st) {
    const int nf = sys.nf;
    const std::size_t E = static_cast<std::size_t>(sys.N) * sys.N * sys.N * sys.N;
    std::vector<double2> L0, Db, Ub;
    tcl2_maps(sys, eps, L0, Db, Ub);
    // device staging of the (small) maps: allocated for the call, released after it
    const std::size_t bytes = (E + 2 * nf * E) * sizeof(double2) + tidx.size() * sizeof(uint32_t);
    void* d = tcl2_scratch(bytes);
    {
        double2* dL0 = static_cast<double2*>(d);
        double2* dD = dL0 + E;
        double2* dU = dD + nf * E;
        uint32_t* dt = reinterpret_cast<uint32_t*>(dU + nf * E);
        cuda_check(cudaMemcpyAsync(dL0, L0.data(), E * sizeof(double2), cudaMemcpyHostToDevice, st), "tcl2 L0");
        cuda_check(cudaMemcpyAsync(dD, Db.data(), nf * E * sizeof(double2), cudaMemcpyHostToDevice, st), "tcl2 D");
        cuda_check(cudaMemcpyAsync(dU, Ub.data(), nf * E * sizeof(double2), cudaMemcpyHostToDevice, st), "tcl2 U");
        cuda_check(cudaMemcpyAsync(dt, tidx.data(), tidx.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st), "tcl2 t");
        const unsigned gx = static_cast<unsigned>((E + 127) / 128);
        for (std::size_t o0 = 0; o0 < tidx.size(); o0 += 65535) {
            const unsigned gy = static_cast<unsigned>(std::min<std::size_t>(65535, tidx.size() - o0));
            k_tcl2_series<<<dim3(gx, gy), 128, 0, st>>>(gamma, Nt, nf, dt + o0, gy, dL0, dD, dU,
                                                         static_cast<uint32_t>(E), out + o0 * E);
            launched("k_tcl2_series");
        }
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(tcl2)");
    }
}

void gamma_trapz_batch_device(const std::vector<GammaRequest>& reqs, cudaStream_t st) {
    if (reqs.empty()) return;
    std::size_t bytes = 256 + reqs.size() * sizeof(GammaJob);
    int max_nb = 0, max_chunks = 0;
    for (const auto& r : reqs) {
        if (!r.C || !r.G || r.N == 0 || r.omegas.empty() || !(r.dt > 0.0))
            throw Error(kInvalidArgument, "gamma_trapz: null or empty input");
        if (r.omegas.size() > 65535) throw Error(kInvalidArgument, "gamma_trapz: too many frequencies");
        const int nch = static_cast<int>((r.N + GT_CHUNK - 1) / GT_CHUNK);
        max_nb = std::max(max_nb, static_cast<int>(r.omegas.size()));
        max_chunks = std::max(max_chunks, nch);
        bytes += ((r.omegas.size() * sizeof(double) + 255) / 256) * 256 +
                 ((r.omegas.size() * nch * sizeof(double2) + 255) / 256) * 256;
    }
    char* base = tcl2_scratch(bytes);
    std::size_t off = 0;
    auto take = [&](std::size_t n) {
        char* p = base + off;
        off += (n + 255) / 256 * 256;
        return p;
    };
    std::vector<GammaJob> jobs(reqs.size());
    GammaJob* dj = reinterpret_cast<GammaJob*>(take(reqs.size() * sizeof(GammaJob)));
    for (std::size_t k = 0; k < reqs.size(); ++k) {
        const GammaRequest& r = reqs[k];
        GammaJob& j = jobs[k];
        j.C = r.C;
        j.N = r.N;
        j.dt = r.dt;
        j.nb = static_cast<int>(r.omegas.size());
        j.nchunks = static_cast<int>((r.N + GT_CHUNK - 1) / GT_CHUNK);
        j.G = r.G;
        double* dom = reinterpret_cast<double*>(take(r.omegas.size() * sizeof(double)));
        cuda_check(cudaMemcpyAsync(dom, r.omegas.data(), r.omegas.size() * sizeof(double), cudaMemcpyHostToDevice, st),
                   "gamma omegas");
        j.omegas = dom;
        j.partial = reinterpret_cast<double2*>(take(static_cast<std::size_t>(j.nb) * j.nchunks * sizeof(double2)));
    }
    cuda_check(cudaMemcpyAsync(dj, jobs.data(), jobs.size() * sizeof(GammaJob), cudaMemcpyHostToDevice, st), "gamma jobs");
    for (std::size_t k0 = 0; k0 < reqs.size(); k0 += 65535) {
        const unsigned nj = static_cast<unsigned>(std::min<std::size_t>(65535, reqs.size() - k0));
        const dim3 grid(static_cast<unsigned>(max_chunks), static_cast<unsigned>(max_nb), nj);
        k_gamma_reduce<<<grid, GT_THREADS, 0, st>>>(dj + k0);
        launched("k_gamma_reduce");
        k_gamma_scan<<<grid, GT_THREADS, 0, st>>>(dj + k0);
        launched("k_gamma_scan");
    }
    cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(gamma)");
}

void gamma_trapz_device(const double2* C, std::size_t N, double dt, const std::vector<double>& omegas, double2* G,
                        cudaStream_t st) {
    GammaRequest r;
    r.C = C;
    r.N = N;
    r.dt = dt;
    r.omegas = omegas;
    r.G = G;
    gamma_trapz_batch_device({r}, st);
}

}  // namespace taco
