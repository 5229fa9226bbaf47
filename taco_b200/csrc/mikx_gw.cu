// mikx_gw.cu -- the unfused MIKX -> GW -> L4 stages as separate device entry points.
//
// The production path never materialises M/I/K/X (the contraction kernel applies the
// merged linear map, contract.cuh).  These kernels serve callers of the reference's
// stage-by-stage API:
//   k_mikx      M, I, K (N^4) and X (N^6) gathered from F/C/R at one time
//               (cpp/src/tcl/tcl4_mikx.cpp:87-177; M uses F[f(j,q)][f(j,k)][f(p,j)]);
//   k_gw_raw    T(n,i,m,j) by the NAKZWAN sums (cpp/src/tcl/tcl4_assemble.cpp:98-186),
//               one thread per entry, fused multiply-adds in FP64;
//   k_gw_sym    GW = T + T^H (tcl4_assemble.cpp:188-200);
//   k_gw_to_l4  L4(n + N m, i + N j) = GW(n + N i, m + N j) (tcl4_assemble.cpp:204-230).
// All are batched over a leading time dimension.
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "engine.hpp"

namespace taco {

namespace {

__device__ __forceinline__ size_t f6(int N, int j, int k, int p, int q, int r, int s) {
    return static_cast<size_t>(j) +
           static_cast<size_t>(N) *
               (k + static_cast<size_t>(N) * (p + static_cast<size_t>(N) * (q + static_cast<size_t>(N) * (r + static_cast<size_t>(N) * s))));
}

__global__ void k_mikx(const double2* __restrict__ F, const double2* __restrict__ Cc, const double2* __restrict__ R,
                       const int* __restrict__ p2f, int N, int nf, double2* __restrict__ M, double2* __restrict__ I,
                       double2* __restrict__ K, double2* __restrict__ X) {
    const size_t nf3 = static_cast<size_t>(nf) * nf * nf;
    const size_t N2 = static_cast<size_t>(N) * N, N4 = N2 * N2, N6 = N4 * N2;
    const size_t t = blockIdx.y;
    const double2* Ft = F + t * nf3;
    const double2* Ct = Cc + t * nf3;
    const double2* Rt = R + t * nf3;
    auto f = [&](int a, int b) { return static_cast<size_t>(p2f[a + N * b]); };
    auto i3 = [&](size_t a, size_t b, size_t c) { return (a * nf + b) * nf + c; };
    for (size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; idx < N6;
         idx += static_cast<size_t>(gridDim.x) * blockDim.x) {
        // X(j,k,p,q,r,s) = C + R at [f(j,k), f(p,q), f(r,s)]
        size_t rem = idx;
        const int j = static_cast<int>(rem % N); rem /= N;
        const int k = static_cast<int>(rem % N); rem /= N;
        const int p = static_cast<int>(rem % N); rem /= N;
        const int q = static_cast<int>(rem % N); rem /= N;
        const int r = static_cast<int>(rem % N); rem /= N;
        const int s = static_cast<int>(rem);
        const size_t e = i3(f(j, k), f(p, q), f(r, s));
        X[t * N6 + idx] = cadd(Ct[e], Rt[e]);
        if (idx < N4) {
            // M, I, K entry (row (j,k) = j + N k, col (p,q) = p + N q), column-major N^2 x N^2
            const size_t row = idx % N2, col = idx / N2;
            const int jj = static_cast<int>(row % N), kk = static_cast<int>(row / N);
            const int pp = static_cast<int>(col % N), qq = static_cast<int>(col / N);
            M[t * N4 + idx] = csub(Ft[i3(f(jj, qq), f(jj, kk), f(pp, jj))], Rt[i3(f(jj, qq), f(pp, qq), f(qq, kk))]);
            I[t * N4 + idx] = Ft[i3(f(jj, kk), f(qq, pp), f(kk, qq))];
            K[t * N4 + idx] = Rt[i3(f(jj, kk), f(pp, qq), f(qq, jj))];
        }
    }
}

__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {  // c + a b
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}

__global__ void k_gw_raw(const double2* __restrict__ M, const double2* __restrict__ Ia, const double2* __restrict__ K,
                         const double2* __restrict__ X, const double2* __restrict__ ops, int N, int num_ops,
                         double2* __restrict__ T) {
    const size_t N2 = static_cast<size_t>(N) * N, N4 = N2 * N2, N6 = N4 * N2;
    const size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    const size_t tt = blockIdx.y;
    if (idx >= N4) return;
    const double2* Mt = M + tt * N4;
    const double2* It = Ia + tt * N4;
    const double2* Kt = K + tt * N4;
    const double2* Xt = X + tt * N6;
    const size_t row = idx % N2, col = idx / N2;
    const int n = static_cast<int>(row % N), i = static_cast<int>(row / N);
    const int m = static_cast<int>(col % N), j = static_cast<int>(col / N);
    auto mat = [&](const double2* P, int r1, int c1, int r2, int c2) {
        return P[(r1 + static_cast<size_t>(N) * c1) + N2 * (r2 + static_cast<size_t>(N) * c2)];
    };
    double2 res = make_double2(0.0, 0.0);
    for (int iA = 0; iA < num_ops; ++iA) {
        const double2* A = ops + static_cast<size_t>(iA) * N2;
        for (int iB = 0; iB < num_ops; ++iB) {
            const double2* B = ops + static_cast<size_t>(iB) * N2;
            auto a_ = [&](int r, int c) { return A[r + N * c]; };
            auto b_ = [&](int r, int c) { return B[r + N * c]; };
            for (int a = 0; a < N; ++a)
                for (int b = 0; b < N; ++b) {
                    // res -= (t1 - t2 + t3 + t4 - t5 - t6 + t7)
                    double2 acc = make_double2(0.0, 0.0);
                    acc = cfma(cmul(cmul(cmul(b_(n, a), a_(a, b)), b_(b, i)), a_(j, m)), mat(Mt, b, i, n, a), acc);
                    acc = cfma(cmul(cmul(cmul(a_(n, a), b_(a, b)), b_(b, i)), a_(j, m)), cscale(mat(It, a, n, i, b), -1.0), acc);
                    acc = cfma(cmul(cmul(cmul(b_(n, a), b_(a, b)), a_(b, i)), a_(j, m)), mat(Kt, i, b, n, a), acc);
                    acc = cfma(cmul(cmul(cmul(a_(n, a), b_(a, i)), b_(j, b)), a_(b, m)), Xt[f6(N, a, n, j, b, n, i)], acc);
                    acc = cfma(cmul(cmul(cmul(b_(n, a), a_(a, i)), b_(j, b)), a_(b, m)), cscale(Xt[f6(N, i, a, j, b, n, i)], -1.0), acc);
                    acc = cfma(cmul(cmul(cmul(a_(n, a), a_(a, b)), b_(b, i)), b_(j, m)), cscale(Xt[f6(N, b, a, j, m, a, i)], -1.0), acc);
                    acc = cfma(cmul(cmul(cmul(a_(n, a), b_(a, b)), a_(b, i)), b_(j, m)), Xt[f6(N, i, b, j, m, a, i)], acc);
                    res = csub(res, acc);
                }
            if (j == m) {
                for (int a = 0; a < N; ++a)
                    for (int b = 0; b < N; ++b)
                        for (int c = 0; c < N; ++c) {
                            double2 acc = make_double2(0.0, 0.0);
                            acc = cfma(cmul(cmul(cmul(a_(n, a), b_(a, b)), a_(b, c)), b_(c, i)), mat(Mt, c, i, a, b), acc);
                            acc = cfma(cmul(cmul(cmul(a_(n, a), b_(a, b)), b_(b, c)), a_(c, i)), mat(Kt, i, c, a, b), acc);
                            acc = cfma(cmul(cmul(cmul(a_(n, a), a_(a, b)), b_(b, c)), b_(c, i)), cscale(mat(It, b, a, i, c), -1.0), acc);
                            res = cadd(res, acc);
                        }
            }
        }
    }
    T[tt * N4 + idx] = res;
}

__global__ void k_gw_sym(const double2* __restrict__ T, int N, double2* __restrict__ GW) {
    const size_t N2 = static_cast<size_t>(N) * N, N4 = N2 * N2;
    const size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    const size_t tt = blockIdx.y;
    if (idx >= N4) return;
    const size_t r = idx % N2, c = idx / N2;
    // the upper triangle (r <= c) is T(r,c) + conj(T(c,r)); the lower its conjugate
    const size_t rr = r <= c ? r : c, cc = r <= c ? c : r;
    const double2 g = cadd(T[tt * N4 + rr + N2 * cc], cconj(T[tt * N4 + cc + N2 * rr]));
    GW[tt * N4 + idx] = r <= c ? g : cconj(g);
}

__global__ void k_gw_to_l4(const double2* __restrict__ GW, int N, double2* __restrict__ L4) {
    const size_t N2 = static_cast<size_t>(N) * N, N4 = N2 * N2;
    const size_t idx = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    const size_t tt = blockIdx.y;
    if (idx >= N4) return;
    const size_t rowL = idx % N2, colL = idx / N2;
    const size_t n = rowL % N, m = rowL / N, i = colL % N, j = colL / N;
    L4[tt * N4 + idx] = GW[tt * N4 + (n + N * i) + N2 * (m + N * j)];
}

unsigned grid_for(std::size_t n) { return static_cast<unsigned>(std::min<std::size_t>((n + 255) / 256, 65535)); }

}  // namespace

void mikx_device(const double2* F, const double2* C, const double2* R, const int* p2f_dev, int N, int nf, std::size_t T,
                 double2* M, double2* I, double2* K, double2* X, cudaStream_t st) {
    const std::size_t N6 = static_cast<std::size_t>(N) * N * N * N * N * N;
    for (std::size_t t0 = 0; t0 < T; t0 += 65535) {
        const unsigned nt = static_cast<unsigned>(std::min<std::size_t>(65535, T - t0));
        const std::size_t nf3 = static_cast<std::size_t>(nf) * nf * nf, N4 = static_cast<std::size_t>(N) * N * N * N;
        k_mikx<<<dim3(grid_for(N6), nt), 256, 0, st>>>(F + t0 * nf3, C + t0 * nf3, R + t0 * nf3, p2f_dev, N, nf,
                                                       M + t0 * N4, I + t0 * N4, K + t0 * N4, X + t0 * N6);
        launched("k_mikx");
    }
}

void gw_device(const double2* M, const double2* I, const double2* K, const double2* X, const double2* ops_dev, int N,
               int num_ops, std::size_t T, bool symmetrize, double2* GW, double2* tmp, cudaStream_t st) {
    const std::size_t N4 = static_cast<std::size_t>(N) * N * N * N, N6 = N4 * N * N;
    for (std::size_t t0 = 0; t0 < T; t0 += 65535) {
        const unsigned nt = static_cast<unsigned>(std::min<std::size_t>(65535, T - t0));
        double2* dst = symmetrize ? tmp + t0 * N4 : GW + t0 * N4;
        k_gw_raw<<<dim3(static_cast<unsigned>((N4 + 127) / 128), nt), 128, 0, st>>>(M + t0 * N4, I + t0 * N4, K + t0 * N4,
                                                                                   X + t0 * N6, ops_dev, N, num_ops, dst);
        launched("k_gw_raw");
        if (symmetrize) {
            k_gw_sym<<<dim3(static_cast<unsigned>((N4 + 255) / 256), nt), 256, 0, st>>>(dst, N, GW + t0 * N4);
            launched("k_gw_sym");
        }
    }
}

void gw_to_l4_device(const double2* GW, int N, std::size_t T, double2* L4, cudaStream_t st) {
    const std::size_t N4 = static_cast<std::size_t>(N) * N * N * N;
    for (std::size_t t0 = 0; t0 < T; t0 += 65535) {
        const unsigned nt = static_cast<unsigned>(std::min<std::size_t>(65535, T - t0));
        k_gw_to_l4<<<dim3(static_cast<unsigned>((N4 + 255) / 256), nt), 256, 0, st>>>(GW + t0 * N4, N, L4 + t0 * N4);
        launched("k_gw_to_l4");
    }
}

}  // namespace taco
