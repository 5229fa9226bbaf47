// taco_oracle.cpp -- CPU oracle (test infrastructure only) for the TCL4 L4(t) path.
//
// A plain C++17 + OpenMP restatement of the reference's CPU algorithm.  Each
// function names the reference file:line it follows.  This file is the checker
// for the CUDA product and the timed CPU baseline; the product never links it.
// See taco_oracle.h for the parity status and the memory layouts.

#include "taco_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cd = std::complex<double>;
constexpr double kPi = 3.141592653589793238462643383279502884;

thread_local std::string g_err;
std::size_t g_pad_factor = 0;  // tcl4_kernels.cpp:15 (process-global FFT pad factor)

inline cd* C(oc128* p) { return reinterpret_cast<cd*>(p); }
inline const cd* C(const oc128* p) { return reinterpret_cast<const cd*>(p); }

struct OracleError : std::runtime_error {
    int code;
    OracleError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

template <class Fn>
int guard(Fn&& fn) {
    try {
        fn();
        return ORACLE_OK;
    } catch (const OracleError& e) {
        g_err = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_err = e.what();
        return ORACLE_ERUNTIME;
    }
}

// correlation_fft.hpp:27-34
std::size_t next_pow2(std::size_t n) {
    if (n == 0) return 1;
    --n;
    for (std::size_t s = 1; s < sizeof(std::size_t) * 8; s <<= 1) n |= n >> s;
    return n + 1;
}

// In-place iterative radix-2 FFT with a per-stage twiddle recurrence
// (correlation_fft.hpp:38-73): forward uses exp(-2*pi*i*k*n/N); the inverse
// scales by 1/N.
void fft_radix2(std::vector<cd>& a, bool forward) {
    const std::size_t n = a.size();
    if (n == 0) return;
    if ((n & (n - 1)) != 0) throw OracleError(ORACLE_EINVAL, "fft: length must be a power of two");
    for (std::size_t i = 1, j = 0; i < n; ++i) {
        std::size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (std::size_t len = 2; len <= n; len <<= 1) {
        const double ang = (forward ? -2.0 : 2.0) * kPi / static_cast<double>(len);
        const cd step(std::cos(ang), std::sin(ang));
        const std::size_t half = len >> 1;
        for (std::size_t base = 0; base < n; base += len) {
            cd w(1.0, 0.0);
            for (std::size_t k = 0; k < half; ++k) {
                const cd u = a[base + k];
                const cd v = w * a[base + k + half];
                a[base + k] = u + v;
                a[base + k + half] = u - v;
                w *= step;
            }
        }
    }
    if (!forward) {
        const double s = 1.0 / static_cast<double>(n);
        for (auto& x : a) x *= s;
    }
}

// Nfft rule of tcl4_kernels.cpp:40-49.
std::size_t conv_length(std::size_t Nt) {
    const std::size_t L = 2 * Nt - 1;
    std::size_t target = L;
    if (g_pad_factor > 0) target = std::max(L, g_pad_factor * Nt);
    std::size_t n = next_pow2(target);
    return n < 2 ? 2 : n;
}

// tcl4_kernels.cpp:31-68 (causal linear convolution by zero-padded FFT, times dt).
void causal_conv_fft(const std::vector<cd>& f, const std::vector<cd>& g, double dt,
                     std::vector<cd>& out) {
    const std::size_t N = f.size();
    out.assign(N, cd(0.0, 0.0));
    if (N == 0) return;
    const std::size_t nfft = conv_length(N);
    std::vector<cd> A(nfft, cd(0.0, 0.0)), B(nfft, cd(0.0, 0.0));
    std::copy(f.begin(), f.end(), A.begin());
    std::copy(g.begin(), g.end(), B.begin());
    fft_radix2(A, true);
    fft_radix2(B, true);
    for (std::size_t k = 0; k < nfft; ++k) A[k] *= B[k];
    fft_radix2(A, false);
    for (std::size_t k = 0; k < N; ++k) out[k] = dt * A[k];
}

// tcl4_kernels.cpp:19-29 (inclusive left-Riemann prefix: out[k] = dt * sum_{m<=k} y[m]).
void prefix_int_left(const std::vector<cd>& y, double dt, std::vector<cd>& out) {
    out.resize(y.size());
    cd acc(0.0, 0.0);
    for (std::size_t k = 0; k < y.size(); ++k) {
        acc += y[k];
        out[k] = acc * dt;
    }
}

void phases(std::size_t Nt, double omega, double dt, std::vector<cd>& plus, std::vector<cd>& minus) {
    plus.resize(Nt);
    minus.resize(Nt);
    for (std::size_t k = 0; k < Nt; ++k) {
        const double tk = static_cast<double>(k) * dt;  // tcl4_kernels.cpp:116-120
        plus[k] = std::exp(cd(0.0, omega * tk));
        minus[k] = std::exp(cd(0.0, -omega * tk));
    }
}

// F by convolution: tcl4_kernels.cpp:105-127.
void F_conv(const cd* g1, const cd* g2, std::size_t Nt, double omega, double dt, cd* out) {
    std::vector<cd> pp, pm;
    phases(Nt, omega, dt, pp, pm);
    std::vector<cd> g1p(Nt), y(Nt), pre, conv;
    for (std::size_t k = 0; k < Nt; ++k) {
        g1p[k] = g1[k] * pm[k];
        y[k] = g2[k] * pp[k];
    }
    prefix_int_left(y, dt, pre);
    std::vector<cd> g2v(g2, g2 + Nt);
    causal_conv_fft(g1p, g2v, dt, conv);
    for (std::size_t k = 0; k < Nt; ++k) out[k] = g1p[k] * pre[k] - conv[k];
}

// C by convolution: tcl4_kernels.cpp:129-152.
void C_conv(const cd* g1, const cd* g2, std::size_t Nt, double omega, double dt, cd* out) {
    std::vector<cd> pp, pm;
    phases(Nt, omega, dt, pp, pm);
    std::vector<cd> g1p(Nt), g2c(Nt), y(Nt), pre, conv;
    for (std::size_t k = 0; k < Nt; ++k) {
        g1p[k] = g1[k] * pm[k];
        g2c[k] = std::conj(g2[k]);
        y[k] = g2c[k] * pp[k];
    }
    prefix_int_left(y, dt, pre);
    causal_conv_fft(g1p, g2c, dt, conv);
    for (std::size_t k = 0; k < Nt; ++k) out[k] = g1p[k] * pre[k] - conv[k];
}

// R by prefix integrals: tcl4_kernels.cpp:154-175.
void R_conv(const cd* g1, const cd* g2, std::size_t Nt, double omega, double dt, cd* out) {
    std::vector<cd> pp, pm;
    phases(Nt, omega, dt, pp, pm);
    std::vector<cd> y(Nt), yp(Nt), pre, preP;
    for (std::size_t k = 0; k < Nt; ++k) {
        y[k] = g2[k] * pm[k];
        yp[k] = (g1[k] * g2[k]) * pm[k];
    }
    prefix_int_left(y, dt, pre);
    prefix_int_left(yp, dt, preP);
    for (std::size_t k = 0; k < Nt; ++k) out[k] = g1[k] * pre[k] - preP[k];
}

// Direct O(Nt^2) forms: tcl4_kernels.cpp:188-281.
void F_direct(const cd* g1, const cd* g2, std::size_t Nt, double omega, double dt, cd* out) {
    std::vector<cd> pp, pm;
    phases(Nt, omega, dt, pp, pm);
    cd pre(0.0, 0.0);
    for (std::size_t k = 0; k < Nt; ++k) {
        pre += g2[k] * pp[k] * dt;
        const cd first = g1[k] * pre * pm[k];
        cd second(0.0, 0.0);
        for (std::size_t m = 0; m <= k; ++m) second += g1[k - m] * g2[m] * pm[k - m];
        out[k] = first - dt * second;
    }
}

void C_direct(const cd* g1, const cd* g2, std::size_t Nt, double omega, double dt, cd* out) {
    std::vector<cd> pp, pm;
    phases(Nt, omega, dt, pp, pm);
    cd pre(0.0, 0.0);
    for (std::size_t k = 0; k < Nt; ++k) {
        pre += std::conj(g2[k]) * pp[k] * dt;
        const cd first = g1[k] * pre * pm[k];
        cd second(0.0, 0.0);
        for (std::size_t m = 0; m <= k; ++m) second += g1[k - m] * std::conj(g2[m]) * pm[k - m];
        out[k] = first - dt * second;
    }
}

void R_direct(const cd* g1, const cd* g2, std::size_t Nt, double omega, double dt, cd* out) {
    std::vector<cd> pp, pm;
    phases(Nt, omega, dt, pp, pm);
    cd pre(0.0, 0.0), preP(0.0, 0.0);
    for (std::size_t k = 0; k < Nt; ++k) {
        pre += g2[k] * pm[k] * dt;
        const cd term1 = g1[k] * pre;
        preP += (g1[k] * g2[k]) * pm[k] * dt;
        out[k] = term1 - preP;
    }
}

inline std::size_t flat6(std::size_t N, int j, int k, int p, int q, int r, int s) {
    return static_cast<std::size_t>(j) +
           N * (static_cast<std::size_t>(k) +
           N * (static_cast<std::size_t>(p) +
           N * (static_cast<std::size_t>(q) +
           N * (static_cast<std::size_t>(r) + N * static_cast<std::size_t>(s)))));
}

// MIKX gathers at one time: tcl4_mikx.cpp:87-177 (M uses F[f(j,q)][f(j,k)][f(p,j)],
// the implementation/MATLAB form of matlab/MIKX.m:23-26).
void mikx_at(const cd* F, const cd* Cc, const cd* R, int nf, const int* p2f, int N,
             cd* M, cd* I, cd* K, cd* X) {
    const std::size_t n = static_cast<std::size_t>(N);
    const std::size_t N2 = n * n;
    auto f = [&](int a, int b) -> std::size_t {
        const int v = p2f[a + N * b];
        if (v < 0) throw OracleError(ORACLE_ERUNTIME, "mikx: pair_to_freq contains -1 for a required pair");
        return static_cast<std::size_t>(v);
    };
    auto idx3 = [&](std::size_t a, std::size_t b, std::size_t c) {
        return (a * static_cast<std::size_t>(nf) + b) * static_cast<std::size_t>(nf) + c;
    };
    for (std::size_t idx = 0; idx < N2 * N2; ++idx) {
        const std::size_t row = idx / N2, col = idx % N2;
        const int j = static_cast<int>(row % n), k = static_cast<int>(row / n);
        const int p = static_cast<int>(col % n), q = static_cast<int>(col / n);
        const std::size_t f_jk = f(j, k), f_jq = f(j, q), f_pj = f(p, j), f_pq = f(p, q);
        const std::size_t f_qk = f(q, k), f_kq = f(k, q), f_qp = f(q, p), f_qj = f(q, j);
        M[row + N2 * col] = F[idx3(f_jq, f_jk, f_pj)] - R[idx3(f_jq, f_pq, f_qk)];
        I[row + N2 * col] = F[idx3(f_jk, f_qp, f_kq)];
        K[row + N2 * col] = R[idx3(f_jk, f_pq, f_qj)];
        for (int r = 0; r < N; ++r)
            for (int s = 0; s < N; ++s) {
                const std::size_t f_rs = f(r, s);
                X[flat6(n, j, k, p, q, r, s)] = Cc[idx3(f_jk, f_pq, f_rs)] + R[idx3(f_jk, f_pq, f_rs)];
            }
    }
}

// NAKZWAN contraction + symmetrisation: tcl4_assemble.cpp:53-202 (matlab/NAKZWAN_v9.m:7-40).
void assemble_gw(const cd* M, const cd* Ia, const cd* K, const cd* X, const cd* ops, int num_ops,
                 int N, cd* GW, bool parallel) {
    const std::size_t n = static_cast<std::size_t>(N);
    const std::size_t N2 = n * n;
    auto f2 = [&](int r, int c) { return static_cast<std::size_t>(r) + n * static_cast<std::size_t>(c); };
    auto mat = [&](const cd* m, std::size_t r, std::size_t c) { return m[r + N2 * c]; };
    const std::ptrdiff_t total = static_cast<std::ptrdiff_t>(N2 * N2);
#ifdef _OPENMP
#pragma omp parallel for schedule(static) if (parallel && !omp_in_parallel())
#endif
    for (std::ptrdiff_t idx = 0; idx < total; ++idx) {
        const std::size_t row = static_cast<std::size_t>(idx) % N2;
        const std::size_t col = static_cast<std::size_t>(idx) / N2;
        const int nn = static_cast<int>(row % n), i = static_cast<int>(row / n);
        const int m = static_cast<int>(col % n), j = static_cast<int>(col / n);
        cd res(0.0, 0.0);
        for (int iA = 0; iA < num_ops; ++iA) {
            const cd* A = ops + static_cast<std::size_t>(iA) * N2;
            auto a_ = [&](int r, int c) { return A[f2(r, c)]; };
            for (int iB = 0; iB < num_ops; ++iB) {
                const cd* B = ops + static_cast<std::size_t>(iB) * N2;
                auto b_ = [&](int r, int c) { return B[f2(r, c)]; };
                for (int a = 0; a < N; ++a)
                    for (int b = 0; b < N; ++b) {
                        const cd M_bi_na = mat(M, f2(b, i), f2(nn, a));
                        const cd I_an_ib = mat(Ia, f2(a, nn), f2(i, b));
                        const cd K_ib_na = mat(K, f2(i, b), f2(nn, a));
                        const cd X1 = X[flat6(n, a, nn, j, b, nn, i)];
                        const cd X2 = X[flat6(n, i, a, j, b, nn, i)];
                        const cd X3 = X[flat6(n, b, a, j, m, a, i)];
                        const cd X4 = X[flat6(n, i, b, j, m, a, i)];
                        const cd t1 = b_(nn, a) * a_(a, b) * b_(b, i) * a_(j, m) * M_bi_na;
                        const cd t2 = a_(nn, a) * b_(a, b) * b_(b, i) * a_(j, m) * I_an_ib;
                        const cd t3 = b_(nn, a) * b_(a, b) * a_(b, i) * a_(j, m) * K_ib_na;
                        const cd t4 = a_(nn, a) * b_(a, i) * b_(j, b) * a_(b, m) * X1;
                        const cd t5 = b_(nn, a) * a_(a, i) * b_(j, b) * a_(b, m) * X2;
                        const cd t6 = a_(nn, a) * a_(a, b) * b_(b, i) * b_(j, m) * X3;
                        const cd t7 = a_(nn, a) * b_(a, b) * a_(b, i) * b_(j, m) * X4;
                        res -= (t1 - t2 + t3 + t4 - t5 - t6 + t7);
                    }
                if (j == m) {
                    for (int a = 0; a < N; ++a)
                        for (int b = 0; b < N; ++b)
                            for (int c = 0; c < N; ++c) {
                                const cd M_ci_ab = mat(M, f2(c, i), f2(a, b));
                                const cd K_ic_ab = mat(K, f2(i, c), f2(a, b));
                                const cd I_ba_ic = mat(Ia, f2(b, a), f2(i, c));
                                const cd add1 = a_(nn, a) * b_(a, b) * a_(b, c) * b_(c, i) * M_ci_ab;
                                const cd add2 = a_(nn, a) * b_(a, b) * b_(b, c) * a_(c, i) * K_ic_ab;
                                const cd add3 = -a_(nn, a) * a_(a, b) * b_(b, c) * b_(c, i) * I_ba_ic;
                                res += (add1 + add2 + add3);
                            }
                }
            }
        }
        GW[row + N2 * col] = res;
    }
    // GW <- T + T^H (tcl4_assemble.cpp:188-200)
    for (std::size_t c = 0; c < N2; ++c)
        for (std::size_t r = 0; r <= c; ++r) {
            const cd g = GW[r + N2 * c] + std::conj(GW[c + N2 * r]);
            GW[r + N2 * c] = g;
            if (r != c) GW[c + N2 * r] = std::conj(g);
        }
}

// tcl4_assemble.cpp:204-230: L4(n + N m, i + N j) = GW(n + N i, m + N j).
void gw_to_l4(const cd* GW, int N, cd* L4) {
    const std::size_t n = static_cast<std::size_t>(N), N2 = n * n;
    for (std::size_t a = 0; a < n; ++a)
        for (std::size_t m = 0; m < n; ++m)
            for (std::size_t i = 0; i < n; ++i)
                for (std::size_t j = 0; j < n; ++j)
                    L4[(a + n * m) + N2 * (i + n * j)] = GW[(a + n * i) + N2 * (m + n * j)];
}

double J_eval(int model, const double* p, double w) {
    if (!(w > 0.0)) return 0.0;
    double v = p[0] * w * std::exp(-w / p[1]);
    if (model == ORACLE_J_OHMIC_DRUDE) v += 2.0 * p[2] * p[3] * w / (w * w + p[3] * p[3]);
    return v;
}

// ---- Hermitian eigensolver (cyclic complex Jacobi) for the system builder ----
// The reference uses Eigen's SelfAdjointEigenSolver (system.hpp:37-52); eigenvalues
// ascending.  Eigenvector phases here: the largest-magnitude component of each
// column (first within 1e-9 relative) is made real and positive.
void jacobi_herm(int d, std::vector<cd>& A, std::vector<double>& eps, std::vector<cd>& V) {
    const std::size_t n = static_cast<std::size_t>(d);
    V.assign(n * n, cd(0.0, 0.0));
    for (std::size_t i = 0; i < n; ++i) V[i + n * i] = 1.0;
    auto at = [&](std::vector<cd>& m, std::size_t r, std::size_t c) -> cd& { return m[r + n * c]; };
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (std::size_t c = 0; c < n; ++c)
            for (std::size_t r = 0; r < n; ++r) {
                if (r != c) off += std::norm(at(A, r, c));
                else diag += std::norm(at(A, r, c));
            }
        if (off <= 1e-30 * std::max(diag, 1e-300)) break;
        for (std::size_t p = 0; p + 1 < n; ++p)
            for (std::size_t q = p + 1; q < n; ++q) {
                const cd z = at(A, p, q);
                const double az = std::abs(z);
                if (az == 0.0) continue;
                const cd ph = z / az;  // e^{i phi}
                const double a = at(A, p, p).real(), b = at(A, q, q).real();
                const double theta = (b - a) / (2.0 * az);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                // J = diag(1, conj(ph)) * [[c, s], [-s, c]] on (p, q)
                const cd Jpp = c, Jpq = s, Jqp = -s * std::conj(ph), Jqq = c * std::conj(ph);
                for (std::size_t k = 0; k < n; ++k) {  // A <- A J, V <- V J
                    const cd akp = at(A, k, p), akq = at(A, k, q);
                    at(A, k, p) = akp * Jpp + akq * Jqp;
                    at(A, k, q) = akp * Jpq + akq * Jqq;
                    const cd vkp = at(V, k, p), vkq = at(V, k, q);
                    at(V, k, p) = vkp * Jpp + vkq * Jqp;
                    at(V, k, q) = vkp * Jpq + vkq * Jqq;
                }
                for (std::size_t k = 0; k < n; ++k) {  // A <- J^H A
                    const cd apk = at(A, p, k), aqk = at(A, q, k);
                    at(A, p, k) = std::conj(Jpp) * apk + std::conj(Jqp) * aqk;
                    at(A, q, k) = std::conj(Jpq) * apk + std::conj(Jqq) * aqk;
                }
                at(A, p, q) = 0.0;
                at(A, q, p) = 0.0;
            }
    }
    std::vector<std::size_t> order(n);
    for (std::size_t i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](std::size_t x, std::size_t y) { return at(A, x, x).real() < at(A, y, y).real(); });
    eps.resize(n);
    std::vector<cd> W(n * n);
    for (std::size_t c = 0; c < n; ++c) {
        eps[c] = at(A, order[c], order[c]).real();
        double mx = 0.0;
        for (std::size_t r = 0; r < n; ++r) mx = std::max(mx, std::abs(at(V, r, order[c])));
        std::size_t piv = 0;
        for (std::size_t r = 0; r < n; ++r)
            if (std::abs(at(V, r, order[c])) >= mx * (1.0 - 1e-9)) { piv = r; break; }
        const cd v = at(V, piv, order[c]);
        const cd rot = std::conj(v) / std::abs(v);
        for (std::size_t r = 0; r < n; ++r) W[r + n * c] = at(V, r, order[c]) * rot;
    }
    V.swap(W);
}

}  // namespace

extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

size_t oracle_next_pow2(size_t n) { return next_pow2(n); }

int oracle_fft(oc128* a, size_t n, int forward) {
    return guard([&] {
        std::vector<cd> v(C(a), C(a) + n);
        fft_radix2(v, forward != 0);
        std::copy(v.begin(), v.end(), C(a));
    });
}

void oracle_set_fcr_fft_pad_factor(size_t f) { g_pad_factor = f; }
size_t oracle_get_fcr_fft_pad_factor(void) { return g_pad_factor; }

// correlation_fft.hpp:153-214 (KMS spectrum with the `KMS *= r` recurrence, DC and
// Nyquist half weights, forward FFT, scale domega/pi, N+1 samples).
int oracle_bcf_fft(size_t N, double dt, int model, const double* params, double beta,
                   double* t_out, oc128* C_out) {
    return guard([&] {
        if (!(dt > 0.0)) throw OracleError(ORACLE_EINVAL, "dt must be > 0");
        const std::size_t Nt = N + 1;
        std::size_t nfft = 2 * Nt;
        if ((nfft & (nfft - 1)) != 0) nfft = next_pow2(nfft);
        const double tf = dt * static_cast<double>(nfft);
        const double dw = 2.0 * kPi / tf;
        const double wny = kPi / dt;
        const std::size_t pos = nfft / 2 - 1;
        std::vector<cd> S(nfft, cd(0.0, 0.0));
        auto J = [&](double w) { return J_eval(model, params, w); };
        if (std::isinf(beta)) {
            for (std::size_t k = 1; k <= pos; ++k) S[k] = cd((kPi / 2.0) * J(dw * static_cast<double>(k)), 0.0);
            S[0] = 0.0;
            S[nfft / 2] = cd(0.25 * kPi * J(wny), 0.0);
        } else {
            const double r = std::exp(-beta * dw);
            double kms = r;
            for (std::size_t k = 1; k <= pos; ++k) {
                const double w = dw * static_cast<double>(k);
                const double sp = (kPi / 2.0) * J(w) / (1.0 - kms);
                S[k] = cd(sp, 0.0);
                S[nfft - k] = cd(sp * kms, 0.0);
                kms *= r;
            }
            S[0] = cd(0.5 * (kPi / 2.0) * J(dw) * (1.0 + r) / (1.0 - r), 0.0);
            const double eny = std::exp(beta * wny);
            S[nfft / 2] = cd(0.25 * kPi * J(wny) * (1.0 + 2.0 / (eny - 1.0)), 0.0);
        }
        fft_radix2(S, true);
        const double scale = dw / kPi;
        for (std::size_t k = 0; k < Nt; ++k) {
            t_out[k] = dt * static_cast<double>(k);
            C(C_out)[k] = S[k] * scale;
        }
    });
}

// gamma.hpp:166-213 (trapezoid prefix integrals with phase recurrence; G(0)=0).
int oracle_gamma_trapz(const oc128* Cin, size_t N, double dt, const double* omegas, size_t M,
                       oc128* G_out) {
    return guard([&] {
        if (N == 0 || M == 0 || !(dt > 0.0)) throw OracleError(ORACLE_EINVAL, "gamma_trapz: empty input");
        const cd* Cv = C(Cin);
        cd* G = C(G_out);
        const cd half(dt / 2.0, 0.0);
#ifdef _OPENMP
#pragma omp parallel for schedule(static) if (N * M >= 200000)
#endif
        for (std::ptrdiff_t jj = 0; jj < static_cast<std::ptrdiff_t>(M); ++jj) {
            const std::size_t j = static_cast<std::size_t>(jj);
            const cd step = std::exp(cd(0.0, omegas[j] * dt));
            cd phi(1.0, 0.0), acc(0.0, 0.0), prev = Cv[0];
            G[0 + N * j] = 0.0;
            for (std::size_t k = 1; k < N; ++k) {
                const cd nxt = phi * step;
                acc += half * (phi * prev + nxt * Cv[k]);
                G[k + N * j] = acc;
                phi = nxt;
                prev = Cv[k];
            }
        }
    });
}

// gamma.hpp:127-160 (rectangle prefix integrals).
int oracle_gamma_rect(const oc128* Cin, size_t N, double dt, const double* omegas, size_t M,
                      oc128* G_out) {
    return guard([&] {
        if (N == 0 || M == 0 || !(dt > 0.0)) throw OracleError(ORACLE_EINVAL, "gamma_rect: empty input");
        const cd* Cv = C(Cin);
        cd* G = C(G_out);
        for (std::size_t j = 0; j < M; ++j) {
            const cd step = std::exp(cd(0.0, omegas[j] * dt));
            cd phi(1.0, 0.0);
            cd acc = dt * phi * Cv[0];
            G[0 + N * j] = acc;
            for (std::size_t k = 1; k < N; ++k) {
                phi *= step;
                acc += dt * phi * Cv[k];
                G[k + N * j] = acc;
            }
        }
    });
}

// system.hpp:37-226: eigensystem, Bohr frequencies, buckets (tol grouping against the
// first-seen representative, row-major (m,n) scan, then sorted ascending), A_eig = U^H A U.
int oracle_system_build(const oc128* H, int d, const oc128* A_lab, int num_ops, double tol,
                        double* eps, oc128* U, int* nf_out, double* omegas, int* p2f,
                        oc128* A_eig) {
    return guard([&] {
        if (d <= 0) throw OracleError(ORACLE_EINVAL, "system_build: dimension must be > 0");
        const std::size_t n = static_cast<std::size_t>(d);
        std::vector<cd> A(C(H), C(H) + n * n), V;
        std::vector<double> ev;
        jacobi_herm(d, A, ev, V);
        for (std::size_t i = 0; i < n; ++i) eps[i] = ev[i];
        std::copy(V.begin(), V.end(), C(U));
        const double ftol = std::max(tol, std::numeric_limits<double>::epsilon());
        struct Bucket { double w; std::vector<std::pair<int, int>> pairs; };
        std::vector<Bucket> bk;
        for (int m = 0; m < d; ++m)
            for (int q = 0; q < d; ++q) {
                const double w = ev[m] - ev[q];
                std::size_t idx = bk.size();
                for (std::size_t b = 0; b < bk.size(); ++b)
                    if (std::abs(bk[b].w - w) <= ftol) { idx = b; break; }
                if (idx == bk.size()) bk.push_back(Bucket{w, {}});
                bk[idx].pairs.emplace_back(m, q);
            }
        std::sort(bk.begin(), bk.end(), [](const Bucket& a, const Bucket& b) { return a.w < b.w; });
        *nf_out = static_cast<int>(bk.size());
        for (std::size_t b = 0; b < bk.size(); ++b) {
            omegas[b] = bk[b].w;
            for (auto& pr : bk[b].pairs) p2f[pr.first + d * pr.second] = static_cast<int>(b);
        }
        for (int op = 0; op < num_ops; ++op) {
            const cd* Al = C(A_lab) + static_cast<std::size_t>(op) * n * n;
            cd* Ae = C(A_eig) + static_cast<std::size_t>(op) * n * n;
            for (std::size_t r = 0; r < n; ++r)
                for (std::size_t c = 0; c < n; ++c) {
                    cd acc(0.0, 0.0);
                    for (std::size_t a = 0; a < n; ++a)
                        for (std::size_t b = 0; b < n; ++b)
                            acc += std::conj(V[a + n * r]) * Al[a + n * b] * V[b + n * c];
                    Ae[r + n * c] = acc;
                }
        }
    });
}

// tcl4.cpp:40-101 (mirror: closest bucket to -w, self when |w| <= max(1e-12, tol)).
int oracle_build_map(const double* omegas, int nf, double tol, int* mirror, int* zero_index) {
    return guard([&] {
        const double t = std::max(1e-12, tol);
        int zero = -1;
        for (int b = 0; b < nf; ++b) {
            const double w = omegas[b];
            int best = -1;
            if (std::abs(w) <= t) {
                best = b;
                if (zero < 0) zero = b;
            } else {
                double best_abs = std::numeric_limits<double>::infinity();
                for (int bp = 0; bp < nf; ++bp) {
                    const double dw = std::abs(omegas[bp] + w);
                    if (dw < best_abs) { best_abs = dw; best = bp; }
                }
            }
            mirror[b] = best;
        }
        if (zero < 0) {
            double best_abs = std::numeric_limits<double>::infinity();
            for (int b = 0; b < nf; ++b)
                if (std::abs(omegas[b]) < best_abs) { best_abs = std::abs(omegas[b]); zero = b; }
            if (zero < 0) zero = 0;
        }
        if (zero_index) *zero_index = zero;
    });
}

// tcl4.cpp:103-183: for all (i,j,k), omega = w_i + w_j + w_k; F uses g2 = gamma[:, mirror j],
// C and R use gamma[:, j]; OpenMP over the nf^2 (i,j) pairs.
int oracle_fcr_series(const oc128* gamma, size_t Nt, int nf, const double* omegas,
                      const int* mirror, double dt, int method,
                      oc128* F, oc128* Cc, oc128* R) {
    return guard([&] {
        if (nf <= 0 || Nt == 0) throw OracleError(ORACLE_EINVAL, "fcr_series: empty gamma");
        const cd* g = C(gamma);
        const std::ptrdiff_t total = static_cast<std::ptrdiff_t>(nf) * nf;
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
        for (std::ptrdiff_t idx = 0; idx < total; ++idx) {
            const int i = static_cast<int>(idx / nf), j = static_cast<int>(idx % nf);
            const int jm = mirror[j] >= 0 ? mirror[j] : j;
            const cd* g1 = g + Nt * static_cast<std::size_t>(i);
            const cd* g2 = g + Nt * static_cast<std::size_t>(j);
            const cd* g2m = g + Nt * static_cast<std::size_t>(jm);
            for (int k = 0; k < nf; ++k) {
                const double w = omegas[i] + omegas[j] + omegas[k];
                const std::size_t o = (static_cast<std::size_t>(i * nf + j) * nf + k) * Nt;
                if (method == ORACLE_FCR_DIRECT) {
                    F_direct(g1, g2m, Nt, w, dt, C(F) + o);
                    C_direct(g1, g2, Nt, w, dt, C(Cc) + o);
                    R_direct(g1, g2, Nt, w, dt, C(R) + o);
                } else {
                    F_conv(g1, g2m, Nt, w, dt, C(F) + o);
                    C_conv(g1, g2, Nt, w, dt, C(Cc) + o);
                    R_conv(g1, g2, Nt, w, dt, C(R) + o);
                }
            }
        }
    });
}

int oracle_mikx(const oc128* Ft, const oc128* Ct, const oc128* Rt, int nf, const int* p2f, int N,
                oc128* M, oc128* I, oc128* K, oc128* X) {
    return guard([&] {
        if (N <= 0) throw OracleError(ORACLE_EINVAL, "mikx: N must be > 0");
        mikx_at(C(Ft), C(Ct), C(Rt), nf, p2f, N, C(M), C(I), C(K), C(X));
    });
}

int oracle_assemble_gw(const oc128* M, const oc128* I, const oc128* K, const oc128* X,
                       const oc128* ops, int num_ops, int N, oc128* GW) {
    return guard([&] {
        if (N <= 0) throw OracleError(ORACLE_EINVAL, "assemble: N must be > 0");
        if (num_ops <= 0) throw OracleError(ORACLE_EINVAL, "assemble: coupling_ops must be non-empty");
        assemble_gw(C(M), C(I), C(K), C(X), C(ops), num_ops, N, C(GW), true);
    });
}

int oracle_gw_to_l4(const oc128* GW, int N, oc128* L4) {
    return guard([&] {
        if (N <= 0) throw OracleError(ORACLE_EINVAL, "gw_to_liouvillian: N must be > 0");
        gw_to_l4(C(GW), N, C(L4));
    });
}

// compute_triple_kernels (tcl4.cpp:103-183), then per requested time the
// MIKX -> GW -> L4 chain (tcl4.cpp:322-358), OpenMP over time indices as in
// build_correction_series and the MPI+OpenMP batch (tcl4_mpi_omp.cpp:238-248).
int oracle_tcl4_build_batch(int N, int nf, const double* omegas, const int* mirror,
                            const int* p2f, const oc128* ops, int num_ops,
                            const oc128* gamma, size_t Nt, double dt,
                            const uint32_t* tidx, size_t T, int method,
                            oc128* L4_out, double* fcr_ms, double* per_t_ms) {
    return guard([&] {
        if (N <= 0 || nf <= 0 || Nt == 0) throw OracleError(ORACLE_EINVAL, "tcl4_build_batch: empty input");
        if (num_ops <= 0) throw OracleError(ORACLE_EINVAL, "tcl4_build_batch: coupling_ops must be non-empty");
        std::vector<uint32_t> tids;
        if (T == 0) {
            tids.resize(Nt);
            for (std::size_t t = 0; t < Nt; ++t) tids[t] = static_cast<uint32_t>(t);
        } else {
            tids.assign(tidx, tidx + T);
        }
        for (auto t : tids)
            if (t >= Nt) throw OracleError(ORACLE_ERANGE, "tcl4_build_batch: time_index out of range");
        for (int a = 0; a < N * N; ++a)
            if (p2f[a] < 0) throw OracleError(ORACLE_ERUNTIME, "tcl4_build_batch: pair_to_freq contains -1");
        const std::size_t nf3 = static_cast<std::size_t>(nf) * nf * nf;
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<cd> F(nf3 * Nt), Cc(nf3 * Nt), R(nf3 * Nt);
        {
            const int rc = oracle_fcr_series(gamma, Nt, nf, omegas, mirror, dt, method,
                                             reinterpret_cast<oc128*>(F.data()),
                                             reinterpret_cast<oc128*>(Cc.data()),
                                             reinterpret_cast<oc128*>(R.data()));
            if (rc != ORACLE_OK) throw OracleError(rc, g_err);
        }
        const auto t1 = std::chrono::steady_clock::now();
        const std::size_t n = static_cast<std::size_t>(N), N2 = n * n, N4 = N2 * N2, N6 = N4 * N2;
        const std::ptrdiff_t nt = static_cast<std::ptrdiff_t>(tids.size());
        bool failed = false;
        std::string msg;
#ifdef _OPENMP
#pragma omp parallel
#endif
        {
            std::vector<cd> Ft(nf3), Ct(nf3), Rt(nf3), M(N4), I(N4), K(N4), X(N6), GW(N4);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
            for (std::ptrdiff_t o = 0; o < nt; ++o) {
                const std::size_t t = tids[static_cast<std::size_t>(o)];
                for (std::size_t e = 0; e < nf3; ++e) {
                    Ft[e] = F[e * Nt + t];
                    Ct[e] = Cc[e * Nt + t];
                    Rt[e] = R[e * Nt + t];
                }
                try {
                    mikx_at(Ft.data(), Ct.data(), Rt.data(), nf, p2f, N, M.data(), I.data(), K.data(), X.data());
                    assemble_gw(M.data(), I.data(), K.data(), X.data(), C(ops), num_ops, N, GW.data(), false);
                    gw_to_l4(GW.data(), N, C(L4_out) + static_cast<std::size_t>(o) * N4);
                } catch (const std::exception& e) {
#ifdef _OPENMP
#pragma omp critical
#endif
                    { failed = true; msg = e.what(); }
                }
            }
        }
        if (failed) throw OracleError(ORACLE_ERUNTIME, msg);
        const auto t2 = std::chrono::steady_clock::now();
        if (fcr_ms) *fcr_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        if (per_t_ms) *per_t_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
    });
}

// generator.cpp:81-90: -i (kron(I, H) - kron(H^T, I)).
int oracle_unitary_superop(int N, const oc128* H_eff, oc128* L_out) {
    return guard([&] {
        const std::size_t n = static_cast<std::size_t>(N), D = n * n;
        const cd* H = C(H_eff);
        cd* L = C(L_out);
        for (std::size_t k = 0; k < D * D; ++k) L[k] = 0.0;
        // kron(A,B)(r1*n + r2, c1*n + c2) = A(r1,c1) B(r2,c2); column-major storage.
        for (std::size_t r1 = 0; r1 < n; ++r1)
            for (std::size_t c1 = 0; c1 < n; ++c1)
                for (std::size_t r2 = 0; r2 < n; ++r2)
                    for (std::size_t c2 = 0; c2 < n; ++c2) {
                        const std::size_t row = r1 * n + r2, col = c1 * n + c2;
                        cd left = (r1 == c1) ? H[r2 + n * c2] : cd(0.0, 0.0);   // kron(I, H)
                        cd right = (r2 == c2) ? H[c1 + n * r1] : cd(0.0, 0.0);  // kron(H^T, I)
                        L[row + D * col] += cd(0.0, -1.0) * (left - right);
                    }
    });
}

// generator.cpp:92-177 with the spin-boson example's kernel fill
// (TCL4_spin_boson_example.cpp:303-315: Gamma(a,a) = gamma_b for every channel a).
int oracle_tcl2_total(int N, int nf, const double* eps, const int* p2f,
                      const oc128* A_eig, int num_ops, const oc128* gamma_b,
                      oc128* L_out, oc128* H_ls_out) {
    return guard([&] {
        const std::size_t n = static_cast<std::size_t>(N), D = n * n;
        std::vector<cd> Ldiss(D * D, cd(0.0, 0.0)), Hls(n * n, cd(0.0, 0.0));
        auto kron_add = [&](const std::vector<cd>& A, const std::vector<cd>& B, cd s) {
            for (std::size_t r1 = 0; r1 < n; ++r1)
                for (std::size_t c1 = 0; c1 < n; ++c1) {
                    const cd a = A[r1 + n * c1];
                    if (a == cd(0.0, 0.0)) continue;
                    for (std::size_t r2 = 0; r2 < n; ++r2)
                        for (std::size_t c2 = 0; c2 < n; ++c2)
                            Ldiss[(r1 * n + r2) + D * (c1 * n + c2)] += s * a * B[r2 + n * c2];
                }
        };
        std::vector<cd> I(n * n, cd(0.0, 0.0));
        for (std::size_t i = 0; i < n; ++i) I[i + n * i] = 1.0;
        for (int b = 0; b < nf; ++b) {
            for (int al = 0; al < num_ops; ++al) {
                // A_alpha(w_b): entries of A_eig on pairs in bucket b (system.hpp:163-182).
                std::vector<cd> Aw(n * n, cd(0.0, 0.0));
                const cd* Ae = C(A_eig) + static_cast<std::size_t>(al) * n * n;
                double nrm = 0.0;
                for (std::size_t c = 0; c < n; ++c)
                    for (std::size_t r = 0; r < n; ++r)
                        if (p2f[r + n * c] == b) { Aw[r + n * c] = Ae[r + n * c]; nrm += std::norm(Ae[r + n * c]); }
                if (nrm == 0.0) continue;
                const int be = al;  // diagonal-in-channel fill: Gamma(alpha, beta) = 0 for alpha != beta
                (void)be;
                const cd G = C(gamma_b)[b];
                const double gam = 2.0 * G.real();
                const double S = G.imag();
                std::vector<cd> AdA(n * n, cd(0.0, 0.0)), Aconj(n * n), AdAT(n * n);
                for (std::size_t r = 0; r < n; ++r)
                    for (std::size_t c = 0; c < n; ++c) {
                        cd acc(0.0, 0.0);
                        for (std::size_t k = 0; k < n; ++k) acc += std::conj(Aw[k + n * r]) * Aw[k + n * c];
                        AdA[r + n * c] = acc;
                    }
                double an = 0.0;
                for (auto& v : AdA) an += std::norm(v);
                if (an == 0.0) continue;
                const bool need_jump = std::abs(gam) > 0.0;
                const bool need_ls = std::abs(S) > 0.0;
                if (need_ls)
                    for (std::size_t k = 0; k < n * n; ++k) Hls[k] += S * AdA[k];
                if (!need_jump) continue;
                for (std::size_t r = 0; r < n; ++r)
                    for (std::size_t c = 0; c < n; ++c) {
                        Aconj[r + n * c] = std::conj(Aw[r + n * c]);
                        AdAT[r + n * c] = AdA[c + n * r];
                    }
                kron_add(Aconj, Aw, gam);
                kron_add(I, AdA, -0.5 * gam);
                kron_add(AdAT, I, -0.5 * gam);
            }
        }
        // hermitize(H_ls) (ops.hpp:234)
        std::vector<cd> Hh(n * n);
        for (std::size_t r = 0; r < n; ++r)
            for (std::size_t c = 0; c < n; ++c) Hh[r + n * c] = 0.5 * (Hls[r + n * c] + std::conj(Hls[c + n * r]));
        std::vector<cd> Heff(Hh);
        for (std::size_t i = 0; i < n; ++i) Heff[i + n * i] += eps[i];
        std::vector<cd> Lu(D * D);
        const int rc = oracle_unitary_superop(N, reinterpret_cast<const oc128*>(Heff.data()),
                                              reinterpret_cast<oc128*>(Lu.data()));
        if (rc != ORACLE_OK) throw OracleError(rc, g_err);
        for (std::size_t k = 0; k < D * D; ++k) C(L_out)[k] = Lu[k] + Ldiss[k];
        if (H_ls_out) std::copy(Hh.begin(), Hh.end(), C(H_ls_out));
    });
}

namespace {
void matvec(const cd* L, const cd* x, cd* y, std::size_t D) {
    for (std::size_t i = 0; i < D; ++i) {
        cd s(0.0, 0.0);
        for (std::size_t j = 0; j < D; ++j) s += L[i + D * j] * x[j];
        y[i] = s;
    }
}
// rk4_dense.cpp:133-160.
void rk4_step(const cd* L0, const cd* Lh, const cd* L1, cd* r, std::size_t D, double dt,
              std::vector<cd>& k1, std::vector<cd>& k2, std::vector<cd>& k3, std::vector<cd>& k4,
              std::vector<cd>& tmp) {
    matvec(L0, r, k1.data(), D);
    for (std::size_t i = 0; i < D; ++i) tmp[i] = r[i] + 0.5 * dt * k1[i];
    matvec(Lh, tmp.data(), k2.data(), D);
    for (std::size_t i = 0; i < D; ++i) tmp[i] = r[i] + 0.5 * dt * k2[i];
    matvec(Lh, tmp.data(), k3.data(), D);
    for (std::size_t i = 0; i < D; ++i) tmp[i] = r[i] + dt * k3[i];
    matvec(L1, tmp.data(), k4.data(), D);
    for (std::size_t i = 0; i < D; ++i) r[i] += (dt / 6.0) * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
}
}  // namespace

int oracle_rk4_update(const oc128* L0, const oc128* Lh, const oc128* L1, int D, oc128* r, double dt) {
    return guard([&] {
        if (!(dt > 0.0)) throw OracleError(ORACLE_EINVAL, "rk4_update: dt must be > 0");
        const std::size_t n = static_cast<std::size_t>(D);
        std::vector<cd> k1(n), k2(n), k3(n), k4(n), tmp(n);
        rk4_step(C(L0), C(Lh), C(L1), C(r), n, dt, k1, k2, k3, k4, tmp);
    });
}

// rk4_dense.cpp:246-321 (endpoint overload averages neighbours for the midpoint).
int oracle_rk4_propagate(const oc128* L_series, const oc128* L_half, size_t steps, int D,
                         double dt, oc128* r, size_t sample_every, oc128* samples,
                         size_t* n_samples_out) {
    return guard([&] {
        if (!(dt > 0.0)) throw OracleError(ORACLE_EINVAL, "propagate_rk4_dense: dt must be > 0");
        if (sample_every == 0) throw OracleError(ORACLE_EINVAL, "propagate_rk4_dense: sample_every must be > 0");
        if (steps < 1) throw OracleError(ORACLE_EINVAL, "propagate_rk4_dense: L_series must have at least 2 matrices (endpoints)");
        const std::size_t n = static_cast<std::size_t>(D), DD = n * n;
        std::vector<cd> k1(n), k2(n), k3(n), k4(n), tmp(n), Lh(DD);
        std::size_t ns = 0;
        for (std::size_t i = 0; i < steps; ++i) {
            if (samples && (i % sample_every == 0)) std::copy(C(r), C(r) + n, C(samples) + (ns++) * n);
            const cd* L0 = C(L_series) + i * DD;
            const cd* L1 = C(L_series) + (i + 1) * DD;
            const cd* Lhp;
            if (L_half) {
                Lhp = C(L_half) + i * DD;
            } else {
                for (std::size_t k = 0; k < DD; ++k) Lh[k] = 0.5 * (L0[k] + L1[k]);
                Lhp = Lh.data();
            }
            rk4_step(L0, Lhp, L1, C(r), n, dt, k1, k2, k3, k4, tmp);
        }
        if (samples) std::copy(C(r), C(r) + n, C(samples) + (ns++) * n);
        if (n_samples_out) *n_samples_out = ns;
    });
}

// rk4_dense.cpp:222-244 (constant L; loop while t + dt/2 <= tf + 1e-15).
int oracle_rk4_propagate_const(const oc128* L, int D, double t0, double tf, double dt, oc128* r) {
    return guard([&] {
        if (!(dt > 0.0)) throw OracleError(ORACLE_EINVAL, "propagate_rk4_dense: dt must be > 0");
        const std::size_t n = static_cast<std::size_t>(D);
        std::vector<cd> k1(n), k2(n), k3(n), k4(n), tmp(n);
        double t = t0;
        while (t + 0.5 * dt <= tf + 1e-15) {
            rk4_step(C(L), C(L), C(L), C(r), n, dt, k1, k2, k3, k4, tmp);
            t += dt;
        }
    });
}

}  // extern "C"
