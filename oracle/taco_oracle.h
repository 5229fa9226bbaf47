/*
 * taco_oracle.h -- CPU oracle for the TCL4 L4(t) path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain C++17 + OpenMP restatement
 * of the reference's CPU algorithm for the fourth-order TCL generator.  It is the
 * checker for the CUDA product path and the timed CPU baseline: only the test
 * suite, the smoke check and the CPU-baseline leg of the benchmark load it.  The
 * product library (libtaco_b200.so) never links or calls it.
 *
 * Parity status: the reference cannot be compiled here (every hot-path
 * translation unit needs Eigen 3.4, which is absent).  The oracle is pinned by
 *   - the reference's known-answer tests restated as pytest cases
 *     (MIKX gather formulas: cpp/tests/tcl4_mikx_tests.cpp:49-160 with the M
 *     expectation taken from the implementation and matlab/MIKX.m:23-26;
 *     RK4 analytic cases: tests/rk4_dense_tests.cpp:43-101;
 *     Gamma analytic case: tests/gamma_tests.cpp:22-81;
 *     Direct-vs-Convolution F/C/R: tests/tcl4_tests.cpp:177-234), and
 *   - golden vectors produced by an independent numpy restatement of the MATLAB
 *     specification (matlab/tcl4_kernels.m, matlab/MIKX.m, matlab/NAKZWAN_v9.m),
 *     committed under tests/golden/ with the script that made them.
 * No output of the reference binary itself pins it; eigenvector phases are
 * solver dependent and are therefore never compared elementwise (the same
 * eigenbasis operators feed both sides of every parity test).
 *
 * Layouts (all complex values are interleaved double pairs, column-major):
 *   gamma  [Nt x nf]          gamma[t + Nt*b]            (tcl4_fcr_kernels_cuda.hpp:15-16)
 *   F/C/R  [nf^3][Nt]         series[(idx3)*Nt + t], idx3 = (i*nf + j)*nf + k
 *   pair_to_freq [N x N] int  p2f[a + N*b]
 *   ops    [num_ops][N x N]   ops[op*N*N + r + N*c]      (eigenbasis coupling operators)
 *   M,I,K  [N^2 x N^2]        row (j,k) = j + N*k, col (p,q) = p + N*q
 *   X      [N^6]              flat6(j,k,p,q,r,s) = j + N*(k + N*(p + N*(q + N*(r + N*s))))
 *   GW     [N^2 x N^2]        row (n,i) = n + N*i, col (m,j) = m + N*j
 *   L4     [N^2 x N^2]        row (n,m) = n + N*m, col (i,j) = i + N*j
 */
#ifndef TACO_ORACLE_H
#define TACO_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double re, im; } oc128;

enum { ORACLE_OK = 0, ORACLE_EINVAL = 1, ORACLE_ERANGE = 2, ORACLE_ERUNTIME = 3 };
enum { ORACLE_FCR_CONVOLUTION = 0, ORACLE_FCR_DIRECT = 1 };
/* Spectral density models J(w) for the bath correlation function. */
enum { ORACLE_J_OHMIC = 0,            /* params: alpha, omega_c            -> alpha*w*exp(-w/wc), w>0 */
       ORACLE_J_OHMIC_DRUDE = 1 };    /* params: alpha, wc, lambda, gamma  -> ohmic + 2*l*g*w/(w^2+g^2), w>0 */

const char* oracle_last_error(void);
int oracle_max_threads(void);
void oracle_set_threads(int n);

size_t oracle_next_pow2(size_t n);
int oracle_fft(oc128* a, size_t n, int forward);

void oracle_set_fcr_fft_pad_factor(size_t f);
size_t oracle_get_fcr_fft_pad_factor(void);

int oracle_bcf_fft(size_t N, double dt, int model, const double* params, double beta,
                   double* t_out, oc128* C_out /* N+1 */);
int oracle_gamma_trapz(const oc128* C, size_t N, double dt, const double* omegas, size_t M,
                       oc128* G_out /* N x M col-major */);
int oracle_gamma_rect(const oc128* C, size_t N, double dt, const double* omegas, size_t M,
                      oc128* G_out);

/* Hermitian eigensystem + Bohr buckets + eigenbasis operators.
 * Outputs sized for the worst case: omegas[d*d], p2f[d*d], A_eig[num_ops*d*d]. */
int oracle_system_build(const oc128* H, int d, const oc128* A_lab, int num_ops, double tol,
                        double* eps, oc128* U, int* nf_out, double* omegas, int* p2f,
                        oc128* A_eig);
int oracle_build_map(const double* omegas, int nf, double tol, int* mirror, int* zero_index);

int oracle_fcr_series(const oc128* gamma, size_t Nt, int nf, const double* omegas,
                      const int* mirror, double dt, int method,
                      oc128* F, oc128* C, oc128* R /* each [nf^3][Nt] */);
int oracle_mikx(const oc128* Ft, const oc128* Ct, const oc128* Rt, int nf,
                const int* p2f, int N, oc128* M, oc128* I, oc128* K, oc128* X);
int oracle_assemble_gw(const oc128* M, const oc128* I, const oc128* K, const oc128* X,
                       const oc128* ops, int num_ops, int N, oc128* GW);
int oracle_gw_to_l4(const oc128* GW, int N, oc128* L4);

/* Full L4 builds at the requested time indices (T == 0 means all Nt).
 * fcr_ms / per_t_ms receive the wall time of the two stages (may be NULL). */
int oracle_tcl4_build_batch(int N, int nf, const double* omegas, const int* mirror,
                            const int* p2f, const oc128* ops, int num_ops,
                            const oc128* gamma, size_t Nt, double dt,
                            const uint32_t* tidx, size_t T, int method,
                            oc128* L4_out, double* fcr_ms, double* per_t_ms);

/* TCL2 generator total() = -i[diag(eps)+H_LS, .] + D2 with the diagonal-in-channel
 * kernel fill of the spin-boson example (gamma_b given per bucket at one time). */
int oracle_tcl2_total(int N, int nf, const double* eps, const int* p2f,
                      const oc128* A_eig, int num_ops, const oc128* gamma_b,
                      oc128* L_out, oc128* H_ls_out /* nullable */);
int oracle_unitary_superop(int N, const oc128* H_eff, oc128* L_out);

int oracle_rk4_update(const oc128* L0, const oc128* Lh, const oc128* L1, int D,
                      oc128* r, double dt);
/* steps+1 endpoint generators; Lhalf may be NULL (midpoints by averaging).
 * samples (nullable) receives r after every sample_every steps, plus the final state:
 * row s = state at step s*sample_every, last row = final. n_samples_out gets the count. */
int oracle_rk4_propagate(const oc128* L_series, const oc128* L_half, size_t steps, int D,
                         double dt, oc128* r, size_t sample_every, oc128* samples,
                         size_t* n_samples_out);
int oracle_rk4_propagate_const(const oc128* L, int D, double t0, double tf, double dt,
                               oc128* r);

#ifdef __cplusplus
}
#endif
#endif
