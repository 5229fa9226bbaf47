"""Generate the golden fixtures that pin the CPU oracle and the CUDA path.

The expected values here come from an independent numpy restatement of the
reference's MATLAB specification, written without the C++ oracle:

* F/C/R kernels: matlab/tcl4_kernels.m:38-57 (prefix_int_left = dt*cumsum,
  Volterra part = dt * ifft(fft(f, L) * fft(g, L))[:N] with L = 2N-1, numpy FFT),
  with the Gamma-column choice of the C++ driver (cpp/src/tcl/tcl4.cpp:163-178:
  F pairs gamma[:, i] with gamma[:, mirror(j)], C and R with gamma[:, j]).
* MIKX: matlab/MIKX.m:17-50, literally, with np.tensordot in place of MATLAB's
  tensorprod (identical dimension semantics) and np.transpose for permute.
* NAKZWAN: matlab/NAKZWAN_v9.m:1-41, literal loops, T reshaped column-major,
  GW = T + T'.
* L4 reshuffle: cpp/src/tcl/tcl4_assemble.cpp:204-230.
* Bath correlation: cpp/include/taco/correlation_fft.hpp:153-214 (numpy FFT for
  the forward transform); Gamma: cpp/include/taco/gamma.hpp:166-213.
* TCL2: cpp/src/tcl/generator.cpp:81-177; RK4: cpp/src/core/rk4_dense.cpp:133-160.

Fixtures (small, complex128, stored with np.savez_compressed):
  mikx_makeval.npz     cpp/tests/tcl4_mikx_tests.cpp:53-87 + tests/tcl4_tests.cpp:40-90 inputs
  synthetic_gamma.npz  tests/tcl4_mpi_omp_tests.cpp:37-55 inputs (Nt=16, tids {0, 8, 15})
  spin_boson_small.npz d=2 spin-boson, Ohmic bath, Nt=257, end to end incl. TCL2 + RK4

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

SX = np.array([[0, 1], [1, 0]], np.complex128)
SZ = np.array([[1, 0], [0, -1]], np.complex128)


# ----------------------------------------------------------------- system ---
def eig_system(H, A_list, tol=1e-9):
    """Eigenbasis, Bohr buckets (system.hpp:137-157) and A_eig = U^H A U.

    Phase convention (shared with the oracle): the largest-magnitude component
    of each eigenvector (first within 1e-9 relative) is real and positive.
    """
    w, U = np.linalg.eigh(H)
    for c in range(U.shape[1]):
        mags = np.abs(U[:, c])
        piv = int(np.nonzero(mags >= mags.max() * (1 - 1e-9))[0][0])
        U[:, c] *= np.conj(U[piv, c]) / abs(U[piv, c])
    d = H.shape[0]
    reps, pairs = [], []
    for m in range(d):
        for n in range(d):
            x = w[m] - w[n]
            for b, r in enumerate(reps):
                if abs(r - x) <= tol:
                    pairs[b].append((m, n))
                    break
            else:
                reps.append(x)
                pairs.append([(m, n)])
    order = np.argsort(np.array(reps), kind="stable")
    omegas = np.array(reps)[order]
    p2f = -np.ones((d, d), np.int32)
    for nb, ob in enumerate(order):
        for (m, n) in pairs[ob]:
            p2f[m, n] = nb
    A_eig = [U.conj().T @ A @ U for A in A_list]
    return w, U, omegas, p2f, A_eig


def mirror_map(omegas, tol=1e-9):
    t = max(1e-12, tol)
    mir = np.zeros(len(omegas), np.int32)
    for b, w in enumerate(omegas):
        mir[b] = b if abs(w) <= t else int(np.argmin(np.abs(omegas + w)))
    return mir


# ---------------------------------------------------------------- kernels ---
def tcl4_kernels_scalar(G1, G2, Omega, dt):
    """matlab/tcl4_kernels.m:38-57 for scalar series (op2 = 'T' is the identity)."""
    N = G1.shape[0]
    t = np.arange(N) * dt
    pm = np.exp(-1j * Omega * t)
    pp = np.exp(+1j * Omega * t)

    def prefix(y):
        return dt * np.cumsum(y)

    def conv(f, g):
        L = 2 * N - 1
        return dt * np.fft.ifft(np.fft.fft(f, L) * np.fft.fft(g, L))[:N]

    F = G1 * pm * prefix(G2 * pp) - conv(G1 * pm, G2)
    Cc = G1 * pm * prefix(np.conj(G2) * pp) - conv(G1 * pm, np.conj(G2))
    R = G1 * prefix(G2 * pm) - prefix(G1 * G2 * pm)
    return F, Cc, R


def fcr_all(gamma, omegas, mirror, dt):
    """gamma [nf, Nt] -> F, C, R [nf, nf, nf, Nt] (cpp/src/tcl/tcl4.cpp:163-178 pairing)."""
    nf, Nt = gamma.shape
    F = np.zeros((nf, nf, nf, Nt), np.complex128)
    Cc = np.zeros_like(F)
    R = np.zeros_like(F)
    for i in range(nf):
        for j in range(nf):
            for k in range(nf):
                w = omegas[i] + omegas[j] + omegas[k]
                F[i, j, k], _, _ = tcl4_kernels_scalar(gamma[i], gamma[mirror[j]], w, dt)
                _, Cc[i, j, k], R[i, j, k] = tcl4_kernels_scalar(gamma[i], gamma[j], w, dt)
    return F, Cc, R


# ------------------------------------------------------------ MIKX (spec) ---
def tensorprod(A, B, da, db):
    """MATLAB tensorprod(A, B, dimA, dimB) with 1-based dims."""
    return np.tensordot(A, B, axes=([d - 1 for d in da], [d - 1 for d in db]))


def permute(A, order):
    return np.transpose(A, [o - 1 for o in order])


def six(Tt, p2f, N):
    """reshape(T(map.ij, map.ij, map.ij), [N N N N N N]) (tcl4_driver.m:48-50), column-major."""
    ij = p2f.reshape(-1, order="F")  # map.ij: pair (a, b) -> a + N*b
    T3 = Tt[np.ix_(ij, ij, ij)]
    return T3.reshape((N,) * 6, order="F")


def mikx_spec(Ft, Ct, Rt, p2f, N):
    """matlab/MIKX.m:17-50.  Returns M, I, K as 4-index arrays and X as a 6-index array."""
    I3 = np.zeros((N, N, N))
    for a in range(N):
        I3[a, a, a] = 1.0
    A = six(Ft, p2f, N)
    B = six(Rt, p2f, N)
    Cs = six(Ct, p2f, N)
    M1 = permute(tensorprod(tensorprod(A, I3, [3, 6], [1, 2]), I3, [1, 5], [1, 2]), [4, 2, 3, 1])
    M2 = permute(tensorprod(tensorprod(B, I3, [2, 5], [1, 2]), I3, [3, 5], [1, 2]), [1, 3, 2, 4])
    M = M1 - M2
    I1 = permute(tensorprod(tensorprod(A, I3, [3, 6], [1, 2]), I3, [2, 4], [1, 2]), [1, 4, 2, 3])
    K1 = permute(tensorprod(tensorprod(B, I3, [1, 6], [1, 2]), I3, [3, 4], [1, 2]), [3, 1, 2, 4])
    X = Cs + B
    return M, I1, K1, X


def nakzwan_spec(M, Ia, K, X, ops):
    """matlab/NAKZWAN_v9.m:1-41 (0-based loops)."""
    nd = M.shape[0]
    T = np.zeros((nd, nd, nd, nd), np.complex128)
    for n in range(nd):
        for i in range(nd):
            for m in range(nd):
                for j in range(nd):
                    res = 0j
                    for A in ops:
                        for B in ops:
                            for a in range(nd):
                                for b in range(nd):
                                    res = res - (
                                        B[n, a] * A[a, b] * B[b, i] * A[j, m] * M[b, i, n, a]
                                        - A[n, a] * B[a, b] * B[b, i] * A[j, m] * Ia[a, n, i, b]
                                        + B[n, a] * B[a, b] * A[b, i] * A[j, m] * K[i, b, n, a]
                                        + A[n, a] * B[a, i] * B[j, b] * A[b, m] * X[a, n, j, b, n, i]
                                        - B[n, a] * A[a, i] * B[j, b] * A[b, m] * X[i, a, j, b, n, i]
                                        - A[n, a] * A[a, b] * B[b, i] * B[j, m] * X[b, a, j, m, a, i]
                                        + A[n, a] * B[a, b] * A[b, i] * B[j, m] * X[i, b, j, m, a, i])
                                    if j == m:
                                        for c in range(nd):
                                            res = res + (
                                                A[n, a] * B[a, b] * A[b, c] * B[c, i] * M[c, i, a, b]
                                                + A[n, a] * B[a, b] * B[b, c] * A[c, i] * K[i, c, a, b]
                                                - A[n, a] * A[a, b] * B[b, c] * B[c, i] * Ia[b, a, i, c])
                    T[n, i, m, j] = res
    T2 = T.reshape(nd * nd, nd * nd, order="F")
    return T2 + T2.conj().T


def gw_to_l4(GW, N):
    L = np.zeros_like(GW)
    for n in range(N):
        for m in range(N):
            for i in range(N):
                for j in range(N):
                    L[n + N * m, i + N * j] = GW[n + N * i, m + N * j]
    return L


def l4_at(F, Cc, R, t, p2f, N, ops):
    nf = F.shape[0]
    Ft = F[..., t].reshape(nf, nf, nf)
    Ct = Cc[..., t].reshape(nf, nf, nf)
    Rt = R[..., t].reshape(nf, nf, nf)
    M, I1, K1, X = mikx_spec(Ft, Ct, Rt, p2f, N)
    GW = nakzwan_spec(M, I1, K1, X, ops)
    return GW, gw_to_l4(GW, N)


# ------------------------------------------------------------ bath / Gamma ---
def bcf_fft(N, dt, J, beta):
    Nt = N + 1
    nfft = 2 * Nt
    if nfft & (nfft - 1):
        nfft = 1 << (nfft - 1).bit_length()
    dw = 2 * np.pi / (dt * nfft)
    wny = np.pi / dt
    S = np.zeros(nfft, np.complex128)
    r = np.exp(-beta * dw)
    kms = r
    for k in range(1, nfft // 2):
        sp = (np.pi / 2) * J(dw * k) / (1 - kms)
        S[k] = sp
        S[nfft - k] = sp * kms
        kms *= r
    S[0] = 0.5 * (np.pi / 2) * J(dw) * (1 + r) / (1 - r)
    S[nfft // 2] = 0.25 * np.pi * J(wny) * (1 + 2 / (np.exp(beta * wny) - 1))
    Cf = np.fft.fft(S) * (dw / np.pi)
    return np.arange(Nt) * dt, Cf[:Nt]


def gamma_trapz(C, dt, omegas):
    N = C.size
    G = np.zeros((len(omegas), N), np.complex128)
    for j, w in enumerate(omegas):
        step = np.exp(1j * w * dt)
        phi = 1.0 + 0j
        acc = 0j
        for k in range(1, N):
            nxt = phi * step
            acc += (dt / 2) * (phi * C[k - 1] + nxt * C[k])
            G[j, k] = acc
            phi = nxt
    return G


# ------------------------------------------------------------- TCL2 + RK4 ---
def tcl2_total(eps, p2f, A_eig, gamma_b):
    N = eps.size
    I = np.eye(N)
    L = np.zeros((N * N, N * N), np.complex128)
    Hls = np.zeros((N, N), np.complex128)
    for b in range(gamma_b.size):
        for A in A_eig:
            Aw = np.where(p2f == b, A, 0)
            if np.sum(np.abs(Aw) ** 2) == 0:
                continue
            G = gamma_b[b]
            AdA = Aw.conj().T @ Aw
            if np.sum(np.abs(AdA) ** 2) == 0:
                continue
            Hls += G.imag * AdA
            g = 2 * G.real
            L += g * (np.kron(Aw.conj(), Aw) - 0.5 * np.kron(I, AdA) - 0.5 * np.kron(AdA.T, I))
    Hls = 0.5 * (Hls + Hls.conj().T)
    Heff = np.diag(eps) + Hls
    Lu = -1j * (np.kron(I, Heff) - np.kron(Heff.T, I))
    return Lu + L


def rk4(L_series, r, dt):
    r = r.copy()
    for i in range(L_series.shape[0] - 1):
        L0, L1 = L_series[i], L_series[i + 1]
        Lh = 0.5 * (L0 + L1)
        k1 = L0 @ r
        k2 = Lh @ (r + 0.5 * dt * k1)
        k3 = Lh @ (r + 0.5 * dt * k2)
        k4 = L1 @ (r + dt * k3)
        r = r + (dt / 6) * (k1 + 2 * k2 + 2 * k3 + k4)
    return r


# --------------------------------------------------------------- fixtures ---
def make_makeval():
    """MIKX and GW fixtures of cpp/tests/tcl4_mikx_tests.cpp:53-87 / tests/tcl4_tests.cpp:40-90."""
    N, nf, Nt = 2, 4, 4
    p2f = np.array([[0, 1], [2, 3]], np.int32)  # p2f[a, b]; (0,0)=0 (0,1)=1 (1,0)=2 (1,1)=3

    def make_val(base, a, b, c, t):
        return complex(base + 100.0 * a + 10.0 * b + c + 0.001 * t,
                       0.1 * base + 0.01 * a - 0.001 * b + 0.0001 * c + 0.00001 * t)

    F = np.zeros((nf, nf, nf, Nt), np.complex128)
    Cc = np.zeros_like(F)
    R = np.zeros_like(F)
    for a in range(nf):
        for b in range(nf):
            for c in range(nf):
                for t in range(Nt):
                    F[a, b, c, t] = make_val(1.0, a, b, c, t)
                    Cc[a, b, c, t] = make_val(2.0, a, b, c, t)
                    R[a, b, c, t] = make_val(3.0, a, b, c, t)
    ops = [np.eye(2, dtype=np.complex128), SX.copy()]
    tids = np.array([0, Nt // 2, Nt - 1])
    Ms, Is, Ks, Xs, GWs, L4s = [], [], [], [], [], []
    for t in tids:
        M, I1, K1, X = mikx_spec(F[..., t], Cc[..., t], R[..., t], p2f, N)
        GW = nakzwan_spec(M, I1, K1, X, ops)
        Ms.append(M.reshape(N * N, N * N, order="F"))
        Is.append(I1.reshape(N * N, N * N, order="F"))
        Ks.append(K1.reshape(N * N, N * N, order="F"))
        Xs.append(X.reshape(-1, order="F"))
        GWs.append(GW)
        L4s.append(gw_to_l4(GW, N))
    np.savez_compressed(os.path.join(HERE, "mikx_makeval.npz"), N=N, nf=nf, Nt=Nt, p2f=p2f,
                        F=F.reshape(nf ** 3, Nt), C=Cc.reshape(nf ** 3, Nt), R=R.reshape(nf ** 3, Nt),
                        ops=np.stack(ops), tids=tids, M=np.stack(Ms), I=np.stack(Is), K=np.stack(Ks),
                        X=np.stack(Xs), GW=np.stack(GWs), L4=np.stack(L4s))


def make_synthetic_gamma():
    """tests/tcl4_mpi_omp_tests.cpp:37-55: H = sx/2, A = sz/2, Nt = 16, dt = 0.01."""
    w, U, omegas, p2f, A_eig = eig_system(0.5 * SX, [0.5 * SZ])
    mirror = mirror_map(omegas)
    nf, Nt, dt = omegas.size, 16, 0.01
    gamma = np.zeros((nf, Nt), np.complex128)
    for t in range(Nt):
        for b in range(nf):
            gamma[b, t] = complex(0.01 * (t + 1) * (b + 1), 0.005 * t - 0.002 * b)
    F, Cc, R = fcr_all(gamma, omegas, mirror, dt)
    tids = np.array([0, Nt // 2, Nt - 1])
    N = 2
    L4 = np.stack([l4_at(F, Cc, R, t, p2f, N, A_eig)[1] for t in range(Nt)])
    np.savez_compressed(os.path.join(HERE, "synthetic_gamma.npz"), N=N, nf=nf, Nt=Nt, dt=dt,
                        eps=w, omegas=omegas, mirror=mirror, p2f=p2f, ops=np.stack(A_eig),
                        gamma=gamma, F=F.reshape(nf ** 3, Nt), C=Cc.reshape(nf ** 3, Nt),
                        R=R.reshape(nf ** 3, Nt), tids=tids, L4_all=L4)


def make_spin_boson_small():
    """d=2 spin-boson: H = (eps*sz + Delta*sx)/2, A = sz, J = alpha*w*exp(-w/wc), end to end."""
    eps_, Delta, alpha, wc, beta = 1.0, 1.0, 0.05, 10.0, 1.0
    N_grid, dt = 256, 0.005
    H = 0.5 * eps_ * SZ + 0.5 * Delta * SX
    w, U, omegas, p2f, A_eig = eig_system(H, [SZ])
    mirror = mirror_map(omegas)

    def J(x):
        return alpha * x * np.exp(-x / wc) if x > 0 else 0.0

    t, C = bcf_fft(N_grid, dt, J, beta)
    gamma = gamma_trapz(C, dt, omegas)
    F, Cc, R = fcr_all(gamma, omegas, mirror, dt)
    N = 2
    nf, Nt = omegas.size, C.size
    steps = 64
    L4 = np.stack([l4_at(F, Cc, R, k, p2f, N, A_eig)[1] for k in range(steps + 1)])
    L2 = np.stack([tcl2_total(w, p2f, A_eig, gamma[:, k]) for k in range(steps + 1)])
    rho0_lab = np.array([[1, 0], [0, 0]], np.complex128)
    rho0 = U.conj().T @ rho0_lab @ U
    r0 = rho0.reshape(-1, order="F")
    r_final = rk4(L2 + L4, r0, dt)
    np.savez_compressed(os.path.join(HERE, "spin_boson_small.npz"), N=N, nf=nf, Nt=Nt, dt=dt,
                        params=np.array([eps_, Delta, alpha, wc, beta]), eps=w, U=U, omegas=omegas,
                        mirror=mirror, p2f=p2f, ops=np.stack(A_eig), C=C, gamma=gamma,
                        F=F.reshape(nf ** 3, Nt), Cf=Cc.reshape(nf ** 3, Nt), R=R.reshape(nf ** 3, Nt),
                        steps=steps, L4=L4, L2=L2, r0=r0, r_final=r_final)


if __name__ == "__main__":
    make_makeval()
    make_synthetic_gamma()
    make_spin_boson_small()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")
