"""Host-side input preparation for the TCL4 path (the reference builds these on the host too).

* System: Hermitian eigensystem, Bohr-frequency buckets, coupling operators in the
  eigenbasis and the mirror map (cpp/include/taco/system.hpp:37-226,
  cpp/src/tcl/tcl4.cpp:40-101).  Eigenvector phase convention: the largest-magnitude
  component of each eigenvector (first within 1e-9 relative) is real and positive.
* bcf_fft: bath correlation function C(t) from J(w) and beta
  (cpp/include/taco/correlation_fft.hpp:153-214).
* gamma_trapz: Gamma_b(t_k) = int_0^{t_k} exp(i w_b tau) C(tau) dtau by the trapezoid rule
  (cpp/include/taco/gamma.hpp:166-213), as the [nf, Nt] array the engine consumes.
"""
from __future__ import annotations

import numpy as np

SX = np.array([[0, 1], [1, 0]], np.complex128)
SY = np.array([[0, -1j], [1j, 0]], np.complex128)
SZ = np.array([[1, 0], [0, -1]], np.complex128)


class System:
    def __init__(self, H=None, A_lab_list=(), tol: float = 1e-9):
        self.tol = float(tol)
        if H is None:
            return
        H = np.asarray(H, np.complex128)
        w, U = np.linalg.eigh(0.5 * (H + H.conj().T))
        for c in range(U.shape[1]):
            mags = np.abs(U[:, c])
            piv = int(np.nonzero(mags >= mags.max() * (1 - 1e-9))[0][0])
            U[:, c] *= np.conj(U[piv, c]) / abs(U[piv, c])
        d = H.shape[0]
        reps, pairs = [], []
        ftol = max(self.tol, np.finfo(float).eps)
        for m in range(d):
            for n in range(d):
                x = w[m] - w[n]
                for b, r in enumerate(reps):
                    if abs(r - x) <= ftol:
                        pairs[b].append((m, n))
                        break
                else:
                    reps.append(x)
                    pairs.append([(m, n)])
        order = np.argsort(np.array(reps), kind="stable")
        # first-seen (m, n) pair of each bucket: omega_b = eps_m - eps_n (the representative)
        self.rep_pairs = [pairs[ob][0] for ob in order]
        self.N = d
        self.eps = w
        self.U = U
        self.omegas = np.array(reps)[order]
        self.nf = self.omegas.size
        self.pair_to_freq = -np.ones((d, d), np.int32)
        for nb, ob in enumerate(order):
            for (m, n) in pairs[ob]:
                self.pair_to_freq[m, n] = nb
        self.A_lab = [np.asarray(A, np.complex128) for A in A_lab_list]
        self.A_eig = [U.conj().T @ A @ U for A in self.A_lab]
        self.mirror, self.zero_index = build_map(self.omegas, self.tol)

    @classmethod
    def from_arrays(cls, N, omegas, pair_to_freq, A_eig, mirror=None, tol=1e-9, eps=None):
        s = cls(None, (), tol)
        s.N = int(N)
        s.omegas = np.asarray(omegas, np.float64)
        s.nf = s.omegas.size
        s.pair_to_freq = np.asarray(pair_to_freq, np.int32)
        s.A_eig = [np.asarray(A, np.complex128) for A in A_eig]
        s.eps = None if eps is None else np.asarray(eps, np.float64)
        s.U = None
        if mirror is None:
            s.mirror, s.zero_index = build_map(s.omegas, tol)
        else:
            s.mirror = np.asarray(mirror, np.int32)
            s.zero_index = int(np.argmin(np.abs(s.omegas)))
        return s


def build_map(omegas, tol=1e-9):
    """mirror[b]: bucket closest to -omega_b (itself when |omega_b| <= max(1e-12, tol))."""
    t = max(1e-12, tol)
    om = np.asarray(omegas, np.float64)
    mirror = np.zeros(om.size, np.int32)
    zero = -1
    for b, w in enumerate(om):
        if abs(w) <= t:
            mirror[b] = b
            if zero < 0:
                zero = b
        else:
            mirror[b] = int(np.argmin(np.abs(om + w)))
    if zero < 0:
        zero = int(np.argmin(np.abs(om))) if om.size else 0
    return mirror, zero


def spin_boson_system(eps=1.0, delta=1.0, a_scale=1.0):
    """H = (eps sz + delta sx)/2, A = a_scale sz (examples/TCL4_spin_boson_example.cpp:196-197)."""
    H = 0.5 * eps * SZ + 0.5 * delta * SX
    return System(H, [a_scale * SZ])


def ohmic(alpha, omega_c, lam=0.0, gam=1.0):
    """J(w) = alpha w exp(-w/wc) [+ 2 lam gam w / (w^2 + gam^2)] for w > 0, else 0."""
    def J(w):
        w = np.asarray(w, np.float64)
        v = alpha * w * np.exp(-w / omega_c)
        if lam:
            v = v + 2.0 * lam * gam * w / (w * w + gam * gam)
        return np.where(w > 0, v, 0.0)
    return J


def bcf_fft(N: int, dt: float, J, beta: float):
    """(t[0..N], C[0..N]) from the KMS spectrum (KMS factors by the r^k recurrence)."""
    Nt = N + 1
    nfft = 2 * Nt
    if nfft & (nfft - 1):
        nfft = 1 << (nfft - 1).bit_length()
    dw = 2 * np.pi / (dt * nfft)
    wny = np.pi / dt
    k = np.arange(1, nfft // 2)
    S = np.zeros(nfft, np.complex128)
    Jk = J(dw * k)
    if np.isinf(beta):
        S[k] = (np.pi / 2) * Jk
        S[0] = 0.0
        S[nfft // 2] = 0.25 * np.pi * J(np.array([wny]))[0]
    else:
        r = np.exp(-beta * dw)
        kms = r ** k
        sp = (np.pi / 2) * Jk / (1.0 - kms)
        S[k] = sp
        S[nfft - k] = sp * kms
        S[0] = 0.5 * (np.pi / 2) * J(np.array([dw]))[0] * (1 + r) / (1 - r)
        x = beta * wny  # coth(x/2) = 1 + 2/(e^x - 1); the term vanishes once e^x overflows
        S[nfft // 2] = 0.25 * np.pi * J(np.array([wny]))[0] * (1 + (2 / np.expm1(x) if x < 700 else 0.0))
    C = np.fft.fft(S) * (dw / np.pi)
    return np.arange(Nt) * dt, C[:Nt]


def gamma_trapz(C, dt: float, omegas):
    """[nf, Nt]: Gamma_b(t_k) by cumulative trapezoid of exp(i w_b tau) C(tau); Gamma(0) = 0."""
    C = np.asarray(C, np.complex128)
    Nt = C.size
    t = np.arange(Nt) * dt
    G = np.zeros((len(omegas), Nt), np.complex128)
    for b, w in enumerate(omegas):
        y = np.exp(1j * w * t) * C
        G[b, 1:] = np.cumsum(0.5 * dt * (y[:-1] + y[1:]))
    return G
