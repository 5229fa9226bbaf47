"""Seeded test cases shared by the GPU parity tests (inputs built with the oracle)."""
import numpy as np

import oracle
import taco_b200 as tb

SX = np.array([[0, 1], [1, 0]], np.complex128)
SZ = np.array([[1, 0], [0, -1]], np.complex128)


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def spin_boson_case(N_grid, dt, eps=1.0, delta=1.0, alpha=0.05, wc=10.0, beta=1.0):
    """Config-1 style spin boson: H = (eps sz + delta sx)/2, A = sz, Ohmic J, trapz Gamma."""
    H = 0.5 * eps * SZ + 0.5 * delta * SX
    osys = oracle.System(H, [SZ])
    _, C = oracle.bcf_fft(N_grid, dt, oracle.J_OHMIC, [alpha, wc], beta)
    G = oracle.gamma_trapz(C, dt, osys.omegas)
    s = tb.System.from_arrays(osys.N, osys.omegas, osys.pair_to_freq, osys.A_eig, mirror=osys.mirror, eps=osys.eps)
    s.U = osys.U
    return osys, s, G


def random_case(d, nops, Nt, dt, seed):
    """GUE-style H and random Hermitian couplings, Ohmic + Drude bath."""
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    H = (X + X.conj().T) / (2 * np.sqrt(2 * d))
    As = []
    for _ in range(nops):
        Y = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
        A = (Y + Y.conj().T) / 2
        As.append(A / np.linalg.norm(A, 2))
    osys = oracle.System(H, As)
    _, C = oracle.bcf_fft(Nt - 1, dt, oracle.J_OHMIC_DRUDE, [0.1, 5.0, 0.05, 2.0], 0.5)
    G = oracle.gamma_trapz(C, dt, osys.omegas)
    s = tb.System.from_arrays(osys.N, osys.omegas, osys.pair_to_freq, osys.A_eig, mirror=osys.mirror)
    return osys, s, G


def oracle_l4(osys, G, dt, tidx=None):
    return oracle.tcl4_build_batch(osys.N, osys.nf, osys.omegas, osys.mirror, osys.p2f_colmajor(),
                                   osys.ops_colmajor(), G, dt, tidx=tidx)
