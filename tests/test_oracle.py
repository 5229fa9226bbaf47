"""The CPU oracle pinned against the reference's known-answer tests and the
golden vectors of tests/golden/ (independent numpy restatement of the MATLAB
specification)."""
import os

import numpy as np
import pytest
import scipy.linalg

import oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden")
SX = np.array([[0, 1], [1, 0]], np.complex128)
SZ = np.array([[1, 0], [0, -1]], np.complex128)


def gold(name):
    return np.load(os.path.join(GOLD, name))


def relerr(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


def test_fft_matches_numpy():
    rng = np.random.default_rng(0)
    for n in (2, 8, 1024):
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert relerr(oracle.fft(x, True), np.fft.fft(x)) < 1e-13
        assert relerr(oracle.fft(x, False), np.fft.ifft(x)) < 1e-13
    with pytest.raises(oracle.OracleError):
        oracle.fft(np.zeros(6), True)


def test_next_pow2():
    assert [oracle.next_pow2(n) for n in (0, 1, 2, 3, 5, 400001)] == [1, 1, 2, 4, 8, 524288]


def test_mikx_makeval_fixture():
    """cpp/tests/tcl4_mikx_tests.cpp:49-160 inputs; expectation from matlab/MIKX.m."""
    g = gold("mikx_makeval.npz")
    N, nf = int(g["N"]), int(g["nf"])
    p2f = np.ascontiguousarray(g["p2f"].T, np.int32)
    for k, t in enumerate(g["tids"]):
        M, I, K, X = oracle.mikx(g["F"][:, t], g["C"][:, t], g["R"][:, t], nf, p2f, N)
        np.testing.assert_allclose(M, g["M"][k].reshape(-1, order="F"), rtol=0, atol=1e-12)
        np.testing.assert_allclose(I, g["I"][k].reshape(-1, order="F"), rtol=0, atol=1e-12)
        np.testing.assert_allclose(K, g["K"][k].reshape(-1, order="F"), rtol=0, atol=1e-12)
        np.testing.assert_allclose(X, g["X"][k], rtol=0, atol=1e-12)
        ops = np.ascontiguousarray(np.transpose(g["ops"], (0, 2, 1)))
        GW = oracle.assemble_gw(M, I, K, X, ops, N)
        np.testing.assert_allclose(GW, g["GW"][k].reshape(-1, order="F"), rtol=1e-13, atol=1e-9)
        L4 = oracle.gw_to_l4(GW, N)
        np.testing.assert_allclose(L4, g["L4"][k].reshape(-1, order="F"), rtol=1e-13, atol=1e-9)


def test_mikx_stale_unit_test_expectation_differs():
    """The reference unit test expects M = F[f_jk][f_jq][f_pj] - R[...] (tcl4_mikx_tests.cpp:133-134);
    the implementation and MATLAB give F[f_jq][f_jk][f_pj].  The fixture makes them differ."""
    g = gold("mikx_makeval.npz")
    N, nf = 2, 4
    p2f = g["p2f"]
    F = g["F"][:, 0].reshape(nf, nf, nf)
    R = g["R"][:, 0].reshape(nf, nf, nf)
    M = g["M"][0]
    stale = np.zeros_like(M)
    for j in range(N):
        for k in range(N):
            for p in range(N):
                for q in range(N):
                    stale[j + N * k, p + N * q] = F[p2f[j, k], p2f[j, q], p2f[p, j]] - R[p2f[j, q], p2f[p, q], p2f[q, k]]
    assert np.max(np.abs(stale - M)) > 1.0


@pytest.mark.parametrize("method", [oracle.FCR_CONVOLUTION, oracle.FCR_DIRECT])
def test_synthetic_gamma_fixture(method):
    """tests/tcl4_mpi_omp_tests.cpp:37-81 inputs; F/C/R and L4 vs the MATLAB-spec restatement."""
    g = gold("synthetic_gamma.npz")
    F, C, R = oracle.fcr_series(g["gamma"], g["omegas"], g["mirror"], float(g["dt"]), method)
    for a, b in ((F, g["F"]), (C, g["C"]), (R, g["R"])):
        assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(b)))
    N = int(g["N"])
    ops = np.ascontiguousarray(np.transpose(g["ops"], (0, 2, 1)))
    p2f = np.ascontiguousarray(g["p2f"].T, np.int32)
    L4 = oracle.tcl4_build_batch(N, int(g["nf"]), g["omegas"], g["mirror"], p2f, ops, g["gamma"],
                                 float(g["dt"]), tidx=None, method=method)
    assert relerr(L4, g["L4_all"]) < 1e-10
    L4s = oracle.tcl4_build_batch(N, int(g["nf"]), g["omegas"], g["mirror"], p2f, ops, g["gamma"],
                                  float(g["dt"]), tidx=g["tids"], method=method)
    # tests/tcl4_mpi_omp_tests.cpp:77-85: batch at tids equals the full series at those tids (1e-10).
    assert np.max(np.abs(L4s - L4[g["tids"]])) <= 1e-10


def _tcl4_tests_system():
    return oracle.System(0.5 * SX, [0.5 * SZ])


@pytest.mark.parametrize("N,dt", [(2048, 0.000625), (4000, 0.0005)])
def test_direct_vs_convolution(N, dt):
    """tests/tcl4_tests.cpp:177-234 (beta=0.5, wc=10, J = w exp(-w/wc)) with a 1e-10 threshold."""
    s = _tcl4_tests_system()
    _, C = oracle.bcf_fft(N, dt, oracle.J_OHMIC, [1.0, 10.0], 0.5)
    G = oracle.gamma_trapz(C, dt, s.omegas)
    Fc, Cc, Rc = oracle.fcr_series(G, s.omegas, s.mirror, dt, oracle.FCR_CONVOLUTION)
    Fd, Cd, Rd = oracle.fcr_series(G, s.omegas, s.mirror, dt, oracle.FCR_DIRECT)
    Nt = G.shape[1]
    tids = [0, Nt // 4, Nt // 2, min(Nt - 1, 3 * Nt // 4), Nt - 1]
    for a, b in ((Fc, Fd), (Cc, Cd), (Rc, Rd)):
        err = np.abs(a[:, tids] - b[:, tids]) / np.maximum(1.0, np.abs(b[:, tids]))
        assert err.max() < 1e-10


def test_fft_pad_factor_keeps_results():
    s = _tcl4_tests_system()
    _, C = oracle.bcf_fft(300, 0.001, oracle.J_OHMIC, [1.0, 10.0], 0.5)
    G = oracle.gamma_trapz(C, 0.001, s.omegas)
    F0, C0, R0 = oracle.fcr_series(G, s.omegas, s.mirror, 0.001)
    oracle.set_fcr_fft_pad_factor(8)
    try:
        assert oracle.get_fcr_fft_pad_factor() == 8
        F1, C1, R1 = oracle.fcr_series(G, s.omegas, s.mirror, 0.001)
    finally:
        oracle.set_fcr_fft_pad_factor(0)
    assert relerr(F1, F0) < 1e-12 and relerr(C1, C0) < 1e-12 and relerr(R1, R0) == 0.0


def test_rk4_constant_L():
    """tests/rk4_dense_tests.cpp:43-70."""
    L = np.zeros((4, 4), np.complex128)
    L[0, 0], L[1, 1], L[2, 2], L[3, 3] = 0.10 - 0.03j, -0.07 + 0.05j, 0.02, -0.04 - 0.02j
    L[0, 2], L[2, 0], L[1, 3] = 0.03 + 0.01j, -0.02 + 0.02j, 0.01 - 0.04j
    r0 = np.array([1.0, 0.5 - 0.2j, -0.7 + 0.1j, 0.1 + 0.3j])
    r = oracle.rk4_propagate_const(L, r0, 0.0, 1.25, 0.0025)
    expect = scipy.linalg.expm(1.25 * L) @ r0
    assert np.linalg.norm(r - expect) / np.linalg.norm(expect) < 1e-6


def test_rk4_time_dependent_midpoints():
    """tests/rk4_dense_tests.cpp:72-102."""
    D, steps, dt = 3, 100, 0.01
    tf = steps * dt
    Ls = np.stack([i * dt * np.eye(D, dtype=np.complex128) for i in range(steps + 1)])
    Lh = np.stack([(i + 0.5) * dt * np.eye(D, dtype=np.complex128) for i in range(steps)])
    r0 = np.array([0.3 + 0.1j, -0.2 + 0.4j, 0.9 - 0.3j])
    r, _ = oracle.rk4_propagate(Ls, r0, dt, L_half=Lh)
    expect = np.exp(0.5 * tf * tf) * r0
    assert np.linalg.norm(r - expect) / np.linalg.norm(expect) < 1e-6
    r2, samples = oracle.rk4_propagate(Ls, r0, dt, sample_every=10)
    assert samples.shape == (11, D) and np.allclose(samples[0], r0) and np.allclose(samples[-1], r2)


def test_gamma_analytic():
    """tests/gamma_tests.cpp:22-81 on a shorter window (dt=1e-3, T=1000)."""
    wc, dt, T = 1.0, 1e-3, 1000.0
    n = int(np.ceil(T / dt))
    t = np.arange(n + 1) * dt
    C = wc * wc / (1 + 1j * wc * t) ** 2
    G = oracle.gamma_trapz(C, dt, [0.0, -1.0, 1.0])
    gfin = G[:, -1]
    J1 = 2 * np.pi * 1.0 * np.exp(-1.0)
    assert abs(2 * gfin[2].real - J1) / max(1.0, J1) < 2e-2
    assert abs(2 * gfin[0].imag - (-2.0 * wc)) < 5e-3


def test_spin_boson_end_to_end_fixture():
    g = gold("spin_boson_small.npz")
    eps_, Delta, alpha, wc, beta = g["params"]
    dt = float(g["dt"])
    H = 0.5 * eps_ * SZ + 0.5 * Delta * SX
    s = oracle.System(H, [SZ])
    assert np.allclose(s.eps, g["eps"], atol=1e-14)
    assert np.allclose(s.omegas, g["omegas"], atol=1e-14)
    assert (s.pair_to_freq == g["p2f"]).all() and (s.mirror == g["mirror"]).all()
    assert np.allclose(s.A_eig[0], g["ops"][0], atol=1e-14)  # same phase convention
    t, C = oracle.bcf_fft(int(g["Nt"]) - 1, dt, oracle.J_OHMIC, [alpha, wc], beta)
    assert relerr(C, g["C"]) < 1e-12
    G = oracle.gamma_trapz(C, dt, s.omegas)
    assert relerr(G, g["gamma"]) < 1e-12
    F, Cc, R = oracle.fcr_series(G, s.omegas, s.mirror, dt)
    assert relerr(F, g["F"]) < 1e-10 and relerr(Cc, g["Cf"]) < 1e-10 and relerr(R, g["R"]) < 1e-12
    steps = int(g["steps"])
    L4 = oracle.tcl4_build_batch(2, s.nf, s.omegas, s.mirror, s.p2f_colmajor(), s.ops_colmajor(), G, dt,
                                 tidx=np.arange(steps + 1))
    assert relerr(L4, g["L4"]) < 1e-10
    L2 = np.stack([oracle.tcl2_total(s, G[:, k])[0] for k in range(steps + 1)])
    assert relerr(L2, g["L2"]) < 1e-13
    r, _ = oracle.rk4_propagate(L2 + L4, g["r0"], dt)
    assert relerr(r, g["r_final"]) < 1e-12
