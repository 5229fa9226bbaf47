"""The unfused MIKX / GW / L4 stages on the device against the golden fixture of the
reference's MIKX unit test and CUDA assemble check (cpp/tests/tcl4_mikx_tests.cpp:53-160,
tests/tcl4_tests.cpp:40-162: N=2, nf=4, identity pair map, ops {I, sigma_x}) and the oracle."""
import os

import numpy as np
import pytest

import oracle
import taco_b200 as tb
from cases import random_case, relerr

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_mikx_gw_l4_makeval_fixture():
    g = np.load(os.path.join(GOLD, "mikx_makeval.npz"))
    t = g["tids"]
    M, I, K, X = tb.build_mikx(g["F"][:, t].T, g["C"][:, t].T, g["R"][:, t].T, g["p2f"], int(g["N"]))
    assert np.max(np.abs(M - g["M"])) <= 1e-12 and np.max(np.abs(I - g["I"])) <= 1e-12
    assert np.max(np.abs(K - g["K"])) <= 1e-12 and np.max(np.abs(X - g["X"])) <= 1e-12
    GW = tb.assemble_liouvillian(M, I, K, X, list(g["ops"]))
    assert relerr(GW, g["GW"]) <= 1e-13  # reference CPU-vs-CUDA bar: 1e-9 (tests/tcl4_tests.cpp:156)
    L4 = tb.gw_to_liouvillian(GW)
    assert relerr(L4, g["L4"]) <= 1e-13
    raw = tb.assemble_liouvillian(M, I, K, X, list(g["ops"]), symmetrize=False)
    assert relerr(raw + np.conj(np.swapaxes(raw, 1, 2)), g["GW"]) <= 1e-13


def test_stages_match_oracle_random_d3():
    osys, s, G = random_case(3, 2, 60, 0.01, seed=5)
    F, C, R = oracle.fcr_series(G, osys.omegas, osys.mirror, 0.01)
    t = [3, 59]
    M, I, K, X = tb.build_mikx(F[:, t].T, C[:, t].T, R[:, t].T, osys.pair_to_freq, 3)
    for k, tt in enumerate(t):
        Mo, Io, Ko, Xo = oracle.mikx(F[:, tt], C[:, tt], R[:, tt], osys.nf, osys.p2f_colmajor(), 3)
        assert np.max(np.abs(M[k] - Mo.reshape(9, 9).T)) <= 1e-14
        assert np.max(np.abs(X[k] - Xo)) <= 1e-14
        GWo = oracle.assemble_gw(Mo, Io, Ko, Xo, osys.ops_colmajor(), 3)
        GW = tb.assemble_liouvillian(M[k:k + 1], I[k:k + 1], K[k:k + 1], X[k:k + 1], osys.A_eig)
        assert relerr(GW[0], GWo.reshape(9, 9).T) <= 1e-13


def test_mikx_rejects_missing_bucket():
    p2f = np.array([[0, -1], [2, 3]])
    z = np.zeros((1, 64), np.complex128)
    with pytest.raises(RuntimeError):
        tb.build_mikx(z, z, z, p2f, 2)
