"""The pybind module `_taco_native` (the reference's module name, cpp/python/_taco_native.cpp:6-9)
against the ctypes path: version on CPU; L4, F/C/R and RK4 on the device."""
import numpy as np
import pytest

import taco_b200 as tb
from cases import relerr, spin_boson_case


def _nat():
    from taco_b200 import _taco_native
    return _taco_native


def test_native_module_loads_and_reports_version():
    nat = _nat()
    assert nat.version() == tb.version()
    old = nat.get_fcr_fft_pad_factor()
    nat.set_fcr_fft_pad_factor(4)
    assert nat.get_fcr_fft_pad_factor() == 4
    nat.set_fcr_fft_pad_factor(old)


@pytest.mark.gpu
def test_native_build_and_kernels_match_ctypes_path():
    nat = _nat()
    osys, s, G = spin_boson_case(1200, 0.005)
    p2f = np.ascontiguousarray(s.pair_to_freq.T, np.int32)
    ops = np.ascontiguousarray(np.stack([A.T for A in s.A_eig]).reshape(len(s.A_eig), -1))
    tidx = np.array([0, 3, 600, 1200], np.uint32)
    L4, ms = nat.build_tcl4_generator_batch(s.N, s.omegas, s.mirror, p2f, ops, 1e-9, G, 0.005, tidx,
                                            tb.TACO_PREC_FP64)
    ref = tb.build_TCL4_generator_batch(s, G, 0.005, tidx)
    assert relerr(L4.reshape(4, 4, 4).transpose(0, 2, 1), ref) <= 1e-14
    assert ms >= 0.0
    L32, _ = nat.build_tcl4_generator_batch(s.N, s.omegas, s.mirror, p2f, ops, 1e-9, G, 0.005, tidx,
                                            tb.TACO_PREC_FP32)
    assert relerr(L32.reshape(4, 4, 4).transpose(0, 2, 1), ref) <= 1e-6
    F, C, R = nat.compute_triple_kernels(s.N, s.omegas, s.mirror, p2f, 1e-9, G, 0.005)
    Ft, Ct, Rt = tb.compute_triple_kernels(s, G, 0.005)
    for a, b in ((F, Ft), (C, Ct), (R, Rt)):
        assert relerr(a, b.reshape(a.shape)) <= 1e-14
    rng = np.random.default_rng(1)
    Ls = 0.3 * (rng.standard_normal((21, 4, 4)) + 1j * rng.standard_normal((21, 4, 4)))
    r0 = rng.standard_normal(4) + 1j * rng.standard_normal(4)
    r = nat.rk4_propagate(np.ascontiguousarray(Ls.transpose(0, 2, 1)), r0, 0.01)
    r_ref, _, _ = tb.propagate_rk4_dense(Ls, r0, 0.01)
    assert relerr(r, r_ref) <= 1e-14
