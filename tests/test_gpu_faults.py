"""Failures made on the host, the way the reference's entry points throw
(cpp/src/backend/cuda/tcl4_fused_cuda.cu:1107-1215): bad pointers at the C-ABI, a work budget
too small for one frequency triple, and NaN/Inf samples in Gamma.  Every rejected call fails
before any launch, and the library works normally afterwards.
"""
import ctypes as ct

import numpy as np
import pytest

import taco_b200 as tb
from taco_b200 import _capi
from cases import oracle_l4, relerr, spin_boson_case

pytestmark = pytest.mark.gpu


def _raw_build(s, gamma_ptr, Nt, dt, tidx, out_ptr, flags, precision=_capi.TACO_PREC_FP64):
    v = tb._View(s)
    tid = np.ascontiguousarray(tidx, np.uint32)
    ms = ct.c_double(0.0)
    _capi.check(_capi.lib().taco_tcl4_build_batch(ct.byref(v.view), ct.c_void_p(gamma_ptr), Nt, float(dt),
                                                  tid.ctypes.data_as(ct.c_void_p), tid.size, 0, precision,
                                                  ct.c_void_p(out_ptr), flags, None, ct.byref(ms)))


def _check_still_works(osys, s, G, dt, tidx):
    ref = oracle_l4(osys, G, dt, tidx)
    assert relerr(tb.build_TCL4_generator_batch(s, G, dt, tidx), ref) <= 1e-10


def test_null_host_and_misaligned_device_pointers_rejected():
    import torch
    osys, s, G = spin_boson_case(600, 0.005)
    tidx = np.arange(0, 101)
    g = torch.from_numpy(G).cuda()
    out = torch.empty((tidx.size + 1, 16), dtype=torch.complex128, device="cuda")
    dev = _capi.TACO_IN_DEVICE | _capi.TACO_OUT_DEVICE
    with pytest.raises(ValueError, match="null"):
        _raw_build(s, 0, G.shape[1], 0.005, tidx, out.data_ptr(), dev)
    with pytest.raises(ValueError, match="host memory"):  # a host array flagged as device memory
        _raw_build(s, G.ctypes.data, G.shape[1], 0.005, tidx, out.data_ptr(), dev)
    with pytest.raises(ValueError, match="aligned"):
        _raw_build(s, g.data_ptr() + 8, G.shape[1], 0.005, tidx, out.data_ptr(), dev)
    with pytest.raises(ValueError, match="aligned"):
        _raw_build(s, g.data_ptr(), G.shape[1], 0.005, tidx, out.data_ptr() + 8, dev)
    host_out = np.empty((tidx.size, 16), np.complex128)
    with pytest.raises(ValueError, match="host memory"):
        _raw_build(s, g.data_ptr(), G.shape[1], 0.005, tidx, host_out.ctypes.data, dev)
    _check_still_works(osys, s, G, 0.005, tidx)


def test_work_budget_below_one_triple_is_an_overflow():
    osys, s, G = spin_boson_case(2000, 0.005)
    tidx = np.arange(0, 1500)
    import torch
    g = torch.from_numpy(G).cuda()
    tb.set_work_budget(1024)
    try:
        with pytest.raises(OverflowError, match="work budget"):
            tb.build_TCL4_generator_batch(s, g, 0.005, tidx)
    finally:
        tb.set_work_budget(0)
    _check_still_works(osys, s, G, 0.005, tidx)


@pytest.mark.parametrize("bad", [np.nan, np.inf])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_nonfinite_gamma_propagates_without_fault(bad, precision):
    """A NaN or Inf sample reaches the outputs (the FFT spreads it over the series, as the
    reference's FFT does); no exception, no fault, and the FP32 guard's growth ends."""
    osys, s, G = spin_boson_case(1500, 0.005)
    tidx = np.arange(0, 1001)
    Gb = G.copy()
    Gb[1, 700] = complex(bad, 0.0)
    out = tb.build_TCL4_generator_batch(s, Gb, 0.005, tidx, precision=precision)
    assert not np.isfinite(out).all()
    if precision == "fp32":
        st = tb.fp32_guard_stats()
        assert st["rounds"] >= 1
    _check_still_works(osys, s, G, 0.005, tidx)
