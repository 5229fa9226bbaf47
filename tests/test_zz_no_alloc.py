"""The no-allocation entry point (taco_tcl4_build_batch_noalloc) against the allocating one.

It exists for callers that cannot allocate device memory while they run (a framework's
caching allocator owns the GPU memory; cudaMalloc would synchronise a latency-critical
loop; a plugin host forbids allocation after start-up).  This file is collected last so
that a failure here never hides the other tests; it passes alone and after them.
"""
import ctypes as ct

import numpy as np
import pytest

import taco_b200 as tb
from taco_b200 import _capi
from cases import relerr, spin_boson_case

pytestmark = pytest.mark.gpu


def _call_noalloc(system, gamma_dev, dt, tidx, precision, out):
    view = tb._View(system)
    tid = np.ascontiguousarray(tidx, np.uint32)
    stream = __import__("torch").cuda.current_stream().cuda_stream
    _capi.check(_capi.lib().taco_tcl4_build_batch_noalloc(
        ct.byref(view.view), ct.c_void_p(gamma_dev.data_ptr()), gamma_dev.shape[1], float(dt),
        tid.ctypes.data_as(ct.c_void_p), tid.size, precision, ct.c_void_p(out.data_ptr()), ct.c_void_p(stream)))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_matches_allocating_entry_point_twice(precision):
    import torch
    osys, s, G = spin_boson_case(4000, 0.005)
    g = torch.from_numpy(G).cuda()
    tidx = np.arange(0, 1001)
    prec = _capi.TACO_PREC_FP64 if precision == "fp64" else _capi.TACO_PREC_FP32
    dtype = torch.complex128 if precision == "fp64" else torch.complex64
    ref = tb.build_TCL4_generator_batch(s, g, 0.005, tidx, precision=precision).cpu().numpy()
    tol = 1e-10 if precision == "fp64" else 1e-6
    outs = []
    for _ in range(2):  # two calls in a row: the shared scratch keeps the previous contents
        out = torch.full((tidx.size, 16), complex(np.nan, np.nan), dtype=dtype, device="cuda")
        _call_noalloc(s, g, 0.005, tidx, prec, out)
        res = out.view(tidx.size, 4, 4).transpose(1, 2).cpu().numpy()
        assert np.isfinite(res).all()
        assert relerr(res, ref) <= tol
        outs.append(res)
    assert np.array_equal(outs[0], outs[1])


def test_noalloc_rejects_requests_above_the_fixed_scratch():
    import torch
    osys, s, G = spin_boson_case(200000, 5e-4)
    g = torch.from_numpy(G).cuda()
    tidx = np.arange(0, 200001, 1)  # needs far more than the fixed scratch
    out = torch.empty((tidx.size, 16), dtype=torch.complex128, device="cuda")
    with pytest.raises(OverflowError) as ei:
        _call_noalloc(s, g, 5e-4, tidx, _capi.TACO_PREC_FP64, out)
    assert "TACO_NOALLOC_SCRATCH_BYTES" in str(ei.value)
    # the library still works afterwards
    small = np.arange(0, 100)
    out2 = torch.empty((small.size, 16), dtype=torch.complex128, device="cuda")
    _call_noalloc(s, g, 5e-4, small, _capi.TACO_PREC_FP64, out2)
    ref = tb.build_TCL4_generator_batch(s, g, 5e-4, small).cpu().numpy()
    assert relerr(out2.view(small.size, 4, 4).transpose(1, 2).cpu().numpy(), ref) <= 1e-10
