"""The no-allocation entry point (taco_tcl4_build_batch_noalloc).

It exists for callers that cannot allocate device memory while they run (a framework's
caching allocator owns the GPU memory; cudaMalloc would synchronise a latency-critical
loop; a plugin host forbids allocation after start-up).  Its results are checked against
the oracle and against the allocating entry point; it is also checked to leave the device's
free memory and torch's reserved memory unchanged, and to reject host, misaligned and
capturing-stream arguments before any launch.  This file is collected last so that a
failure here never hides the other tests; it passes alone and after them.
"""
import ctypes as ct

import numpy as np
import pytest

import taco_b200 as tb
from taco_b200 import _capi
from cases import oracle_l4, random_case, relerr, spin_boson_case

pytestmark = pytest.mark.gpu


def _call_noalloc(system, gamma_ptr, Nt, dt, tidx, precision, out_ptr, stream=None):
    import torch
    view = tb._View(system)
    tid = np.ascontiguousarray(tidx, np.uint32)
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    _capi.check(_capi.lib().taco_tcl4_build_batch_noalloc(
        ct.byref(view.view), ct.c_void_p(gamma_ptr), Nt, float(dt),
        tid.ctypes.data_as(ct.c_void_p), tid.size, precision, ct.c_void_p(out_ptr), ct.c_void_p(stream)))


def _run(system, g, dt, tidx, precision):
    """One call into a fresh NaN-filled output; returns the L4 matrices [T][N^2][N^2]."""
    import torch
    prec = _capi.TACO_PREC_FP64 if precision == "fp64" else _capi.TACO_PREC_FP32
    dtype = torch.complex128 if precision == "fp64" else torch.complex64
    D = system.N * system.N
    out = torch.full((len(tidx), D * D), complex(np.nan, np.nan), dtype=dtype, device="cuda")
    _call_noalloc(system, g.data_ptr(), g.shape[1], dt, tidx, prec, out.data_ptr())
    res = out.view(len(tidx), D, D).transpose(1, 2).cpu().numpy()
    assert np.isfinite(res).all()
    return res


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_matches_allocating_entry_point_twice(precision):
    import torch
    osys, s, G = spin_boson_case(4000, 0.005)
    g = torch.from_numpy(G).cuda()
    tidx = np.arange(0, 1001)
    ref = tb.build_TCL4_generator_batch(s, g, 0.005, tidx, precision=precision).cpu().numpy()
    ora = oracle_l4(osys, G, 0.005, tidx=tidx)
    tol = 1e-10 if precision == "fp64" else 1e-6
    outs = []
    for _ in range(2):  # two calls in a row: the shared scratch keeps the previous contents
        res = _run(s, g, 0.005, tidx, precision)
        assert relerr(res, ref) <= tol
        assert relerr(res, ora) <= tol
        outs.append(res)
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_shuffled_repeated_times_match_oracle(precision):
    """Unsorted, repeated time indices up to 3999 (FFT 8192: the inverse column pass by
    shared-memory tiles rather than the pruned DFT) against the oracle at those times."""
    import torch
    osys, s, G = spin_boson_case(4000, 0.005)
    g = torch.from_numpy(G).cuda()
    rng = np.random.default_rng(11)
    tidx = rng.integers(0, 4000, 300)
    tidx[:5] = 3999
    tidx[5:10] = tidx[10:15]  # duplicates
    ora = oracle_l4(osys, G, 0.005, tidx=tidx)
    res = _run(s, g, 0.005, tidx, precision)
    assert relerr(res, ora) <= (1e-10 if precision == "fp64" else 1e-6)


def test_noalloc_several_triple_chunks_d4_matches_oracle():
    """d = 4 (nf = 13, 2197 triples): the fixed scratch holds fewer FFT work areas than
    triples, so the triples run in several chunks through the same work areas."""
    import torch
    osys, s, G = random_case(4, 1, 400, 0.01, seed=5)
    assert osys.nf ** 3 > 1200
    g = torch.from_numpy(G).cuda()
    rng = np.random.default_rng(3)
    tidx = rng.integers(0, 300, 40)
    tidx[0] = 299
    ora = oracle_l4(osys, G, 0.01, tidx=tidx)
    for _ in range(2):
        res = _run(s, g, 0.01, tidx, "fp64")
        assert relerr(res, ora) <= 1e-10


def test_noalloc_allocates_nothing():
    """After a first call (which loads the kernels), repeated calls change neither the
    device's free memory nor torch's reserved memory."""
    import torch
    osys, s, G = spin_boson_case(4000, 0.005)
    g = torch.from_numpy(G).cuda()
    tidx = np.arange(0, 2001, 2)
    out = torch.empty((tidx.size, 16), dtype=torch.complex128, device="cuda")
    _call_noalloc(s, g.data_ptr(), g.shape[1], 0.005, tidx, _capi.TACO_PREC_FP64, out.data_ptr())
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    for _ in range(3):
        _call_noalloc(s, g.data_ptr(), g.shape[1], 0.005, tidx, _capi.TACO_PREC_FP64, out.data_ptr())
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_reserved() == reserved0


def test_noalloc_rejects_host_misaligned_and_capturing_arguments():
    """Rejected before any launch: a host gamma, a host output, a misaligned output and a
    stream under capture."""
    import torch
    osys, s, G = spin_boson_case(600, 0.005)
    g = torch.from_numpy(G).cuda()
    tidx = np.arange(0, 101)
    out = torch.empty((tidx.size + 1, 16), dtype=torch.complex128, device="cuda")
    host_out = np.empty((tidx.size, 16), np.complex128)
    fp64 = _capi.TACO_PREC_FP64
    with pytest.raises(ValueError, match="gamma"):
        _call_noalloc(s, G.ctypes.data, G.shape[1], 0.005, tidx, fp64, out.data_ptr())
    with pytest.raises(ValueError, match="L4_out"):
        _call_noalloc(s, g.data_ptr(), g.shape[1], 0.005, tidx, fp64, host_out.ctypes.data)
    with pytest.raises(ValueError, match="aligned"):
        _call_noalloc(s, g.data_ptr(), g.shape[1], 0.005, tidx, fp64, out.data_ptr() + 8)
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    msgs = []
    with torch.cuda.graph(graph, stream=side):
        try:
            _call_noalloc(s, g.data_ptr(), g.shape[1], 0.005, tidx, fp64, out.data_ptr(),
                          stream=side.cuda_stream)
        except ValueError as e:
            msgs.append(str(e))
        out.zero_()
    assert msgs and "captured" in msgs[0]
    del graph
    # the library still works afterwards
    res = _run(s, g, 0.005, tidx, "fp64")
    assert relerr(res, oracle_l4(osys, G, 0.005, tidx=tidx)) <= 1e-10


def test_noalloc_rejects_requests_above_the_fixed_scratch():
    import torch
    osys, s, G = spin_boson_case(200000, 5e-4)
    g = torch.from_numpy(G).cuda()
    tidx = np.arange(0, 200001, 1)  # needs far more than the fixed scratch
    out = torch.empty((tidx.size, 16), dtype=torch.complex128, device="cuda")
    with pytest.raises(OverflowError) as ei:
        _call_noalloc(s, g.data_ptr(), g.shape[1], 5e-4, tidx, _capi.TACO_PREC_FP64, out.data_ptr())
    assert "TACO_NOALLOC_SCRATCH_BYTES" in str(ei.value)
    # the library still works afterwards
    small = np.arange(0, 100)
    res = _run(s, g, 5e-4, small, "fp64")
    ref = tb.build_TCL4_generator_batch(s, g, 5e-4, small).cpu().numpy()
    assert relerr(res, ref) <= 1e-10
