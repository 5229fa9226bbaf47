"""The fused F/C/R path (one CTA per triple and half: transforms, spectral product, prefix
integrals and assembly in shared memory) against the four-step passes and the oracle.

Tolerances: FP64 fused vs oracle <= 1e-10 and vs the four-step path <= 1e-12 (relative
Frobenius; the two paths may use different FFT lengths, both exact linear convolutions); FP32 (guard off, the FP32 pass alone) no further from FP64 than twice the
four-step path's error plus 1e-7.
"""
import numpy as np
import pytest

import taco_b200 as tb
from cases import oracle_l4, random_case, relerr, spin_boson_case

pytestmark = pytest.mark.gpu


def build_both(inst, precision, **kw):
    """(fused, four-step) results of one batched build."""
    import torch
    old = tb.fused_conv()
    try:
        tb.set_fused_conv(True)
        a = [x.cpu().numpy() for x in tb.build_instances(inst, precision=precision, **kw)]
        tb.set_fused_conv(False)
        b = [x.cpu().numpy() for x in tb.build_instances(inst, precision=precision, **kw)]
    finally:
        tb.set_fused_conv(old)
    torch.cuda.synchronize()
    return a, b


@pytest.mark.parametrize("tmax,nfft", [(1000, 2048), (1200, 2560), (1500, 3072), (10000, 20480), (4096, 10240)])
def test_fused_matches_four_step_and_oracle(tmax, nfft):
    import torch
    dt = 5e-4 if tmax == 10000 else 0.005
    osys, s, G = spin_boson_case(max(tmax, 4000), dt)
    fz_old = tb.fused_conv()
    try:
        # with the fused path selected, the causal rule takes 3 * 2^k and 5 * 2^k lengths that
        # the four-step column kernels do not cover (the four-step path then rounds up)
        tb.set_fused_conv(True)
        assert tb.fft_length(tmax + 1, "fp32")[0] == nfft
    finally:
        tb.set_fused_conv(fz_old)
    g = torch.from_numpy(G).cuda()
    tidx = np.arange(tmax + 1)
    inst = [(s, g, dt, tidx)]
    f64, s64 = build_both(inst, "fp64")
    assert relerr(f64[0], s64[0]) <= 1e-12
    if tmax <= 1500:
        assert relerr(f64[0], oracle_l4(osys, G, dt, tidx)) <= 1e-10
    old = tb.fp32_guard()
    tb.set_fp32_guard(0.0)
    try:
        f32, s32 = build_both(inst, "fp32")
    finally:
        tb.set_fp32_guard(old)
    ef, es = relerr(f32[0], f64[0]), relerr(s32[0], f64[0])
    assert ef <= 2 * es + 1e-7, (ef, es)


def test_fused_random_system_unsorted_times_vs_oracle():
    import torch
    osys, s, G = random_case(3, 2, 1300, 0.01, seed=21)
    g = torch.from_numpy(G).cuda()
    rng = np.random.default_rng(4)
    tidx = rng.integers(0, 1200, 200)
    tidx[:4] = tidx[4]
    f64, s64 = build_both([(s, g, 0.01, tidx)], "fp64")
    ref = oracle_l4(osys, G, 0.01, tidx)
    assert relerr(f64[0], ref) <= 1e-10
    assert relerr(f64[0], s64[0]) <= 1e-12


def test_fused_batched_instances_match_four_step():
    """64 headline-shaped instances (FFT 20480, 1728 triples: the four-step path's
    single-pass scan) in FP32 and 8 in FP64."""
    import torch
    from taco_b200.workloads import spin_boson_batch
    _, systems, gammas = spin_boson_batch(torch, 64, 200000, 5e-4, seed=9)
    tidx = np.arange(10001)
    inst = [(s, g, 5e-4, tidx) for s, g in zip(systems, gammas)]
    f64, s64 = build_both(inst[:8], "fp64")
    for a, b in zip(f64, s64):
        assert relerr(a, b) <= 1e-12
    f32, s32 = build_both(inst, "fp32")
    for k in range(8):
        ef, es = relerr(f32[k], f64[k]), relerr(s32[k], f64[k])
        assert ef <= 2 * es + 1e-7, (k, ef, es)


def test_fused_fcr_series_match_four_step():
    """The F/C/R series entry point (FP64 sources) through both paths."""
    osys, s, G = spin_boson_case(2500, 0.005)
    old = tb.fused_conv()
    try:
        tb.set_fused_conv(True)
        F1, C1, R1 = tb.compute_triple_kernels(s, G, 0.005)
        tb.set_fused_conv(False)
        F2, C2, R2 = tb.compute_triple_kernels(s, G, 0.005)
    finally:
        tb.set_fused_conv(old)
    for a, b in ((F1, F2), (C1, C2), (R1, R2)):
        assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(b)))
