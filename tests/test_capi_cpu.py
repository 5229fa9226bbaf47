"""CPU-side checks of the product library: it loads, exports every symbol the header
declares, its host logic (coefficient table, argument checks) is right, and device
entry points fail loudly without a GPU (no CPU fallback)."""
import os
import re

import numpy as np
import pytest

import oracle
import taco_b200 as tb
from taco_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "taco_b200.h")).read()
    declared = set(re.findall(r"^(?:int|void|size_t|const char\*)\s+(taco_\w+)\(", hdr, re.M))
    assert declared == set(_capi.EXPORTED)
    L = _capi.lib()
    for name in declared:
        assert hasattr(L, name), name
    assert tb.version() == "0.1.0"


def test_pad_factor_roundtrip():
    tb.set_fcr_fft_pad_factor(4)
    assert tb.get_fcr_fft_pad_factor() == 4
    tb.set_fcr_fft_pad_factor(0)
    assert tb.get_fcr_fft_pad_factor() == 0


def test_fp32_guard_setting_roundtrip():
    old = tb.fp32_guard()
    assert old == pytest.approx(5e-7)
    tb.set_fp32_guard(1e-6)
    assert tb.fp32_guard() == pytest.approx(1e-6)
    tb.set_fp32_guard(0.0)  # off
    assert tb.fp32_guard() == 0.0
    with pytest.raises(ValueError):
        tb.set_fp32_guard(-1.0)
    with pytest.raises(ValueError):
        tb.set_fp32_guard(float("nan"))
    tb.set_fp32_guard(old)
    assert tb.fp32_guard() == old


def test_fused_conv_setting_roundtrip():
    assert tb.fused_conv() is False  # the four-step passes are the default
    tb.set_fused_conv(True)
    assert tb.fused_conv() is True
    tb.set_fused_conv(False)
    assert tb.fused_conv() is False


def _synthetic_system():
    g = np.load(os.path.join(GOLD, "synthetic_gamma.npz"))
    s = tb.System.from_arrays(int(g["N"]), g["omegas"], g["p2f"], list(g["ops"]), mirror=g["mirror"])
    return g, s


def _apply_coef(rp, src, coef, V):
    E = rp.size - 1
    out = np.zeros((V.shape[1], E), np.complex128)
    for e in range(E):
        for k in range(rp[e], rp[e + 1]):
            x = V[src[k] & 0x7FFFFFFF]
            out[:, e] += coef[k] * (np.conj(x) if src[k] >> 31 else x)
    return out


def test_l4_coefficients_reproduce_golden_l4():
    g, s = _synthetic_system()
    rp, src, coef = tb.l4_coefficients(s)
    V = np.concatenate([g["F"], g["C"], g["R"]])
    L4 = _apply_coef(rp, src, coef, V).reshape(-1, 4, 4).transpose(0, 2, 1)
    assert np.linalg.norm(L4 - g["L4_all"]) <= 1e-14 * np.linalg.norm(g["L4_all"])


@pytest.mark.parametrize("d,nops", [(3, 1), (4, 2)])
def test_l4_coefficients_match_oracle_random_systems(d, nops):
    rng = np.random.default_rng(d)
    X = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    H = (X + X.conj().T) / 2
    As = []
    for _ in range(nops):
        Y = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
        As.append((Y + Y.conj().T) / 2)
    s = tb.System(H, As)
    Nt, dt = 12, 0.05
    gamma = rng.standard_normal((s.nf, Nt)) + 1j * rng.standard_normal((s.nf, Nt))
    F, C, R = oracle.fcr_series(gamma, s.omegas, s.mirror, dt)
    ops = np.ascontiguousarray(np.stack([A.T for A in s.A_eig]))
    p2f = np.ascontiguousarray(s.pair_to_freq.T, np.int32)
    L4o = oracle.tcl4_build_batch(d, s.nf, s.omegas, s.mirror, p2f, ops, gamma, dt)
    rp, src, coef = tb.l4_coefficients(s)
    L4 = _apply_coef(rp, src, coef, np.concatenate([F, C, R])).reshape(Nt, d * d, d * d).transpose(0, 2, 1)
    assert np.linalg.norm(L4 - L4o) <= 1e-12 * np.linalg.norm(L4o)


def test_host_system_matches_oracle_system():
    H = 0.5 * tb.inputs.SZ + 0.5 * tb.inputs.SX
    s = tb.System(H, [tb.inputs.SZ])
    o = oracle.System(H, [tb.inputs.SZ])
    assert np.allclose(s.eps, o.eps, atol=1e-14) and np.allclose(s.omegas, o.omegas, atol=1e-14)
    assert (s.pair_to_freq == o.pair_to_freq).all() and (s.mirror == o.mirror).all()
    assert np.allclose(s.A_eig[0], o.A_eig[0], atol=1e-13)


def test_host_bcf_and_gamma_match_oracle():
    J = tb.inputs.ohmic(0.05, 10.0)
    t, C = tb.bcf_fft(500, 0.005, J, 1.0)
    t2, C2 = oracle.bcf_fft(500, 0.005, oracle.J_OHMIC, [0.05, 10.0], 1.0)
    assert np.linalg.norm(C - C2) <= 1e-12 * np.linalg.norm(C2)
    om = [-1.0, 0.0, 1.0]
    G = tb.gamma_trapz(C, 0.005, om)
    G2 = oracle.gamma_trapz(C2, 0.005, om)
    assert np.linalg.norm(G - G2) <= 1e-12 * np.linalg.norm(G2)


def test_l4_coefficients_reject_missing_bucket():
    g, s = _synthetic_system()
    s.pair_to_freq = s.pair_to_freq.copy()
    s.pair_to_freq[0, 1] = -1
    with pytest.raises(tb.TacoError) as ei:
        tb.l4_coefficients(s)
    assert ei.value.code == _capi.TACO_ERR_RUNTIME


def test_direct_method_rejected_like_reference():
    g, s = _synthetic_system()
    with pytest.raises(ValueError):
        tb.build_TCL4_generator_batch(s, g["gamma"], float(g["dt"]), [0], method=1)


@pytest.mark.skipif(tb.device_count() > 0, reason="checks the no-GPU behaviour")
def test_device_entry_points_fail_loudly_without_gpu():
    g, s = _synthetic_system()
    with pytest.raises(tb.TacoError) as ei:
        tb.build_TCL4_generator_batch(s, g["gamma"], float(g["dt"]), [0, 1])
    assert ei.value.code == _capi.TACO_ERR_NO_DEVICE
    with pytest.raises(tb.TacoError):
        tb.compute_triple_kernels(s, g["gamma"], float(g["dt"]))
    with pytest.raises(tb.TacoError):
        tb.propagate_rk4_dense(np.zeros((3, 2, 2)), np.zeros(2), 0.1)


def test_system_views_are_reused_only_while_unchanged():
    """The Python marshalling reuses a System's packed view while its arrays keep their
    bytes, types and shapes, and rebuilds it after an in-place change or a replaced array;
    marshalled instances name the same time-index array once."""
    s = tb.spin_boson_system(1.0, 0.7)
    v1 = tb._system_view(s)
    assert tb._system_view(s) is v1
    s.omegas[0] += 0.25  # in place
    v2 = tb._system_view(s)
    assert v2 is not v1 and v2.omegas[0] == s.omegas[0]
    s.A_eig = [A.copy() * 2.0 for A in s.A_eig]  # replaced, new contents
    v3 = tb._system_view(s)
    assert v3 is not v2 and np.allclose(v3.ops[0], np.asarray(s.A_eig[0]).T)
    s.mirror = s.mirror.astype(np.int64)  # same values, another type
    assert tb._system_view(s) is not v3
    # addresses: writable, read-only and empty arrays
    for a in (np.arange(6.0), np.arange(6.0)[::2].copy(), np.zeros(0)):
        assert tb._addr(a) == a.__array_interface__["data"][0]
    r = np.arange(4.0)
    r.flags.writeable = False
    assert tb._addr(r) == r.__array_interface__["data"][0]
    tidx = np.arange(0, 40, 4, dtype=np.uint32)
    g = np.zeros((s.nf, 50), np.complex128)
    outs = [np.empty((tidx.size, s.N ** 4), np.complex64) for _ in range(3)]
    arr, keep, res, dev = tb._instance_array([(s, g, 0.1, tidx)] * 3, _capi.TACO_PREC_FP32, outs)
    assert not dev and len({arr[k].tidx for k in range(3)}) == 1 and arr[0].T == tidx.size
    assert [arr[k].L4_out for k in range(3)] == [tb._addr(o) for o in outs]


def test_committed_tuning_table_is_applied():
    """Every tile schedule of taco_b200/tuning.json is in effect after import (entries that
    carry only the radix choice leave the tiles alone)."""
    import json
    import os
    from taco_b200 import autotune
    path = os.path.join(os.path.dirname(tb.__file__), "tuning.json")
    with open(path) as f:
        table = json.load(f)
    tb.version()  # loads the library and applies the table
    n = 0
    for key, sch in table.items():
        if key.startswith("_") or "col_tile" not in sch:
            continue
        L, prec = key.split(":")
        got = autotune.get_schedule(int(L), prec)
        for k in ("col_tile", "row_tile", "chunk_bytes", "inv_dft_rows"):
            assert got[k] == sch[k], (key, k)
        n += 1
    assert n >= 10  # the batching form's lengths 2^15..2^19 and the headline's, in both precisions
