"""Parity of the CUDA path (through the C-ABI) with the CPU oracle and the golden vectors.

Tolerances (relative Frobenius unless stated):
  plain FP64 path   L4 <= 1e-10, F/C/R <= 1e-10 of max |series|
  FP32 form         L4 <= 1e-6
  RK4 (FP64 state)  <= 1e-10 against the oracle; analytic cases <= 1e-6
"""
import os

import numpy as np
import pytest

import oracle
import taco_b200 as tb
from cases import oracle_l4, random_case, relerr, spin_boson_case

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def torch_dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def test_synthetic_gamma_triple_kernels_and_l4():
    g = np.load(os.path.join(GOLD, "synthetic_gamma.npz"))
    s = tb.System.from_arrays(int(g["N"]), g["omegas"], g["p2f"], list(g["ops"]), mirror=g["mirror"])
    dt = float(g["dt"])
    F, C, R = tb.compute_triple_kernels(s, g["gamma"], dt)
    nf = int(g["nf"])
    for a, b in ((F, g["F"]), (C, g["C"]), (R, g["R"])):
        a = a.reshape(nf ** 3, -1)
        assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, np.max(np.abs(b)))
    L4 = tb.build_correction_series(s, g["gamma"], dt)
    assert relerr(L4, g["L4_all"]) <= 1e-10
    L4s = tb.build_TCL4_generator_batch(s, g["gamma"], dt, g["tids"])
    assert relerr(L4s, g["L4_all"][g["tids"]]) <= 1e-10
    one = tb.build_TCL4_generator(s, g["gamma"], dt, 8)
    assert relerr(one, g["L4_all"][8]) <= 1e-10


def test_spin_boson_golden_end_to_end():
    g = np.load(os.path.join(GOLD, "spin_boson_small.npz"))
    s = tb.System.from_arrays(int(g["N"]), g["omegas"], g["p2f"], list(g["ops"]), mirror=g["mirror"])
    dt = float(g["dt"])
    steps = int(g["steps"])
    L4 = tb.build_TCL4_generator_batch(s, g["gamma"], dt, np.arange(steps + 1))
    assert relerr(L4, g["L4"]) <= 1e-10
    L = g["L2"] + np.asarray(L4)
    r, _, _ = tb.propagate_rk4_dense(L, g["r0"], dt)
    assert relerr(r, g["r_final"]) <= 1e-10
    r2, _, _ = tb.propagate_rk4_dense(torch_dev(g["L2"]), torch_dev(g["r0"]), dt, L_add=torch_dev(np.asarray(L4)))
    assert relerr(r2.cpu().numpy(), g["r_final"]) <= 1e-10


@pytest.mark.parametrize("device_io", [False, True])
def test_config1_shape_fp64_vs_oracle(device_io):
    """d=2 spin boson, alpha=0.05, wc=10, beta=1, dt=0.005, on a 4001-sample grid, tidx 0..1000."""
    osys, s, G = spin_boson_case(4000, 0.005)
    tidx = np.arange(1001)
    ref = oracle_l4(osys, G, 0.005, tidx)
    if device_io:
        out = tb.build_TCL4_generator_batch(s, torch_dev(G), 0.005, tidx).cpu().numpy()
    else:
        out = tb.build_TCL4_generator_batch(s, G, 0.005, tidx)
    assert relerr(out, ref) <= 1e-10


def test_fp32_form_error_bound():
    osys, s, G = spin_boson_case(4000, 0.005)
    tidx = np.arange(0, 4001, 3)
    ref = oracle_l4(osys, G, 0.005, tidx)
    out = tb.build_TCL4_generator_batch(s, G, 0.005, tidx, precision="fp32")
    assert out.dtype == np.complex64
    assert relerr(out, ref) <= 1e-6


def test_triple_kernels_match_oracle_full_series():
    osys, s, G = spin_boson_case(3000, 0.005)
    F, C, R = tb.compute_triple_kernels(s, G, 0.005)
    Fo, Co, Ro = oracle.fcr_series(G, osys.omegas, osys.mirror, 0.005)
    nf = osys.nf
    for a, b in ((F, Fo), (C, Co), (R, Ro)):
        assert relerr(a.reshape(nf ** 3, -1), b) <= 1e-10


@pytest.mark.parametrize("d,nops,Nt", [(3, 1, 700), (4, 2, 300)])
def test_random_systems_vs_oracle(d, nops, Nt):
    osys, s, G = random_case(d, nops, Nt, 0.01, seed=d)
    tidx = np.array([0, 1, Nt // 3, Nt // 2, Nt - 1, 5, 5])
    ref = oracle_l4(osys, G, 0.01, tidx)
    out = tb.build_TCL4_generator_batch(s, G, 0.01, tidx)
    assert relerr(out, ref) <= 1e-10
    out32 = tb.build_TCL4_generator_batch(s, G, 0.01, tidx, precision="fp32")
    assert relerr(out32, ref) <= 1e-6


def test_pad_factor_and_full_length_keep_results():
    osys, s, G = spin_boson_case(2000, 0.005)
    tidx = np.arange(0, 300)
    base = tb.build_TCL4_generator_batch(s, G, 0.005, tidx)
    tb.set_fcr_fft_pad_factor(8)
    try:
        padded = tb.build_TCL4_generator_batch(s, G, 0.005, tidx)
    finally:
        tb.set_fcr_fft_pad_factor(0)
    full = tb.build_TCL4_generator_batch(s, G, 0.005, tidx, full_length=True)
    assert relerr(padded, base) <= 1e-12 and relerr(full, base) <= 1e-12
    full32 = tb.build_TCL4_generator_batch(s, G, 0.005, tidx, precision="fp32", full_length=True)
    ref = oracle_l4(osys, G, 0.005, tidx)
    assert relerr(full, ref) <= 1e-10 and relerr(full32, ref) <= 1e-6


def test_plan_replay_matches_direct_call():
    import torch
    cases = [spin_boson_case(1200, 0.005, eps=e) for e in (0.8, 1.0, 1.7)]
    inst = [(s, torch_dev(G), 0.005, np.arange(0, 1201, 2)) for _, s, G in cases]
    # the FP32 pass alone: a guarded plan replays the heads its creation chose, which can
    # be shorter than those a direct call checks (both within the guard's tolerance)
    old_guard = tb.fp32_guard()
    tb.set_fp32_guard(0.0)
    direct = [x.cpu().numpy() for x in tb.build_instances(inst, precision="fp32")]
    plan = tb.Tcl4Plan(inst, precision="fp32")
    tb.set_fp32_guard(old_guard)
    n0 = tb.kernel_launches()
    for _ in range(3):
        res = plan.run()
    torch.cuda.synchronize()
    assert tb.kernel_launches() > n0
    for a, b in zip(res, direct):
        assert np.array_equal(a.cpu().numpy(), b)
    plan64 = tb.Tcl4Plan(inst, precision="fp64")
    res64 = plan64.run()
    torch.cuda.synchronize()
    for (osys, _, G), r in zip(cases, res64):
        assert relerr(r.cpu().numpy(), oracle_l4(osys, G, 0.005, np.arange(0, 1201, 2))) <= 1e-10
    plan.close()
    plan64.close()
    with pytest.raises(ValueError):
        tb.Tcl4Plan([(s, G, 0.005, None) for _, s, G in cases])


def test_plan_groups_of_several_lengths_run_as_branches():
    """Instances of four FFT lengths (and two system sizes) in one plan: the groups run as
    concurrent branches of the plan's graph, each in its own region of the work buffer.
    Every result equals the direct call's (same kernels) and matches the oracle."""
    import torch
    cases = [spin_boson_case(n, 0.005, eps=e) for n, e in ((400, 0.8), (900, 1.0), (1700, 1.7), (900, 1.3))]
    cases.append(random_case(3, 1, 700, 0.01, seed=17))
    inst = [(s, torch_dev(G), 0.005 if k < 4 else 0.01, np.arange(0, G.shape[1], 3))
            for k, (_, s, G) in enumerate(cases)]
    assert len({tb.fft_length(int(x[3].max()) + 1, "fp64")[0] for x in inst}) >= 3
    direct = [x.cpu().numpy() for x in tb.build_instances(inst, precision="fp64")]
    plan = tb.Tcl4Plan(inst, precision="fp64")
    for _ in range(2):
        res = plan.run()
    torch.cuda.synchronize()
    for (osys, _, G), x, a, b in zip(cases, inst, res, direct):
        assert np.array_equal(a.cpu().numpy(), b)
        assert relerr(b, oracle_l4(osys, G, x[2], x[3])) <= 1e-10
    plan.close()


def test_batched_instances_match_single_calls():
    cases = [spin_boson_case(1500, 0.005, eps=e, delta=dl, alpha=a) for e, dl, a in
             ((1.0, 1.0, 0.05), (0.7, 1.3, 0.1), (1.5, 0.6, 0.02))]
    cases.append(random_case(3, 1, 900, 0.01, seed=7))
    inst = []
    for k, (osys, s, G) in enumerate(cases):
        dtk = 0.01 if k == 3 else 0.005
        inst.append((s, G, dtk, np.arange(0, G.shape[1], 7 + k)))
    outs = tb.build_instances(inst)
    for (s, G, dtk, tidx), (osys, _, _), out in zip(inst, cases, outs):
        ref = oracle_l4(osys, G, dtk, tidx)
        assert relerr(out, ref) <= 1e-10
    outs32 = tb.build_instances(inst, precision="fp32")
    for (s, G, dtk, tidx), (osys, _, _), out in zip(inst, cases, outs32):
        assert relerr(out, oracle_l4(osys, G, dtk, tidx)) <= 1e-6


def test_errors_follow_reference_exceptions():
    osys, s, G = spin_boson_case(100, 0.005)
    with pytest.raises(IndexError):
        tb.build_TCL4_generator_batch(s, G, 0.005, [0, 101])
    with pytest.raises(ValueError):
        tb.build_TCL4_generator_batch(s, G, -1.0, [0])
    bad = tb.System.from_arrays(s.N, s.omegas, s.pair_to_freq, [], mirror=s.mirror)
    with pytest.raises(ValueError):
        tb.build_TCL4_generator_batch(bad, G, 0.005, [0])


def test_rk4_analytic_cases_on_device():
    """tests/rk4_dense_tests.cpp:43-101 (constant L via a constant series; L = t I with midpoints)."""
    import scipy.linalg
    L = np.zeros((4, 4), np.complex128)
    L[0, 0], L[1, 1], L[2, 2], L[3, 3] = 0.10 - 0.03j, -0.07 + 0.05j, 0.02, -0.04 - 0.02j
    L[0, 2], L[2, 0], L[1, 3] = 0.03 + 0.01j, -0.02 + 0.02j, 0.01 - 0.04j
    r0 = np.array([1.0, 0.5 - 0.2j, -0.7 + 0.1j, 0.1 + 0.3j])
    steps = 500
    r, _, _ = tb.propagate_rk4_dense(np.repeat(L[None], steps + 1, 0), r0, 0.0025)
    assert relerr(r, scipy.linalg.expm(1.25 * L) @ r0) <= 1e-6
    D, steps, dt = 3, 100, 0.01
    Ls = np.stack([i * dt * np.eye(D, dtype=np.complex128) for i in range(steps + 1)])
    Lh = np.stack([(i + 0.5) * dt * np.eye(D, dtype=np.complex128) for i in range(steps)])
    r0 = np.array([0.3 + 0.1j, -0.2 + 0.4j, 0.9 - 0.3j])
    r, _, _ = tb.propagate_rk4_dense(Ls, r0, dt, L_half=Lh)
    assert relerr(r, np.exp(0.5) * r0) <= 1e-6


@pytest.mark.parametrize("D", [4, 9, 36])
def test_rk4_vs_oracle_with_samples(D):
    rng = np.random.default_rng(D)
    steps = 257
    Ls = 0.1 * (rng.standard_normal((steps + 1, D, D)) + 1j * rng.standard_normal((steps + 1, D, D)))
    r0 = rng.standard_normal(D) + 1j * rng.standard_normal(D)
    obs = rng.standard_normal(D) + 1j * rng.standard_normal(D)
    r_ref, s_ref = oracle.rk4_propagate(Ls, r0, 0.01, sample_every=16)
    r, samples, ov = tb.propagate_rk4_dense(Ls, r0, 0.01, sample_every=16, obs=obs)
    assert relerr(r, r_ref) <= 1e-12
    assert samples.shape == s_ref.shape and relerr(samples, s_ref) <= 1e-12
    assert relerr(ov, s_ref @ obs) <= 1e-12


@pytest.mark.parametrize("tmax,nfft", [(10000, 5 << 12), (12000, 3 << 13)])
def test_mixed_radix_fft_lengths_vs_oracle(tmax, nfft):
    """The causal rule rounds 2 (tmax + 1) - 1 up to 5 * 2^k or 3 * 2^k when shorter than the
    next power of two; results match the oracle Direct method on the truncated series."""
    assert tb.fft_length(tmax + 1, "fp64")[0] == nfft
    assert tb.fft_length(tmax + 1, "fp32")[0] == nfft
    assert tb.fft_length(tmax + 1, "fp64", full_length=True)[0] == 1 << (2 * tmax + 1).bit_length()
    osys, s, G = spin_boson_case(tmax + 500, 0.005)
    Gt = np.ascontiguousarray(G[:, :tmax + 1])
    tidx = np.array([0, 1, 17, tmax // 3, tmax - 1, tmax])
    ref = oracle.tcl4_build_batch(osys.N, osys.nf, osys.omegas, osys.mirror, osys.p2f_colmajor(),
                                  osys.ops_colmajor(), Gt, 0.005, tidx=tidx, method=oracle.FCR_DIRECT)
    out = tb.build_TCL4_generator_batch(s, G, 0.005, tidx)
    assert relerr(out, ref) <= 1e-10
    out32 = tb.build_TCL4_generator_batch(s, G, 0.005, tidx, precision="fp32")
    assert relerr(out32, ref) <= 1e-6
    F, C, R = tb.compute_triple_kernels(s, Gt, 0.005)
    Fo, Co, Ro = oracle.fcr_series(Gt, osys.omegas, osys.mirror, 0.005)
    for a, b in ((F, Fo), (C, Co), (R, Ro)):
        assert relerr(a.reshape(osys.nf ** 3, -1), b) <= 1e-10


def test_pipelined_direct_build_matches_single_calls():
    """72 instances with host buffers run as sub-batches on two lanes; each result equals the
    single-instance call (same kernels; tolerance for summation order)."""
    rng = np.random.default_rng(5)
    cases = [spin_boson_case(600, 0.01, eps=rng.uniform(0.5, 2.0), delta=rng.uniform(0.5, 2.0),
                             alpha=rng.uniform(0.01, 0.1)) for _ in range(72)]
    tidx = np.arange(0, 300, 3)
    inst = [(s, G, 0.01, tidx) for (_, s, G) in cases]
    for precision, tol in (("fp64", 1e-12), ("fp32", 1e-6)):
        batch = [np.asarray(x) for x in tb.build_instances(inst, precision=precision)]
        for k in (0, 1, 35, 36, 70, 71):
            single = np.asarray(tb.build_instances([inst[k]], precision=precision)[0])
            assert relerr(batch[k], single) <= tol


def test_coefficient_cache_follows_the_coupling_operators():
    """Two systems with the same H (same frequencies and pair_to_freq) and different coupling
    operators, built in turn (and again): each result matches the oracle for its own
    operators, so the coefficient-table cache never serves another system's table."""
    osys, s, G = spin_boson_case(800, 0.01)
    A2 = np.array([[0.3, 0.8 - 0.2j], [0.8 + 0.2j, -0.3]])
    # same eigenbasis, rotated coupling: A_eig' = U^H A2 U
    A_eig2 = osys.U.conj().T @ A2 @ osys.U
    s2 = tb.System.from_arrays(osys.N, osys.omegas, osys.pair_to_freq, [A_eig2], mirror=osys.mirror, eps=osys.eps)
    tidx = np.arange(0, 400, 5)
    ref1 = oracle.tcl4_build_batch(osys.N, osys.nf, osys.omegas, osys.mirror, osys.p2f_colmajor(),
                                   osys.ops_colmajor(), G, 0.01, tidx=tidx)
    ops2 = np.ascontiguousarray(np.stack([A_eig2.T]))
    ref2 = oracle.tcl4_build_batch(osys.N, osys.nf, osys.omegas, osys.mirror, osys.p2f_colmajor(),
                                   ops2, G, 0.01, tidx=tidx)
    assert relerr(ref1, ref2) > 1e-3  # the operators matter
    for _ in range(2):
        out1, out2 = tb.build_instances([(s, G, 0.01, tidx), (s2, G, 0.01, tidx)])
        assert relerr(out1, ref1) <= 1e-10
        assert relerr(out2, ref2) <= 1e-10


def test_triple_kernels_batch_matches_single_calls():
    """compute_triple_kernels_batch (device buffers, instances of two lengths in separate
    build groups) against one compute_triple_kernels call per instance."""
    cases = [spin_boson_case(700, 0.01, eps=e, delta=dl) for e, dl in ((1.0, 1.0), (0.6, 1.4), (1.7, 0.4))]
    cases.append(random_case(3, 1, 401, 0.01, seed=3))
    gammas = [torch_dev(G) for (_, _, G) in cases]
    systems = [s for (_, s, _) in cases]
    batch = tb.compute_triple_kernels_batch(systems, gammas, 0.01)
    for s, g, out in zip(systems, gammas, batch):
        single = tb.compute_triple_kernels(s, g, 0.01)
        for a, b in zip(out, single):
            assert relerr(a.cpu().numpy(), b.cpu().numpy()) <= 1e-12


def test_shared_time_lists_match_single_calls():
    """Instances that share one time-index array (one derived time map and one upload per
    build group), instances with their own unsorted lists with repeats, and one equal list
    in a separate array: each result equals its single-instance call, in the pipelined
    (72 instances) and the single-lane (5 instances) paths.  A shared list that exceeds a
    shorter instance's gamma raises the reference's out-of-range error."""
    rng = np.random.default_rng(11)
    cases = [spin_boson_case(600, 0.01, eps=rng.uniform(0.5, 2.0), delta=rng.uniform(0.5, 2.0))
             for _ in range(72)]
    shared = np.arange(0, 300, 3)
    own = rng.integers(0, 400, 90)  # unsorted, with repeats
    equal = shared.copy()
    lists = [shared if k % 3 == 0 else (own if k % 3 == 1 else equal) for k in range(72)]
    inst = [(s, G, 0.01, lists[k]) for k, (_, s, G) in enumerate(cases)]
    for sel in (list(range(72)), [0, 1, 2, 3, 4]):
        batch = [np.asarray(x) for x in tb.build_instances([inst[k] for k in sel], precision="fp64")]
        for pos in sorted({0, 1, 2, len(sel) - 2, len(sel) - 1}):
            k = sel[pos]
            single = np.asarray(tb.build_instances([inst[k]], precision="fp64")[0])
            assert batch[pos].shape == single.shape
            assert relerr(batch[pos], single) <= 1e-12
    _, s_short, G_short = spin_boson_case(200, 0.01)
    with pytest.raises(tb.TacoOutOfRange):
        tb.build_instances([inst[0], (s_short, G_short, 0.01, shared)], precision="fp64")


def test_pipelined_slots_are_reused_safely():
    """336 host-buffer instances make seven sub-batches, more than the buffer slots of three
    lanes: the last sub-batch reuses the first one's metadata and input buffers after it has
    finished, and each lane's output staging serves its next sub-batch once the download
    has left it.  Results equal single-instance calls in the first and the last sub-batches,
    and every instance equals the others of its case."""
    rng = np.random.default_rng(21)
    cases = [spin_boson_case(400, 0.01, eps=rng.uniform(0.5, 2.0), delta=rng.uniform(0.5, 2.0))
             for _ in range(13)]
    tidx = np.arange(0, 200, 2)
    inst = [(cases[k % 13][1], cases[k % 13][2], 0.01, tidx) for k in range(336)]
    batch = [np.asarray(x) for x in tb.build_instances(inst, precision="fp32")]
    for k in (0, 5, 47, 290, 301, 335):
        single = np.asarray(tb.build_instances([inst[k]], precision="fp32")[0])
        assert relerr(batch[k], single) <= 1e-6
    # every instance (a lane's output staging is reused by its next sub-batch once the
    # previous download has left it) equals the first instance of its case
    for k in range(13, 336):
        assert relerr(batch[k], batch[k % 13]) <= 1e-6, k


def test_long_host_buckets_match_device_inputs():
    """Host gamma with buckets of 5000 consumed samples (uploaded as one plain copy per
    bucket) gives the same result as the same gamma on the device, alone and in a
    48-instance pipelined batch."""
    import torch
    osys, s, G = spin_boson_case(6000, 0.002)
    tidx = np.arange(0, 5000, 7)
    host = tb.build_TCL4_generator_batch(s, G, 0.002, tidx)
    dev = tb.build_TCL4_generator_batch(s, torch_dev(G), 0.002, tidx).cpu().numpy()
    assert np.array_equal(host, dev)
    Gd = torch_dev(G)
    outs_h = [np.asarray(x) for x in tb.build_instances([(s, G, 0.002, tidx)] * 48, precision="fp32")]
    outs_d = [x.cpu().numpy() for x in tb.build_instances([(s, Gd, 0.002, tidx)] * 48, precision="fp32")]
    torch.cuda.synchronize()
    for k in (0, 23, 47):
        assert np.array_equal(outs_h[k], outs_d[k])


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
def test_pruned_inverse_dft_schedule_matches_column_fft(precision, tol):
    """A schedule with the pruned inverse column DFT (few output rows) gives the column FFT's
    results; the default schedule uses the FFT."""
    from taco_b200 import autotune
    osys, s, G = spin_boson_case(600, 0.005)
    tidx = np.arange(0, 101)
    nfft, key = tb.fft_length(int(tidx[-1]) + 1, precision)
    old = autotune.get_schedule(key, precision)
    assert old["inv_dft_rows"] == 0
    try:
        base = tb.build_TCL4_generator_batch(s, G, 0.005, tidx, precision=precision)
        autotune.set_schedule(key, precision, old["col_tile"], old["row_tile"], old["chunk_bytes"], 16)
        dft = tb.build_TCL4_generator_batch(s, G, 0.005, tidx, precision=precision)
    finally:
        autotune.set_schedule(key, precision, old["col_tile"], old["row_tile"], old["chunk_bytes"], old["inv_dft_rows"])
    assert relerr(dft, base) <= tol
    assert relerr(dft, oracle_l4(osys, G, 0.005, tidx)) <= (1e-10 if precision == "fp64" else 1e-6)
