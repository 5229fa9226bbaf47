"""The propagated generator on the device: L2(t) series, device Gamma and the example's
RK4 propagation (L0 / L2 / L2 + L4) against the CPU oracle.

Tolerances: L2 series <= 1e-13 relative; Gamma <= 1e-10 relative (the reference
accumulates the phase by a running product, the device evaluates it directly); <sigma_z>(t)
<= 1e-10 with the FP64 L4 and <= 1e-6 with the FP32 L4."""
import numpy as np
import pytest

import oracle
import taco_b200 as tb
from cases import SX, SZ, oracle_l4, relerr, spin_boson_case

pytestmark = pytest.mark.gpu


def test_tcl2_series_matches_oracle():
    osys, s, G = spin_boson_case(400, 0.005)
    tidx = np.array([0, 1, 7, 200, 400])
    L2 = tb.tcl2_generator_series(s, G, tidx)
    ref = np.stack([oracle.tcl2_total(osys, G[:, t])[0] for t in tidx])
    assert relerr(L2, ref) <= 1e-13


@pytest.mark.parametrize("nops", [1, 2])
def test_tcl2_series_random_system(nops):
    from cases import random_case
    osys, s, G = random_case(3, nops, 200, 0.01, seed=11 + nops)
    s.eps = osys.eps
    tidx = np.arange(0, 200, 17)
    L2 = tb.tcl2_generator_series(s, G, tidx)
    ref = np.stack([oracle.tcl2_total(osys, G[:, t])[0] for t in tidx])
    assert relerr(L2, ref) <= 1e-12


def test_gamma_trapz_device_matches_oracle():
    import torch
    _, C = oracle.bcf_fft(20000, 0.005, oracle.J_OHMIC, [0.05, 10.0], 1.0)
    om = np.array([-1.4142135623730951, 0.0, 1.4142135623730951])
    ref = oracle.gamma_trapz(C, 0.005, om)
    G = tb.gamma_trapz_device(torch.from_numpy(C).cuda(), 0.005, om).cpu().numpy()
    assert relerr(G, ref) <= 1e-10
    Gh = tb.gamma_trapz_device(C, 0.005, om)
    assert relerr(Gh, ref) <= 1e-10


def _oracle_propagation(osys, G, dt, steps, order, r0, obs):
    Ls = []
    L4 = oracle_l4(osys, G, dt, np.arange(steps + 1)) if order == 4 else None
    for k in range(steps + 1):
        if order == 0:
            L = oracle.unitary_superop(np.diag(osys.eps).astype(np.complex128))
        else:
            L = oracle.tcl2_total(osys, G[:, k])[0]
        if order == 4:
            L = L + L4[k]
        Ls.append(L)
    r, samples = oracle.rk4_propagate(np.stack(Ls), r0, dt, sample_every=1)
    return r, samples @ obs


@pytest.mark.parametrize("order", [0, 2, 4])
def test_propagation_config1_shape(order):
    """d=2 spin boson (eps=Delta=1, alpha=0.05, wc=10, beta=1), dt=0.005, 1000 RK4 steps from
    |0><0| in the lab basis; <sigma_z> in the lab basis."""
    osys, s, G = spin_boson_case(4000, 0.005)
    U = osys.U
    rho0 = U.conj().T @ np.array([[1, 0], [0, 0]], np.complex128) @ U
    r0 = rho0.reshape(-1, order="F")
    Oe = U.conj().T @ SZ @ U
    obs = Oe.T.reshape(-1, order="F")  # <O> = Tr(rho O) = sum_ij rho_ij O_ji
    steps = 1000
    r_ref, o_ref = _oracle_propagation(osys, G, 0.005, steps, order, r0, obs)
    o, r = tb.propagate_tcl(s, G, 0.005, steps, r0, obs=obs, order=order, sample_every=1)
    assert relerr(r, r_ref) <= 1e-10
    assert relerr(o, o_ref) <= 1e-10
    assert np.max(np.abs(o.imag)) <= 1e-10 * np.max(np.abs(o.real))
    if order == 4:
        o32, r32 = tb.propagate_tcl(s, G, 0.005, steps, r0, obs=obs, order=4, precision="fp32")
        assert relerr(o32, o_ref) <= 1e-6


def test_gamma_trapz_batch_matches_single_calls():
    import torch
    cases = [(20000, 0.005, [0.05, 10.0], 1.0, [-1.4, 0.0, 1.4]), (777, 0.01, [0.1, 3.0], 0.4, [-0.3, 0.0, 0.2, 0.5])]
    Cs, dts, oms, refs = [], [], [], []
    for N, dt, prm, beta, om in cases:
        _, C = oracle.bcf_fft(N, dt, oracle.J_OHMIC, prm, beta)
        Cs.append(torch.from_numpy(C).cuda())
        dts.append(dt)
        oms.append(np.array(om))
        refs.append(oracle.gamma_trapz(C, dt, np.array(om)))
    outs = tb.gamma_trapz_device_batch(Cs, dts, oms)
    for o, r in zip(outs, refs):
        assert relerr(o.cpu().numpy(), r) <= 1e-10
