"""Differentiation form on the device: the bath correlation function and its parameter
derivatives, the checkpointed RK4 adjoint, the L4 and L2 adjoints, and the end-to-end
spin-boson gradient against central finite differences of the FP64 oracle.

Tolerances: BCF <= 1e-11 relative to the oracle (the oracle builds e^{-beta k dw} by a
running product); derivative spectra <= 1e-7 against central differences (step 1e-5
relative); directional derivatives of the adjoints <= 1e-7 against central differences
(step 1e-6); the end-to-end gradient <= 1e-5 relative to central differences (h = 1e-6)
of the oracle, and the FP32 precision form's gradient <= 1e-4 of the FP64 one."""
import numpy as np
import pytest

import oracle
from cases import SX, SZ, relerr

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def _adj():
    from taco_b200 import adjoint
    return adjoint


@pytest.mark.parametrize("model,prm,beta", [(0, [0.05, 10.0], 1.0), (1, [0.1, 5.0, 0.05, 2.0], 0.5),
                                            (0, [0.05, 10.0], np.inf), (0, [0.2, 3.0], 5.0)])
def test_bcf_device_matches_oracle(model, prm, beta):
    N, dt = 5000, 0.005
    _, Co = oracle.bcf_fft(N, dt, model, prm, beta)
    req = dict(model=model, which=0, alpha=prm[0], omega_c=prm[1], beta=beta, N=N, dt=dt,
               lam=prm[2] if model else 0.0, gam=prm[3] if model else 1.0)
    C = _adj().bcf_device([req], N + 1).cpu().numpy()[0]
    assert relerr(C, Co) <= 1e-11
    part = _adj().bcf_device([req], 37).cpu().numpy()[0]
    assert np.array_equal(part, C[:37])


def test_bcf_batched_lengths():
    reqs = [dict(alpha=0.05, omega_c=10.0, beta=1.0, N=n, dt=0.01) for n in (100, 1 << 12, 3)]
    for r in reqs:
        C = _adj().bcf_device([r], 4).cpu().numpy()[0]
        _, Co = oracle.bcf_fft(r["N"], 0.01, 0, [0.05, 10.0], 1.0)
        assert relerr(C, Co[:4]) <= 1e-11


@pytest.mark.parametrize("which,key", [(1, "alpha"), (2, "omega_c"), (3, "beta")])
def test_bcf_derivative_spectra_match_fd(which, key):
    N, dt = 2048, 0.01
    p = dict(alpha=0.07, omega_c=6.0, beta=0.8)
    d = _adj().bcf_device([dict(which=which, N=N, dt=dt, **p)], N + 1).cpu().numpy()[0]
    h = 1e-5 * p[key]

    def C(q):
        return oracle.bcf_fft(N, dt, 0, [q["alpha"], q["omega_c"]], q["beta"])[1]

    pp, pm = dict(p), dict(p)
    pp[key] += h
    pm[key] -= h
    fd = (C(pp) - C(pm)) / (2 * h)
    assert relerr(d, fd) <= 1e-7


def _rand_c(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("D,every", [(4, 1), (4, 6), (4, 37), (9, 5)])
def test_rk4_adjoint_matches_fd(D, every):
    torch = _torch()
    rng = np.random.default_rng(D * 100 + every)
    steps, dt = 37, 0.05
    La = 0.4 * _rand_c(rng, steps + 1, D, D)   # [t, row, col]
    Lb = 0.4 * _rand_c(rng, steps + 1, D, D)
    r0 = _rand_c(rng, D)
    ob = _rand_c(rng, D)
    w = _rand_c(rng, steps + 1)

    def loss(A, B, r, o):
        _, samp = oracle.rk4_propagate(A + B, r, dt, sample_every=1)
        return float(np.real(np.sum(np.conj(w) * (samp @ o))))

    dev = "cuda"
    cm = lambda X: torch.from_numpy(np.ascontiguousarray(np.swapaxes(X, 1, 2)).reshape(1, steps + 1, D * D)).to(dev)
    adj = _adj()
    obs, rf, ck = adj.rk4_forward_checkpointed(cm(La), cm(Lb), torch.from_numpy(r0[None]).to(dev),
                                               torch.from_numpy(ob[None]).to(dev), dt, 1, every)
    r_ref, samp = oracle.rk4_propagate(La + Lb, r0, dt, sample_every=1)
    assert relerr(obs.cpu().numpy()[0], samp @ ob) <= 1e-13
    assert relerr(rf.cpu().numpy()[0], r_ref) <= 1e-13
    Lbar, r0b, obb = adj.rk4_adjoint(cm(La), cm(Lb), torch.from_numpy(r0[None]).to(dev),
                                     torch.from_numpy(ob[None]).to(dev), dt, 1, every, ck,
                                     torch.from_numpy(w[None]).to(dev))
    Lbar = Lbar.cpu().numpy()[0].reshape(steps + 1, D, D).transpose(0, 2, 1)  # [t, row, col]
    h = 1e-6
    dL = _rand_c(rng, steps + 1, D, D)
    fd = (loss(La + h * dL, Lb, r0, ob) - loss(La - h * dL, Lb, r0, ob)) / (2 * h)
    an = float(np.real(np.sum(np.conj(Lbar) * dL)))
    assert abs(an - fd) <= 1e-7 * max(1.0, abs(fd))
    dr = _rand_c(rng, D)
    fd = (loss(La, Lb, r0 + h * dr, ob) - loss(La, Lb, r0 - h * dr, ob)) / (2 * h)
    assert abs(float(np.real(np.vdot(r0b.cpu().numpy()[0], dr))) - fd) <= 1e-7 * max(1.0, abs(fd))
    do = _rand_c(rng, D)
    fd = (loss(La, Lb, r0, ob + h * do) - loss(La, Lb, r0, ob - h * do)) / (2 * h)
    assert abs(float(np.real(np.vdot(obb.cpu().numpy()[0], do))) - fd) <= 1e-7 * max(1.0, abs(fd))


class _SysLike:
    """What oracle.tcl2_total reads from a system, with replaceable eps and operators."""

    def __init__(self, osys, eps=None, A_eig=None):
        self.N, self.nf = osys.N, osys.nf
        self.eps = np.asarray(osys.eps if eps is None else eps, np.float64)
        self.A_eig = osys.A_eig if A_eig is None else A_eig
        self._p2f = osys.p2f_colmajor()

    def p2f_colmajor(self):
        return self._p2f

    def ops_colmajor(self):
        return np.ascontiguousarray(np.stack([A.T for A in self.A_eig]), np.complex128)


def _case(d, T, seed):
    from cases import random_case, spin_boson_case
    if d == 2:
        osys, s, G = spin_boson_case(400, 0.01, eps=0.8, delta=1.3, alpha=0.08, wc=5.0, beta=0.7)
    else:
        osys, s, G = random_case(d, 1, 400, 0.01, seed)
        s.eps = osys.eps
    return osys, s, np.ascontiguousarray(G[:, :T])


@pytest.mark.parametrize("d,T", [(2, 48), (3, 20)])
def test_tcl4_adjoint_matches_fd(d, T):
    torch = _torch()
    rng = np.random.default_rng(7 + d)
    osys, s, G = _case(d, T, 21)
    dt = 0.01
    N2 = d * d
    W = _rand_c(rng, T, N2, N2)

    def l4loss(Gm, om, ops):
        L4 = oracle.tcl4_build_batch(osys.N, osys.nf, om, osys.mirror, osys.p2f_colmajor(), ops, Gm, dt,
                                     tidx=np.arange(T))
        return float(np.real(np.sum(np.conj(W) * L4)))

    import taco_b200 as tb
    Gd = torch.from_numpy(G).cuda()
    Lbar = torch.from_numpy(np.ascontiguousarray(W.transpose(0, 2, 1)).reshape(1, T, N2 * N2)).cuda()
    src = [tb.compute_triple_kernels(s, Gd, dt)]
    gbar, wbar, ops = _adj().tcl4_adjoint([s], [Gd], dt, Lbar, src, want_ops=True)
    gbar = gbar[0].cpu().numpy()
    h = 1e-6
    ops0 = osys.ops_colmajor()
    dG = _rand_c(rng, *G.shape)
    fd = (l4loss(G + h * dG, osys.omegas, ops0) - l4loss(G - h * dG, osys.omegas, ops0)) / (2 * h)
    an = float(np.real(np.sum(np.conj(gbar) * dG)))
    assert abs(an - fd) <= 1e-7 * max(1.0, abs(fd)), (an, fd)
    dw = rng.standard_normal(osys.nf)
    fd = (l4loss(G, osys.omegas + h * dw, ops0) - l4loss(G, osys.omegas - h * dw, ops0)) / (2 * h)
    assert abs(float(wbar[0] @ dw) - fd) <= 1e-7 * max(1.0, abs(fd)), (wbar[0] @ dw, fd)
    dA = _rand_c(rng, 1, d, d)
    dAc = np.ascontiguousarray(np.transpose(dA, (0, 2, 1)))
    fd = (l4loss(G, osys.omegas, ops0 + h * dAc) - l4loss(G, osys.omegas, ops0 - h * dAc)) / (2 * h)
    an = float(np.real(np.sum(np.conj(ops[0]) * dA)))
    assert abs(an - fd) <= 1e-7 * max(1.0, abs(fd)), (an, fd)


@pytest.mark.parametrize("d,T", [(2, 30), (3, 12)])
def test_tcl2_adjoint_matches_fd(d, T):
    torch = _torch()
    rng = np.random.default_rng(17 + d)
    osys, s, G = _case(d, T, 23)
    N2 = d * d
    W = _rand_c(rng, T, N2, N2)

    def l2loss(Gm, sl):
        L2 = np.stack([oracle.tcl2_total(sl, Gm[:, t])[0] for t in range(T)])
        return float(np.real(np.sum(np.conj(W) * L2)))

    Gd = torch.from_numpy(G).cuda()
    Lbar = torch.from_numpy(np.ascontiguousarray(W.transpose(0, 2, 1)).reshape(1, T, N2 * N2)).cuda()
    gbar, ops, eps_bar = _adj().tcl2_adjoint([s], [Gd], Lbar)
    gbar = gbar[0].cpu().numpy()
    h = 1e-6
    base = _SysLike(osys)
    dG = _rand_c(rng, *G.shape)
    fd = (l2loss(G + h * dG, base) - l2loss(G - h * dG, base)) / (2 * h)
    assert abs(float(np.real(np.sum(np.conj(gbar) * dG))) - fd) <= 1e-7 * max(1.0, abs(fd))
    de = rng.standard_normal(d)
    fd = (l2loss(G, _SysLike(osys, eps=osys.eps + h * de)) - l2loss(G, _SysLike(osys, eps=osys.eps - h * de))) / (2 * h)
    assert abs(float(eps_bar[0] @ de) - fd) <= 1e-7 * max(1.0, abs(fd))
    dA = _rand_c(rng, d, d)
    fd = (l2loss(G, _SysLike(osys, A_eig=[osys.A_eig[0] + h * dA]))
          - l2loss(G, _SysLike(osys, A_eig=[osys.A_eig[0] - h * dA]))) / (2 * h)
    an = float(np.real(np.sum(np.conj(ops[0][0]) * dA)))
    assert abs(an - fd) <= 1e-7 * max(1.0, abs(fd)), (an, fd)


def oracle_spin_boson_obs(p, cfg):
    return oracle.spin_boson_trajectory(p, cfg.N, cfg.dt, cfg.steps, cfg.rho0, cfg.observable, cfg.sample_every)


def test_spin_boson_gradient_matches_oracle_fd():
    adj = _adj()
    cfg = adj.SpinBosonConfig(N=1 << 11, dt=0.01, steps=96)
    params = np.array([[1.0, 0.7, 0.08, 6.0, 0.9], [0.6, 1.4, 0.03, 12.0, 2.5]])
    rng = np.random.default_rng(5)
    tgt = np.cos(0.9 * np.arange(cfg.n_samples) * cfg.dt)[None, :] * 0.8 + 0.05 * rng.standard_normal((2, cfg.n_samples))
    obs, _ = adj.spin_boson_forward(params, cfg)
    for b in range(2):
        assert relerr(obs.cpu().numpy()[b], oracle_spin_boson_obs(params[b], cfg)) <= 1e-10
    loss, grads = adj.mse_loss_and_grad(params, tgt, cfg)
    h = 1e-6
    for b in range(2):
        fd = np.zeros(5)
        for k in range(5):
            pp, pm = params[b].copy(), params[b].copy()
            pp[k] += h
            pm[k] -= h
            lp = np.mean((oracle_spin_boson_obs(pp, cfg) - tgt[b]) ** 2)
            lm = np.mean((oracle_spin_boson_obs(pm, cfg) - tgt[b]) ** 2)
            fd[k] = (lp - lm) / (2 * h)
        assert np.linalg.norm(grads[b] - fd) <= 1e-5 * np.linalg.norm(fd), (grads[b], fd)
        assert np.all(np.abs(grads[b] - fd) <= 1e-5 * np.abs(fd) + 1e-9), (grads[b], fd)
    cfg32 = adj.SpinBosonConfig(N=1 << 11, dt=0.01, steps=96, precision="fp32")
    _, g32 = adj.mse_loss_and_grad(params, tgt, cfg32)
    assert np.linalg.norm(g32 - grads) <= 1e-4 * np.linalg.norm(grads)


def test_autograd_function_matches_direct_gradient():
    torch = _torch()
    adj = _adj()
    cfg = adj.SpinBosonConfig(N=1 << 10, dt=0.01, steps=40)
    params = torch.tensor([[1.0, 0.7, 0.08, 6.0, 0.9]], dtype=torch.float64, requires_grad=True)
    tgt = torch.full((1, cfg.n_samples), 0.3, dtype=torch.float64)
    obs = adj.SpinBosonTCL4.apply(params, cfg)
    loss = ((obs - tgt) ** 2).mean()
    loss.backward()
    _, g = adj.mse_loss_and_grad(params.detach().numpy(), tgt.cpu().numpy(), cfg)
    assert np.allclose(params.grad.numpy(), g, rtol=1e-12, atol=1e-15)
