"""Differentiation form: the hand-written adjoint of the propagated TCL4 path.

Forward (all on the device, FP64 unless ``precision="fp32"`` selects the FP32 L4 build):

    (eps, Delta) -> H = eps/2 sz + Delta/2 sx -> eigensystem, Bohr buckets, A_eig
    (alpha, wc, beta) -> C(t) (bcf_fft on the device) -> Gamma_b(t) (trapezoid)
    Gamma -> L4(t) (build_TCL4_generator_cuda_fused_batch) and L2(t) (TCL2 total())
    rho(t): RK4 under L = L2 + L4 (the reference example's order-4 propagation,
    examples/TCL4_spin_boson_example.cpp:317-394), <O(t)> sampled every step.

Reverse (the adjoint; every gradient G(z) = dl/dRe z + i dl/dIm z):

    G(<O>) -> RK4 adjoint with sqrt(steps) checkpoints -> G(L(t))
    G(L4(t)) -> sources F/C/R -> G(Gamma), dl/domega_b, G(A_eig)   (taco_tcl4_adjoint)
    G(L2(t)) -> G(Gamma), G(A_eig), dl/deps                          (taco_tcl2_adjoint)
    G(Gamma) . dGamma/d(alpha, wc, beta): tangent correlation functions dC/dtheta from
      the device BCF and their trapezoid integrals; dGamma_b/domega_b the same with
      i tau C(tau)
    eigensystem: first-order perturbation of eigenvalues and eigenvectors for dH/deps =
      sz/2, dH/dDelta = sx/2 (the loss is invariant under eigenvector phases).

``SpinBosonTCL4`` wraps this in a torch.autograd.Function: params [B, 5] (eps, Delta,
alpha, wc, beta) -> <O(t)> [B, n_samples]; any torch loss of the trajectories then
backpropagates to the parameters.  The reference has no derivatives; these entry points
have no counterpart there.
"""
from __future__ import annotations

import contextlib
import ctypes as ct
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import _capi
from .inputs import SX, SZ, System

PARAMS = ("eps", "delta", "alpha", "omega_c", "beta")


def _torch():
    import torch
    return torch


def _p(x):
    return None if x is None else ct.c_void_p(x.data_ptr())


def _stream(dev):
    return ct.c_void_p(_torch().cuda.current_stream(dev).cuda_stream)


# ------------------------------------------------------------------ BCF --
def bcf_device(reqs, n_out: int, device="cuda"):
    """C(t_k) (or a derivative), k < n_out, for each request dict(model, which, alpha,
    omega_c, beta, N, dt[, lam, gam]): complex128 tensor [len(reqs), n_out] on the device."""
    torch = _torch()
    out = torch.empty((len(reqs), n_out), dtype=torch.complex128, device=device)
    arr = (_capi.BcfRequest * len(reqs))()
    for k, r in enumerate(reqs):
        arr[k].model = int(r.get("model", 0))
        arr[k].which = int(r.get("which", 0))
        arr[k].alpha = float(r["alpha"])
        arr[k].omega_c = float(r["omega_c"])
        arr[k].lam = float(r.get("lam", 0.0))
        arr[k].gam = float(r.get("gam", 1.0))
        arr[k].beta = float(r["beta"])
        arr[k].N = int(r["N"])
        arr[k].dt = float(r["dt"])
        arr[k].out = out[k].data_ptr()
        arr[k].n_out = int(n_out)
    _capi.check(_capi.lib().taco_bcf_fft(arr, len(reqs), _capi.TACO_OUT_DEVICE, _stream(out.device)))
    return out


# ------------------------------------------------------------------ RK4 --
def rk4_forward_checkpointed(L, L_add, r0, obs, dt, sample_every, every):
    """Batched checkpointed RK4: L, L_add [B, steps+1, D*D] column-major matrices (complex128),
    r0, obs [B, D].  Returns (obs_out [B, n_samples], r_final [B, D], ckpt [B, n_ckpt, D])."""
    torch = _torch()
    B, T, E = L.shape
    D = int(round(math.sqrt(E)))
    steps = T - 1
    ns = (steps + sample_every - 1) // sample_every + 1
    nck = (steps + every - 1) // every
    dev = L.device
    obs_out = torch.empty((B, ns), dtype=torch.complex128, device=dev)
    r_out = torch.empty((B, D), dtype=torch.complex128, device=dev)
    ckpt = torch.empty((B, nck, D), dtype=torch.complex128, device=dev)
    jobs = (_capi.Rk4GradJob * B)()
    for b in range(B):
        j = jobs[b]
        j.L = L[b].data_ptr()
        j.L_add = L_add[b].data_ptr() if L_add is not None else None
        j.steps = steps
        j.D = D
        j.dt = float(dt)
        j.r0 = r0[b].data_ptr()
        j.obs = obs[b].data_ptr()
        j.sample_every = sample_every
        j.ckpt = ckpt[b].data_ptr()
        j.obs_out = obs_out[b].data_ptr()
        j.r_out = r_out[b].data_ptr()
    _capi.check(_capi.lib().taco_rk4_forward_checkpointed(jobs, B, every, _stream(dev)))
    return obs_out, r_out, ckpt


def rk4_adjoint(L, L_add, r0, obs, dt, sample_every, every, ckpt, obs_bar, r_final_bar=None):
    """Reverse sweep of rk4_forward_checkpointed: returns (L_bar [B, steps+1, D*D], r0_bar [B, D],
    obs_vec_bar [B, D])."""
    torch = _torch()
    B, T, E = L.shape
    D = int(round(math.sqrt(E)))
    dev = L.device
    L_bar = torch.empty((B, T, E), dtype=torch.complex128, device=dev)
    r0_bar = torch.empty((B, D), dtype=torch.complex128, device=dev)
    ob_bar = torch.empty((B, D), dtype=torch.complex128, device=dev)
    obs_bar = obs_bar.to(torch.complex128).contiguous()
    jobs = (_capi.Rk4GradJob * B)()
    for b in range(B):
        j = jobs[b]
        j.L = L[b].data_ptr()
        j.L_add = L_add[b].data_ptr() if L_add is not None else None
        j.steps = T - 1
        j.D = D
        j.dt = float(dt)
        j.r0 = r0[b].data_ptr()
        j.obs = obs[b].data_ptr()
        j.sample_every = sample_every
        j.ckpt = ckpt[b].data_ptr()
        j.obs_bar = obs_bar[b].data_ptr()
        j.r_final_bar = r_final_bar[b].data_ptr() if r_final_bar is not None else None
        j.L_bar = L_bar[b].data_ptr()
        j.r0_bar = r0_bar[b].data_ptr()
        j.obs_vec_bar = ob_bar[b].data_ptr()
    _capi.check(_capi.lib().taco_rk4_adjoint(jobs, B, every, _stream(dev)))
    return L_bar, r0_bar, ob_bar


# ------------------------------------------------------ generator adjoints --
class _Views:
    """taco_system_view structs (and their buffers) for a list of systems."""

    def __init__(self, systems):
        from . import _View
        self.views = [_View(s) for s in systems]


def tcl4_adjoint(systems, gammas, dt, L_bar, sources=None, want_ops=False):
    """Adjoint of L4(t), t < T, for each instance.  gammas: list of [nf, T] complex128 device
    tensors; L_bar [B, T, N^4] (column-major entries); sources: list of (F, C, R) device
    tensors [nf, nf, nf, T] (needed for the A_eig gradient).  Returns (gamma_bar list,
    omega_bar [B, nf] numpy, ops_bar list of [num_ops, N, N] numpy or None)."""
    torch = _torch()
    B = len(systems)
    vs = _Views(systems)
    gbar = [torch.zeros_like(g) for g in gammas]
    wbar = [np.zeros(int(s.nf), np.float64) for s in systems]
    obar = [np.zeros((len(s.A_eig), int(s.N) * int(s.N)), np.complex128) for s in systems]
    jobs = (_capi.Tcl4AdjointJob * B)()
    for b in range(B):
        j = jobs[b]
        j.sys = ct.pointer(vs.views[b].view)
        j.gamma = gammas[b].data_ptr()
        j.T = gammas[b].shape[1]
        j.dt = float(dt)
        j.L_bar = L_bar[b].data_ptr()
        if want_ops and sources is not None:
            F, C, R = sources[b]
            j.F, j.C, j.R = F.data_ptr(), C.data_ptr(), R.data_ptr()
            j.ops_bar = obar[b].ctypes.data
        j.gamma_bar = gbar[b].data_ptr()
        j.omega_bar = wbar[b].ctypes.data
    _capi.check(_capi.lib().taco_tcl4_adjoint(jobs, B, _stream(L_bar.device)))
    ops = [o.reshape(-1, int(s.N), int(s.N)).transpose(0, 2, 1) for o, s in zip(obar, systems)] if want_ops else None
    return gbar, np.stack(wbar), ops


def tcl2_adjoint(systems, gammas, L_bar, gamma_bar=None):
    """Adjoint of the TCL2 series L2(t), t < T.  Accumulates into gamma_bar (a list of [nf, T]
    device tensors, created when None).  Returns (gamma_bar, ops_bar list [num_ops, N, N],
    eps_bar [B, N])."""
    torch = _torch()
    B = len(systems)
    vs = _Views(systems)
    if gamma_bar is None:
        gamma_bar = [torch.zeros_like(g) for g in gammas]
    obar = [np.zeros((len(s.A_eig), int(s.N) * int(s.N)), np.complex128) for s in systems]
    ebar = [np.zeros(int(s.N), np.float64) for s in systems]
    epss = [np.ascontiguousarray(s.eps, np.float64) for s in systems]
    jobs = (_capi.Tcl2AdjointJob * B)()
    for b in range(B):
        j = jobs[b]
        j.sys = ct.pointer(vs.views[b].view)
        j.eps = epss[b].ctypes.data
        j.gamma = gammas[b].data_ptr()
        j.T = gammas[b].shape[1]
        j.L_bar = L_bar[b].data_ptr()
        j.gamma_bar = gamma_bar[b].data_ptr()
        j.ops_bar = obar[b].ctypes.data
        j.eps_bar = ebar[b].ctypes.data
    _capi.check(_capi.lib().taco_tcl2_adjoint(jobs, B, _stream(L_bar.device)))
    ops = [o.reshape(-1, int(s.N), int(s.N)).transpose(0, 2, 1) for o, s in zip(obar, systems)]
    return gamma_bar, ops, np.stack(ebar)


def inner_re(pairs, device):
    """[sum Re(conj(a) b) for (a, b) in pairs] over device tensors, one launch."""
    out = np.zeros(len(pairs), np.float64)
    if not pairs:
        return out
    jobs = (_capi.InnerJob * len(pairs))()
    for k, (a, b) in enumerate(pairs):
        jobs[k].a = a.data_ptr()
        jobs[k].b = b.data_ptr()
        jobs[k].n = a.numel()
    _capi.check(_capi.lib().taco_inner_re(jobs, len(pairs), out.ctypes.data_as(ct.c_void_p), _stream(device)))
    return out


# -------------------------------------------------------------- eigensystem --
def eig_tangent(U, lam, dH):
    """First-order change of eigenvalues and eigenvectors of H = U diag(lam) U^H along dH:
    (dlam, dU) with dU = U K, K_ij = (U^H dH U)_ij / (lam_j - lam_i) (i != j), K_ii = 0."""
    V = U.conj().T @ dH @ U
    dlam = np.real(np.diag(V))
    gap = lam[None, :] - lam[:, None]
    K = np.where(np.eye(lam.size, dtype=bool), 0.0, V / np.where(gap == 0, np.inf, gap))
    return dlam, U @ K


def grad_U_from_rotated(X, GX, U):
    """G(U) of X_eig = U^H X U given G(X_eig)."""
    return X @ U @ GX.conj().T + X.conj().T @ U @ GX


# ------------------------------------------------------------------ model --
@dataclass
class SpinBosonConfig:
    """Differentiation-form workload: spin boson H = eps/2 sz + Delta/2 sx, A = sz, Ohmic
    J = alpha w e^{-w/wc}; grid N (N + 1 bath samples), step dt; `steps` RK4 steps from
    rho0 (lab basis), <O> (lab basis) sampled every `sample_every` steps."""
    N: int = 1 << 16
    dt: float = 1e-3
    steps: int = 4096
    sample_every: int = 1
    precision: str = "fp64"
    checkpoint_every: int = 0  # 0: ceil(sqrt(steps))
    rho0: np.ndarray = field(default_factory=lambda: np.array([[1, 0], [0, 0]], np.complex128))
    observable: np.ndarray = field(default_factory=lambda: SZ.copy())
    coupling: np.ndarray = field(default_factory=lambda: SZ.copy())

    @property
    def every(self):
        return self.checkpoint_every or max(1, int(math.ceil(math.sqrt(self.steps))))

    @property
    def n_samples(self):
        return (self.steps + self.sample_every - 1) // self.sample_every + 1


class Phases:
    """Host wall time per phase (each phase ends with a device synchronisation)."""

    def __init__(self):
        self.ms = {}

    @contextlib.contextmanager
    def __call__(self, name):
        torch = _torch()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        yield
        torch.cuda.synchronize()
        self.ms[name] = self.ms.get(name, 0.0) + (time.perf_counter() - t0) * 1e3


def _phase(phases, name):
    return phases(name) if phases is not None else contextlib.nullcontext()


def _systems(params, cfg):
    out = []
    for eps, delta, *_ in params:
        s = System(0.5 * eps * SZ + 0.5 * delta * SX, [cfg.coupling])
        out.append(s)
    return out


def spin_boson_forward(params, cfg: SpinBosonConfig, device="cuda", phases=None):
    """<O(t)> [B, n_samples] (real, torch float64 on the device) and the saved state."""
    from . import build_instances, gamma_trapz_device_batch, tcl2_generator_series
    torch = _torch()
    params = np.asarray(params, np.float64).reshape(-1, 5)
    B = params.shape[0]
    T = cfg.steps + 1
    if T > cfg.N + 1:
        raise ValueError("steps must not exceed the bath grid N")
    with _phase(phases, "system"):
        systems = _systems(params, cfg)
    nf = systems[0].nf
    if any(s.nf != nf for s in systems):
        raise ValueError("all instances must share the Bohr-bucket count")
    reqs = [dict(model=0, which=0, alpha=a, omega_c=wc, beta=be, N=cfg.N, dt=cfg.dt)
            for (_, _, a, wc, be) in params]
    with _phase(phases, "bcf"):
        C = bcf_device(reqs, T, device)
    with _phase(phases, "gamma"):
        gammas = gamma_trapz_device_batch([C[b] for b in range(B)], [cfg.dt] * B, [s.omegas for s in systems])
    N2 = systems[0].N ** 2
    E = N2 * N2
    cdt = torch.complex128 if cfg.precision == "fp64" else torch.complex64
    with _phase(phases, "l4"):
        outs = [torch.empty((T, E), dtype=cdt, device=device) for _ in range(B)]
        build_instances([(systems[b], gammas[b], cfg.dt, np.arange(T)) for b in range(B)], precision=cfg.precision,
                        outs=outs)
        L4 = torch.stack([o.to(torch.complex128) for o in outs])
    with _phase(phases, "l2"):
        L2 = torch.stack([tcl2_generator_series(systems[b], gammas[b]).transpose(1, 2).reshape(T, E)
                          for b in range(B)]).contiguous()
    with _phase(phases, "rk4"):
        r0 = np.stack([(s.U.conj().T @ cfg.rho0 @ s.U).reshape(-1, order="F") for s in systems])
        ov = np.stack([(s.U.conj().T @ cfg.observable @ s.U).T.reshape(-1, order="F") for s in systems])
        r0_d = torch.from_numpy(r0).to(device)
        ov_d = torch.from_numpy(ov).to(device)
        obs, _, ckpt = rk4_forward_checkpointed(L2, L4, r0_d, ov_d, cfg.dt, cfg.sample_every, cfg.every)
    state = dict(params=params, systems=systems, C=C, gammas=gammas, L2=L2, L4=L4, r0=r0_d, ov=ov_d, ckpt=ckpt)
    return obs.real.contiguous(), state


def spin_boson_backward(state, g_obs, cfg: SpinBosonConfig, phases=None):
    """d(loss)/d(eps, Delta, alpha, wc, beta) [B, 5] from g_obs = d(loss)/d<O(t)> [B, n_samples]."""
    from . import compute_triple_kernels_batch, gamma_trapz_device_batch
    torch = _torch()
    params, systems = state["params"], state["systems"]
    B = params.shape[0]
    dev = state["L2"].device
    T = cfg.steps + 1
    dt = cfg.dt
    obs_bar = g_obs.to(device=dev, dtype=torch.float64).to(torch.complex128)
    with _phase(phases, "rk4_adjoint"):
        L_bar, r0_bar, ov_bar = rk4_adjoint(state["L2"], state["L4"], state["r0"], state["ov"], dt,
                                            cfg.sample_every, cfg.every, state["ckpt"], obs_bar)
    gammas = state["gammas"]
    with _phase(phases, "fcr_sources"):
        sources = compute_triple_kernels_batch(systems, gammas, dt)
    with _phase(phases, "l4_adjoint"):
        gbar, wbar, ops4 = tcl4_adjoint(systems, gammas, dt, L_bar, sources, want_ops=True)
    with _phase(phases, "l2_adjoint"):
        gbar, ops2, eps_bar = tcl2_adjoint(systems, gammas, L_bar, gbar)
    # tangents of Gamma: bath parameters (BCF derivative spectra) and the bucket frequency
    reqs = []
    for (_, _, a, wc, be) in params:
        for which in (1, 2, 3):
            reqs.append(dict(model=0, which=which, alpha=a, omega_c=wc, beta=be, N=cfg.N, dt=dt))
    with _phase(phases, "bath_tangents"):
        dC = bcf_device(reqs, T, dev).view(B, 3, T)
        tau = torch.arange(T, dtype=torch.float64, device=dev) * dt
        srcs, oms = [], []
        for b in range(B):
            for k in range(3):
                srcs.append(dC[b, k])
                oms.append(systems[b].omegas)
            srcs.append(1j * tau * state["C"][b])
            oms.append(systems[b].omegas)
        tg = gamma_trapz_device_batch(srcs, [dt] * len(srcs), oms)
        pairs = []
        for b in range(B):
            for k in range(3):
                pairs.append((gbar[b], tg[4 * b + k]))
            gw = tg[4 * b + 3]
            for j in range(systems[b].nf):
                pairs.append((gbar[b][j].contiguous(), gw[j].contiguous()))
        dots = inner_re(pairs, dev)
    grads = np.zeros((B, 5), np.float64)
    r0b = r0_bar.cpu().numpy()
    ovb = ov_bar.cpu().numpy()
    pos = 0
    for b in range(B):
        s = systems[b]
        N = s.N
        nfb = s.nf
        grads[b, 2:5] = dots[pos:pos + 3]
        wtot = wbar[b] + dots[pos + 3:pos + 3 + nfb]
        pos += 3 + nfb
        g_lam = eps_bar[b].copy()
        for j, (m, n) in enumerate(s.rep_pairs):
            g_lam[m] += wtot[j]
            g_lam[n] -= wtot[j]
        GA = ops4[b][0] + ops2[b][0]
        Grho = r0b[b].reshape(N, N, order="F")
        GO = ovb[b].reshape(N, N, order="F").T
        GU = (grad_U_from_rotated(cfg.coupling, GA, s.U) + grad_U_from_rotated(cfg.rho0, Grho, s.U)
              + grad_U_from_rotated(cfg.observable, GO, s.U))
        for k, dH in enumerate((0.5 * SZ, 0.5 * SX)):
            dlam, dU = eig_tangent(s.U, s.eps, dH)
            grads[b, k] = float(np.real(np.sum(np.conj(GU) * dU)) + g_lam @ dlam)
    return grads


class SpinBosonTCL4:
    """torch.autograd.Function wrapper: ``SpinBosonTCL4.apply(params, cfg)`` with params a
    float64 tensor [B, 5] (eps, Delta, alpha, wc, beta) returns <O(t)> [B, n_samples]."""

    _fn = None

    @classmethod
    def apply(cls, params, cfg: SpinBosonConfig):
        if cls._fn is None:
            torch = _torch()

            class _Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, p, c):
                    obs, state = spin_boson_forward(p.detach().cpu().numpy(), c, device="cuda")
                    ctx.state = state
                    ctx.cfg = c
                    ctx.pdev = p.device
                    return obs.to(p.device)

                @staticmethod
                def backward(ctx, g):
                    grads = spin_boson_backward(ctx.state, g, ctx.cfg)
                    return torch.from_numpy(grads).to(ctx.pdev), None

            cls._fn = _Fn
        return cls._fn.apply(params, cfg)


def mse_loss_and_grad(params, target, cfg: SpinBosonConfig, device="cuda", phases=None):
    """Per-instance loss mean_t (<sz(t)> - target)^2 and its gradient [B, 5] (numpy)."""
    torch = _torch()
    obs, state = spin_boson_forward(params, cfg, device, phases)
    tgt = torch.as_tensor(np.asarray(target, np.float64), device=obs.device)
    diff = obs - tgt
    ns = obs.shape[1]
    loss = (diff * diff).mean(dim=1)
    g = 2.0 * diff / ns
    grads = spin_boson_backward(state, g, cfg, phases)
    return loss.cpu().numpy(), grads
