"""Seeded synthetic workloads of the TCL4 path, and the instance sharding across ranks.

spin_boson_batch(): B spin-boson instances H = (eps sz + Delta sx)/2, A = sz with Ohmic
baths J = alpha w exp(-w/wc); eps, Delta ~ U[0.5, 2], alpha ~ logU[0.01, 0.2],
wc ~ U[1, 20], beta ~ logU[0.2, 5].  C(t) (bcf_fft_fun, correlation_fft.hpp:153-214) and
Gamma (trapezoid prefix integrals, gamma.hpp:166-213) are built by the library's own
device kernels.

Multi-GPU: the path shards over independent instances.  Rank r draws its own instances
from seed + 1000 r (weak scaling: fixed work per rank), no data crosses ranks, and the
step time is the maximum over ranks.
"""
from __future__ import annotations

import math

import numpy as np

from .inputs import SX, SZ, System


def draw_params(rng, B):
    return [dict(eps=rng.uniform(0.5, 2.0), delta=rng.uniform(0.5, 2.0),
                 alpha=math.exp(rng.uniform(math.log(0.01), math.log(0.2))),
                 wc=rng.uniform(1.0, 20.0), beta=math.exp(rng.uniform(math.log(0.2), math.log(5.0))))
            for _ in range(B)]


def rank_seed(seed: int, rank: int) -> int:
    """Seed of rank `rank`'s instance set."""
    return seed + 1000 * rank


def max_over_ranks(dist, x: float, device) -> float:
    """Maximum of a per-rank scalar (the step time) over all ranks; x itself on one rank."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, units_per_rank: int, ms_per_step: float) -> float:
    """Whole-job throughput: the units all ranks processed per second of the slowest rank."""
    return world * units_per_rank / (ms_per_step / 1e3)


def gamma_device(sysm, prm, N, dt, device):
    """[nf, N+1] complex128 Gamma on `device` for an Ohmic bath (device BCF + trapezoid)."""
    from . import gamma_trapz_device
    from .adjoint import bcf_device
    C = bcf_device([dict(alpha=prm["alpha"], omega_c=prm["wc"], beta=prm["beta"], N=N, dt=dt)], N + 1, device)[0]
    return gamma_trapz_device(C, dt, sysm.omegas)


def spin_boson_systems(B, seed=0):
    """-> (params, systems) for B seeded spin-boson instances (host only)."""
    rng = np.random.default_rng(seed)
    params = draw_params(rng, B)
    systems = [System(0.5 * prm["eps"] * SZ + 0.5 * prm["delta"] * SX, [SZ]) for prm in params]
    return params, systems


def spin_boson_batch(torch, B, N=200000, dt=5e-4, seed=0, device="cuda"):
    """-> (params, systems, gammas) for B seeded instances (one batched BCF and one batched
    trapezoid launch pair)."""
    del torch
    from . import gamma_trapz_device_batch
    from .adjoint import bcf_device
    params, systems = spin_boson_systems(B, seed)
    C = bcf_device([dict(alpha=p["alpha"], omega_c=p["wc"], beta=p["beta"], N=N, dt=dt) for p in params], N + 1, device)
    gammas = gamma_trapz_device_batch([C[b] for b in range(B)], [dt] * B, [s.omegas for s in systems])
    return params, systems, gammas


def gue_system(d, rng):
    """Seeded GUE Hamiltonian (H_ii ~ N(0, 1/d), off-diagonal real and imaginary parts
    N(0, 1/(2d))) and a random Hermitian coupling of unit spectral norm."""
    from .inputs import System
    X = rng.normal(0.0, np.sqrt(1.0 / (2 * d)), (d, d)) + 1j * rng.normal(0.0, np.sqrt(1.0 / (2 * d)), (d, d))
    H = np.triu(X, 1)
    H = H + H.conj().T + np.diag(rng.normal(0.0, np.sqrt(1.0 / d), d))
    Y = rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d))
    A = np.triu(Y, 1)
    A = A + A.conj().T + np.diag(rng.normal(size=d))
    A = A / np.linalg.norm(A, 2)
    return System(H, [A]), A
