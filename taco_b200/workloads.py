"""Seeded synthetic workloads of the TCL4 path (input preparation on the device with torch).

spin_boson_batch(): B spin-boson instances H = (eps sz + Delta sx)/2, A = sz with Ohmic
baths J = alpha w exp(-w/wc); eps, Delta ~ U[0.5, 2], alpha ~ logU[0.01, 0.2],
wc ~ U[1, 20], beta ~ logU[0.2, 5].  C(t) follows the KMS construction of
cpp/include/taco/correlation_fft.hpp:153-214 and Gamma the trapezoid prefix integrals of
cpp/include/taco/gamma.hpp:166-213, computed with torch on the GPU (setup only, not the
measured path).
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


def gamma_device(torch, sysm, prm, N, dt, device):
    """[nf, N+1] complex128 Gamma on `device` for an Ohmic bath."""
    Nt = N + 1
    nfft = 1 << (2 * Nt - 1).bit_length()
    dw = 2 * math.pi / (dt * nfft)
    wny = math.pi / dt
    a, wc, beta = prm["alpha"], prm["wc"], prm["beta"]
    k = torch.arange(1, nfft // 2, dtype=torch.float64, device=device)
    w = dw * k
    J = a * w * torch.exp(-w / wc)
    r = math.exp(-beta * dw)
    kms = torch.exp(-beta * dw * k)
    sp = (math.pi / 2) * J / (1.0 - kms)
    S = torch.zeros(nfft, dtype=torch.complex128, device=device)
    S[1:nfft // 2] = sp.to(torch.complex128)
    S[nfft // 2 + 1:] = torch.flip(sp * kms, [0]).to(torch.complex128)
    S[0] = 0.5 * (math.pi / 2) * (a * dw * math.exp(-dw / wc)) * (1 + r) / (1 - r)
    x = beta * wny  # coth(x/2) = 1 + 2/(e^x - 1); the term vanishes once e^x overflows
    S[nfft // 2] = 0.25 * math.pi * (a * wny * math.exp(-wny / wc)) * (1 + (2 / math.expm1(x) if x < 700 else 0.0))
    C = torch.fft.fft(S)[:Nt] * (dw / math.pi)
    t = torch.arange(Nt, dtype=torch.float64, device=device) * dt
    G = torch.zeros((sysm.nf, Nt), dtype=torch.complex128, device=device)
    for b, om in enumerate(sysm.omegas):
        y = torch.exp(1j * om * t) * C
        G[b, 1:] = torch.cumsum(0.5 * dt * (y[:-1] + y[1:]), 0)
    return G


def spin_boson_batch(torch, B, N=200000, dt=5e-4, seed=0, device="cuda"):
    """-> (params, systems, gammas) for B seeded instances."""
    rng = np.random.default_rng(seed)
    params = draw_params(rng, B)
    systems, gammas = [], []
    for prm in params:
        s = System(0.5 * prm["eps"] * SZ + 0.5 * prm["delta"] * SX, [SZ])
        systems.append(s)
        gammas.append(gamma_device(torch, s, prm, N, dt, device))
    return params, systems, gammas
