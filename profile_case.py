"""Small, self-contained workload for profiler captures (ncu) of the TCL4 kernels.

Builds `--instances` C2-shaped spin-boson instances (N=200000, dt=5e-4, tidx 0..tmax)
on the device and runs the batched build `--reps` times through the direct API (no CUDA
graph, so every kernel is a separate launch a profiler can select).

    python profile_case.py --instances 8 --precision fp32 --reps 2

--guard sets the FP32 form's precision-guard tolerance (0: off, the FP32 pass alone).
--rk4 K propagates rho(t) of the first K instances over all tmax steps under L2 + L4 (FP64
L4) instead, one RK4 call per trajectory and repetition:

    python profile_case.py --instances 2 --rk4 2 --reps 2
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--instances", type=int, default=8)
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--N", type=int, default=200000)
    ap.add_argument("--dt", type=float, default=5e-4)
    ap.add_argument("--tmax", type=int, default=10000)
    ap.add_argument("--full-length", action="store_true")
    ap.add_argument("--guard", type=float, default=None)
    ap.add_argument("--fused", action="store_true", help="the fused single-CTA F/C/R path where it fits")
    ap.add_argument("--rk4", type=int, default=0, help="RK4 trajectories of the first instances (0: builds)")
    args = ap.parse_args()
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

    import torch

    import taco_b200 as tb
    from taco_b200.workloads import spin_boson_batch

    _, systems, gammas = spin_boson_batch(torch, args.instances, args.N, args.dt, seed=7)
    tidx = np.arange(args.tmax + 1, dtype=np.uint32)
    inst = [(s, g, args.dt, tidx) for s, g in zip(systems, gammas)]
    if args.guard is not None:
        tb.set_fp32_guard(args.guard)
    if args.fused:
        tb.set_fused_conv(True)
    torch.cuda.synchronize()
    if args.rk4 > 0:
        from taco_b200.inputs import SZ
        k = min(args.rk4, len(inst))
        L4s = tb.build_instances(inst[:k], precision="fp64")
        for _ in range(args.reps):
            t0 = time.perf_counter()
            for s, g, L4 in zip(systems[:k], gammas[:k], L4s):
                L2 = tb.tcl2_generator_series(s, g, tidx)
                U = s.U
                rho0 = np.zeros((2, 2), np.complex128)
                rho0[0, 0] = 1.0
                r0 = torch.from_numpy((U.conj().T @ rho0 @ U).reshape(-1, order="F")).cuda()
                ob = torch.from_numpy((U.conj().T @ SZ @ U).T.reshape(-1, order="F")).cuda()
                tb.propagate_rk4_dense(L2, r0, args.dt, L_add=L4, sample_every=10, obs=ob)  # L4: [t, row, col]
            torch.cuda.synchronize()
            print(f"rk4 {k} x {tidx.size - 1} steps: {(time.perf_counter() - t0) * 1e3:.2f} ms")
        return
    for _ in range(args.reps):
        t0 = time.perf_counter()
        tb.build_instances(inst, precision=args.precision, full_length=args.full_length)
        torch.cuda.synchronize()
        print(f"build {args.instances} x {tidx.size} ({args.precision}): {(time.perf_counter() - t0) * 1e3:.2f} ms")


if __name__ == "__main__":
    main()
