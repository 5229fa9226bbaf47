#!/usr/bin/env python
"""L4(t) builds/s at N=2e5: batched FP32 vs plain FP64 on the GPU.

Workload (one "step"): B seeded spin-boson instances of the reference's compare-tool
size -- d=2, H = (eps sz + Delta sx)/2, A = sz, Ohmic J = alpha w exp(-w/wc), N = 200000
grid steps (Nt = 200001 Gamma samples, FFT length 2^19), dt = 5e-4, tidx = 0..10000
(T = 10001 L4 builds per instance) -- built in one call of the batching form in FP32
(FP64 phases and carries).  Instance parameters: eps, Delta ~ U[0.5, 2],
alpha ~ logU[0.01, 0.2], wc ~ U[1, 20], beta ~ logU[0.2, 5] (seeded, synthetic; there
is no dataset).  Gamma is built on the device outside the timed region (the reference's
timing also excludes it).  Beside it: the plain FP64 path (one instance per call), the
FP32 error against it, an end-to-end leg through the C-ABI with pinned host buffers,
the dominant kernel's roofline from per-kernel CUDA-event timing, and the CPU oracle on
a bounded sample of the same workload.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "L4(t) builds/s at N=2e5: batched-FP32 vs plain-FP64 GPU at <=1e-6 rel err"
SX = np.array([[0, 1], [1, 0]], np.complex128)
SZ = np.array([[1, 0], [0, -1]], np.complex128)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="taco", choices=["taco", "reference"])
    p.add_argument("--instances", type=int, default=256, help="instances per GPU per step")
    p.add_argument("--plain-instances", type=int, default=4)
    p.add_argument("--N", type=int, default=200000)
    p.add_argument("--dt", type=float, default=5e-4)
    p.add_argument("--tmax", type=int, default=10000)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--e2e-steps", type=int, default=3)
    return p.parse_args()


def draw_params(rng, B):
    return [dict(eps=rng.uniform(0.5, 2.0), delta=rng.uniform(0.5, 2.0),
                 alpha=math.exp(rng.uniform(math.log(0.01), math.log(0.2))),
                 wc=rng.uniform(1.0, 20.0), beta=math.exp(rng.uniform(math.log(0.2), math.log(5.0))))
            for _ in range(B)]


def make_gamma_device(torch, sysm, prm, N, dt, device):
    """C(t) (correlation_fft.hpp:153-214) and trapezoid Gamma (gamma.hpp:166-213) with torch."""
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
    S[nfft // 2] = 0.25 * math.pi * (a * wny * math.exp(-wny / wc)) * (1 + 2 / math.expm1(beta * wny))
    C = torch.fft.fft(S)[:Nt] * (dw / math.pi)
    t = torch.arange(Nt, dtype=torch.float64, device=device) * dt
    G = torch.zeros((sysm.nf, Nt), dtype=torch.complex128, device=device)
    for b, om in enumerate(sysm.omegas):
        y = torch.exp(1j * om * t) * C
        G[b, 1:] = torch.cumsum(0.5 * dt * (y[:-1] + y[1:]), 0)
    return G


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.reader.join(timeout=2)
        return False

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def ncu_traffic():
    """DRAM bytes per triple of each kernel from the committed ncu summary (or {})."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def kernel_model_bytes(name, inst_shape):
    """Algorithmic bytes per unit (unit = triple, or spectrum for the spectra passes)."""
    Nt, nfft, tcount, U, nf = inst_shape
    s = 8 if name.endswith("f32") else 16
    base = name.rsplit("_", 1)[0]
    if base == "fwd_col":
        return Nt * 16 + nfft * s, "triple"
    if base == "row_conv":
        return 5 * nfft * s, "triple"
    if base == "inv_col":
        return 2 * nfft * s + 2 * tcount * s, "triple"
    if base == "spectra_col":
        return Nt * 16 + nfft * s, "spectrum"
    if base == "spectra_row":
        return 2 * nfft * s, "spectrum"
    if base == "scan_assemble":
        return 3 * tcount * 16 + 2 * tcount * s + 3 * U * s, "triple"
    return None, None


def reference_arm(args, rank, world):
    """The reference's CPU path (the oracle restatement: the reference needs Eigen, absent here)."""
    if rank != 0:
        return
    import oracle
    threads = oracle.max_threads()
    rng = np.random.default_rng(args.seed)
    prm = draw_params(rng, 1)[0]
    H = 0.5 * prm["eps"] * SZ + 0.5 * prm["delta"] * SX
    osys = oracle.System(H, [SZ])
    _, C = oracle.bcf_fft(args.N, args.dt, oracle.J_OHMIC, [prm["alpha"], prm["wc"]], prm["beta"])
    G = oracle.gamma_trapz(C, args.dt, osys.omegas)
    tidx = np.arange(args.tmax + 1, dtype=np.uint32)
    times = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.tcl4_build_batch(osys.N, osys.nf, osys.omegas, osys.mirror, osys.p2f_colmajor(),
                                osys.ops_colmajor(), G, args.dt, tidx=tidx)
        dt_s = time.perf_counter() - t0
        if it >= args.warmup:
            times.append(dt_s)
    sec = sum(times) / len(times)
    value = tidx.size / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "builds/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"spin-boson d=2, N={args.N}, dt={args.dt}, tidx 0..{args.tmax}",
                   "instances_per_step": 1},
        "cpu_baseline": {"value": value, "unit": "builds/s", "cores": threads, "kind": "port",
                         "sample": f"one instance per step (all 27 triples, FFT 2^19, {tidx.size} L4 builds), "
                                   "C++/OpenMP restatement of the reference CPU path (reference needs Eigen, absent)"},
        "e2e": {"value": value, "unit": "builds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return

    import torch
    import taco_b200 as tb

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    tb._capi.check(tb._capi.lib().taco_set_device(local))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=device)

    B = args.instances
    rng = np.random.default_rng(args.seed + 1000 * rank)
    params = draw_params(rng, B)
    systems, gammas = [], []
    for prm in params:
        s = tb.System(0.5 * prm["eps"] * SZ + 0.5 * prm["delta"] * SX, [SZ])
        systems.append(s)
        gammas.append(make_gamma_device(torch, s, prm, args.N, args.dt, device))
    T = args.tmax + 1
    tidx = np.arange(T, dtype=np.uint32)
    N2 = 4
    outs32 = [torch.empty((T, N2 * N2), dtype=torch.complex64, device=device) for _ in range(B)]
    inst = [(s, g, args.dt, tidx) for s, g in zip(systems, gammas)]
    torch.cuda.synchronize()

    def step32():
        tb.build_instances(inst, precision="fp32", outs=outs32)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        step32()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches0 = tb.kernel_launches()
    with ClockSampler(local) as clk:
        ev0.record()
        for _ in range(args.steps):
            step32()
        ev1.record()
        torch.cuda.synchronize()
    launches = tb.kernel_launches() - launches0
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps)
    value = world * B * T / (ms / 1e3)

    # per-kernel device time of one more step (CUDA events around each launch)
    with tb.profile() as prof:
        step32()
    # plain FP64 path: one instance per call
    P = min(args.plain_instances, B)
    outs64 = [torch.empty((T, N2 * N2), dtype=torch.complex128, device=device) for _ in range(P)]
    for k in range(P):
        tb.build_TCL4_generator_batch(systems[k], gammas[k], args.dt, tidx, precision="fp64", out=outs64[k])
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(P):
        tb.build_TCL4_generator_batch(systems[k], gammas[k], args.dt, tidx, precision="fp64", out=outs64[k])
    e1.record()
    torch.cuda.synchronize()
    ms64 = max_over_ranks(e0.elapsed_time(e1) / P)
    plain_value = T / (ms64 / 1e3)
    err32 = max(float(torch.linalg.vector_norm(outs32[k].to(torch.complex128) - outs64[k])
                      / torch.linalg.vector_norm(outs64[k])) for k in range(P))
    causal_ms = None
    for _ in range(2):
        e0.record()
        tb.build_TCL4_generator_batch(systems[0], gammas[0], args.dt, tidx, precision="fp64",
                                      causal_truncation=True, out=outs64[0])
        e1.record()
        torch.cuda.synchronize()
        causal_ms = e0.elapsed_time(e1)

    # end to end through the C-ABI with pinned host buffers (H2D of Gamma, D2H of L4 inside)
    host_g = [g.cpu().pin_memory() for g in gammas]
    host_out = [torch.empty((T, N2 * N2), dtype=torch.complex64).pin_memory() for _ in range(B)]
    inst_h = [(s, hg.numpy(), args.dt, tidx) for s, hg in zip(systems, host_g)]
    outs_h = [o.numpy() for o in host_out]
    tb.build_instances(inst_h, precision="fp32", outs=outs_h)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        tb.build_instances(inst_h, precision="fp32", outs=outs_h)
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.e2e_steps)
    h2d = sum(g.numel() * 16 for g in gammas)
    d2h = B * T * N2 * N2 * 8
    e2e_value = world * B * T / (e2e_ms / 1e3)
    err_e2e = float(np.abs(outs_h[0] - outs32[0].cpu().numpy()).max())

    # roofline of the dominant kernel
    peaks, peak_kind = measured_peaks()
    nfft = 1 << (2 * (args.N + 1) - 1).bit_length()
    shape = (args.N + 1, nfft, T, T, 3)
    units_total = {"triple": B * 27, "spectrum": B * 6}
    dom = max(prof.entries.items(), key=lambda kv: kv[1][1]) if prof.entries else None
    roofline = None
    kernels = {}
    for name, (n, tot) in prof.entries.items():
        per_unit, unit = kernel_model_bytes(name, shape)
        ent = {"launches": n, "total_ms": round(tot, 4), "share": round(tot / sum(v[1] for v in prof.entries.values()), 4)}
        if per_unit:
            ent["gbs"] = round(per_unit * units_total[unit] / (tot / 1e3) / 1e9, 1)
        kernels[name] = ent
    if dom is not None:
        name, (n, tot) = dom
        per_unit, unit = kernel_model_bytes(name, shape)
        if per_unit:
            per_launch = per_unit * units_total[unit] / n
            avg_s = tot / n / 1e3
            achieved = per_launch / avg_s / 1e9
            tr = ncu_traffic().get(name.rsplit("_", 1)[0] + "_" + name.rsplit("_", 1)[1])
            roofline = {"kernel": name, "bound": "hbm", "achieved": round(achieved, 1),
                        "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4),
                        "peak_source": peak_kind,
                        "algorithmic_bytes_per_launch": per_launch, "avg_launch_ms": round(tot / n, 4),
                        "traffic": (tr * units_total[unit] / n) if tr else None}

    cpu = None
    fp64_vs_oracle = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        s0 = systems[0]
        G0 = gammas[0].cpu().numpy()
        t0 = time.perf_counter()
        L4o = oracle.tcl4_build_batch(s0.N, s0.nf, s0.omegas, s0.mirror,
                                      np.ascontiguousarray(s0.pair_to_freq.T, np.int32),
                                      np.ascontiguousarray(np.stack([A.T for A in s0.A_eig])), G0, args.dt, tidx=tidx)
        sec = time.perf_counter() - t0
        cpu = {"value": T / sec, "unit": "builds/s", "cores": oracle.max_threads(), "kind": "port",
               "sample": f"1 instance ({T} L4 builds, all 27 triples, FFT 2^19) of the {B}-instance step"}
        g64 = outs64[0].view(T, N2, N2).transpose(1, 2).cpu().numpy()
        fp64_vs_oracle = float(np.linalg.norm(g64 - L4o) / np.linalg.norm(L4o))

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "builds/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{B} spin-boson instances per GPU (d=2, nf=3), N={args.N} (Nt={args.N + 1}, "
                                   f"FFT 2^{nfft.bit_length() - 1}), dt={args.dt}, tidx 0..{args.tmax}, "
                                   "batched FP32 form",
                       "instances_per_gpu": B, "builds_per_instance": T,
                       "l2": "inputs larger than L2 (Gamma 9.6 MB x instances, spectra 24 MB per instance)",
                       "parallelism": f"instance-sharded x{world}"},
            "plain_fp64": {"value": plain_value, "unit": "builds/s", "ms_per_instance": ms64,
                           "instances": P, "causal_truncation_ms_per_instance": causal_ms},
            "speedup_vs_plain_fp64": value / (world * plain_value),
            "fp32_rel_err_vs_fp64": err32,
            "fp64_rel_err_vs_oracle": fp64_vs_oracle,
            "e2e": {"value": e2e_value, "unit": "builds/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms, "max_abs_diff_vs_device_run": err_e2e},
            "roofline": roofline, "kernels": kernels,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
