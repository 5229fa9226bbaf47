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
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="taco", choices=["taco", "reference"])
    p.add_argument("--instances", type=int, default=256, help="instances per GPU per step")
    p.add_argument("--plain-instances", type=int, default=4)
    p.add_argument("--N", type=int, default=200000)
    p.add_argument("--dt", type=float, default=5e-4)
    p.add_argument("--tmax", type=int, default=10000)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--e2e-steps", type=int, default=10)
    p.add_argument("--err-instances", type=int, default=32, help="instances compared with FP64 per window")
    p.add_argument("--rk4-instances", type=int, default=8, help="C2 RK4 leg: trajectories (0: skip)")
    p.add_argument("--grad-instances", type=int, default=64, help="differentiation form (0: skip)")
    p.add_argument("--grad-N", type=int, default=1 << 16)
    p.add_argument("--grad-dt", type=float, default=1e-3)
    p.add_argument("--grad-steps", type=int, default=4096)
    p.add_argument("--c3-dims", default="4,6", help="precision form on random systems (empty: skip)")
    p.add_argument("--c3-N", type=int, default=1 << 18)
    p.add_argument("--c3-stride", type=int, default=4)
    p.add_argument("--c4-instances", type=int, default=64,
                   help="heterogeneous batch instances (0: skip; the config names 256, which takes about 15 min)")
    p.add_argument("--c4-budget-gib", type=float, default=0.0,
                   help="work budget of the heterogeneous batch's builds in GiB (0: automatic)")
    p.add_argument("--c4-ref-instances", type=int, default=32,
                   help="heterogeneous batch: instances (evenly spaced) also built in FP64 for the errors")
    return p.parse_args()


class ClockSampler:
    """SM clock and clock-event (throttle) reasons during the timed region: NVML read every
    2 ms in a thread (read-only queries), else nvidia-smi every 200 ms."""

    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.sm = []
        self.reasons = set()
        self.max_mhz = None
        self.nvml = None
        self.stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            self.nvml = (nv, h, bits)
            self.reader = threading.Thread(target=self._poll, daemon=True)
            self.reader.start()
            return self
        except Exception:  # no NVML binding or no GPU: fall back to nvidia-smi
            self.nvml = None
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

    def _poll(self):
        nv, h, bits = self.nvml
        while not self.stop.is_set():
            try:
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for nm, bit in bits.items():
                    if r & bit:
                        self.reasons.add(nm)
            except Exception:
                break
            time.sleep(0.002)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        self.stop.set()
        if self.nvml is not None:
            self.reader.join(timeout=2)
            try:
                self.nvml[0].nvmlShutdown()
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.reader.join(timeout=2)
        return False

    def summary(self):
        sm, mx, reasons = list(self.sm), self.max_mhz, set(self.reasons)
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.nvml is not None else "nvidia-smi"}


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
    """Algorithmic bytes per unit (unit = triple, or spectrum for the spectra passes): the
    traffic the kernel cannot avoid.  Inputs shared by all triples of an instance (its nf
    Gamma columns, its 2 nf partner spectra) count once per instance, spread over its nf^3
    triples; per-triple arrays (Z, W_F, W_C, the convolutions, F/C/R) count in full."""
    n_in, nfft, tcount, U, nf, E = inst_shape
    s = 8 if name.endswith("f32") else 16
    base = name.rsplit("_", 1)[0]
    per_tri = lambda per_instance: per_instance / nf ** 3
    if base == "fwd_col":  # Gamma_i shared; Z written
        return per_tri(nf * n_in * 16) + nfft * s, "triple"
    if base == "row_conv":  # Z in; W_F, W_C out; partner spectra shared
        return 3 * nfft * s + per_tri(2 * nf * nfft * s), "triple"
    if base == "inv_col":  # W_F, W_C in; both convolutions (t <= t_max) out
        return 2 * nfft * s + 2 * tcount * s, "triple"
    if base == "spectra_col":  # each Gamma column feeds two spectra
        return n_in * 16 / 2 + nfft * s, "spectrum"
    if base == "spectra_row":
        return 2 * nfft * s, "spectrum"
    if base == "scan_assemble":  # Gamma shared; conv in; F, C, R at the requested times out
        return per_tri(nf * tcount * 16) + 2 * tcount * s + 3 * U * s, "triple"
    if base == "contract":  # F, C, R at the unique times in; L4 at the requested times out
        return 3 * nf ** 3 * U * s + tcount * E * s, "instance"
    if base == "fz_spectra":  # the partner spectra by the fused transform
        return n_in * 16 / 2 + nfft * s, "spectrum"
    if base == "fz_conv_scan":  # the survey's per-triple figure of the FFT convolution (A-hat
        # written and read twice, B-hat read twice) and the F, C, R writes; Gamma shared
        return per_tri(nf * tcount * 16) + 5 * nfft * s + 3 * U * s, "triple"
    return None, None


def causal_fft_length(tcount):
    """FFT length of the causal rule: the smallest 2^k, 3*2^k or 5*2^k >= 2 tcount - 1."""
    target = 2 * tcount - 1
    best = 1 << max(3, (target - 1).bit_length())
    for r in (3, 5):
        k = 0
        while r << k < target:
            k += 1
        best = min(best, r << k)
    return best


def headline_config(args, world):
    """The workload both arms report (the reference arm times a bounded sample of it)."""
    return {"workload": f"{args.instances} spin-boson instances per GPU (d=2, nf=3), N={args.N} (Nt={args.N + 1}), "
                        f"dt={args.dt}, tidx 0..{args.tmax}, L4(t) builds",
            "instances_per_gpu": args.instances, "builds_per_instance": args.tmax + 1,
            "l2": "inputs larger than L2 (Gamma 9.6 MB x instances; L4 outputs 1.3 MB x instances)",
            "parallelism": f"instance-sharded x{world}"}


def window_errors(a, b, tidx):
    """Relative Frobenius errors over the requested times in [0, 64) and [2^k, 2^(k+1)), k >= 6."""
    out = []
    lo, hi = 0, 64
    while lo <= int(tidx.max()):
        m = (tidx >= lo) & (tidx < hi)
        if m.any():
            out.append((lo, float(np.linalg.norm(a[m] - b[m]) / max(np.linalg.norm(b[m]), 1e-300))))
        lo, hi = hi, 2 * hi
    return out


def reference_arm(args, rank, world):
    """The reference's CPU path (the oracle restatement: the reference needs Eigen, absent here)."""
    if rank != 0:
        return
    import oracle
    from taco_b200.workloads import draw_params
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
        "config": headline_config(args, world),
        "cpu_baseline": {"value": value, "unit": "builds/s", "cores": threads, "kind": "port",
                         "sample": f"one of the {args.instances} instances per step (all 27 triples, FFT 2^19 as the "
                                   f"reference, {tidx.size} L4 builds, FP64), C++/OpenMP restatement of the reference "
                                   "CPU path (the reference needs Eigen, absent here)"},
        "e2e": {"value": value, "unit": "builds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def timed(torch, fn, reps, warmup=1):
    """Average device ms of fn() over reps calls (CUDA events on the current stream)."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def gue_system(d, rng):
    """Seeded GUE system of dimension d (taco_b200.workloads.gue_system)."""
    from taco_b200.workloads import gue_system as g
    return g(d, rng)


def precision_random(args, d, cpu_leg):
    """Precision form on a random system: GUE H (dimension d), random unit-norm A, Ohmic
    (alpha 0.1, wc 5) + Drude-Lorentz (lambda 0.05, gamma 2) bath at beta 0.5, N grid
    points, dt 1e-3, tidx 0:stride:N-1.  L4 in FP32 and FP64 on the device; <A(t)> by RK4
    under L2 + L4 over the sampled times; on the CPU leg, the oracle on the first 2001 steps."""
    import torch
    import taco_b200 as tb
    from taco_b200 import adjoint as adj
    tb.release_workspace()
    torch.cuda.empty_cache()
    rng = np.random.default_rng(args.seed + 300 + d)
    s, A = gue_system(d, rng)
    N, dt = args.c3_N, 1e-3
    tidx = np.arange(0, N, args.c3_stride, dtype=np.uint32)
    T = tidx.size
    C = adj.bcf_device([dict(model=1, alpha=0.1, omega_c=5.0, lam=0.05, gam=2.0, beta=0.5, N=N, dt=dt)], N + 1)[0]
    G = tb.gamma_trapz_device(C, dt, s.omegas)
    out = {"d": d, "nf": int(s.nf), "N": N, "T": int(T), "triples": int(s.nf) ** 3}
    res = {}
    for prec in ("fp32", "fp64"):
        tb.build_TCL4_generator_batch(s, G, dt, tidx, precision=prec)  # warm-up (tables, workspace)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        L4 = tb.build_TCL4_generator_batch(s, G, dt, tidx, precision=prec)
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        res[prec] = L4
        out[prec] = {"value": T / sec, "unit": "builds/s", "seconds": round(sec, 3)}
    L64 = res["fp64"]
    err = float(torch.linalg.vector_norm(res["fp32"].to(torch.complex128) - L64) / torch.linalg.vector_norm(L64))
    out["l4_fp32_rel_err_vs_fp64"] = err
    # <A(t)> under L2 + L4 on the sampled times (RK4 step stride * dt), FP64 state
    L2 = tb.tcl2_generator_series(s, G, tidx)
    U = s.U
    rho0 = np.zeros((d, d), np.complex128)
    rho0[0, 0] = 1.0
    r0 = torch.from_numpy((U.conj().T @ rho0 @ U).reshape(-1, order="F")).cuda()
    ob = torch.from_numpy((U.conj().T @ A @ U).T.reshape(-1, order="F")).cuda()
    trajs = {}
    for prec in ("fp32", "fp64"):
        _, _, o = tb.propagate_rk4_dense(L2, r0, dt * args.c3_stride, L_add=res[prec].to(torch.complex128),
                                         sample_every=16, obs=ob)
        trajs[prec] = o.real.cpu().numpy()
    out["expect_A_fp32_rel_err_vs_fp64"] = float(np.linalg.norm(trajs["fp32"] - trajs["fp64"])
                                                 / np.linalg.norm(trajs["fp64"]))
    if cpu_leg:
        import oracle
        k = int(np.searchsorted(tidx, 2001))
        Gh = np.ascontiguousarray(G[:, :2001].cpu().numpy())
        p2f = np.ascontiguousarray(s.pair_to_freq.T, np.int32)
        ops = np.ascontiguousarray(np.stack([Ae.T for Ae in s.A_eig]))
        t0 = time.perf_counter()
        ref = oracle.tcl4_build_batch(s.N, s.nf, s.omegas, s.mirror, p2f, ops, Gh, dt, tidx=tidx[:k])
        g64 = L64[:k].cpu().numpy()
        g32 = res["fp32"][:k].cpu().numpy()
        out["oracle_window"] = {"tidx": f"0:{args.c3_stride}:2000", "fp64_rel_err": float(np.linalg.norm(g64 - ref) / np.linalg.norm(ref)),
                                "fp32_rel_err": float(np.linalg.norm(g32 - ref) / np.linalg.norm(ref)),
                                "oracle_seconds": round(time.perf_counter() - t0, 2)}
    del res, L64, L2
    torch.cuda.empty_cache()
    return out


def heterogeneous_batch(args, rank, world, cpu_leg):
    """Batching form: seeded instances with d ~ U{2,3,4,6,8} (GUE H, random unit-norm A),
    Ohmic bath alpha ~ logU[0.01, 0.2], wc ~ U[1, 20], beta ~ logU[0.2, 5], N ~ U{2^14..2^18},
    dt = 10 / (N wc), every 8th time index; one plan (the FP32 form with its precision guard)
    replayed as a CUDA graph.  FP64 reference: the same plan in FP64 on an evenly spaced subset
    of the instances (errors over the whole series and every dyadic window; <A(t)> by RK4 under
    L2 + L4 for a few of them).  CPU leg: the oracle on the smallest instance of each dimension,
    at four sampled times within its first 2049 steps."""
    import torch
    import taco_b200 as tb
    from taco_b200 import adjoint as adj
    B = args.c4_instances
    tb.release_workspace()  # earlier sections' transient buffers
    torch.cuda.empty_cache()
    if args.c4_budget_gib > 0:
        tb.set_work_budget(int(args.c4_budget_gib * (1 << 30)))
    try:
        return _heterogeneous_batch(args, rank, world, cpu_leg, B)
    finally:
        tb.set_work_budget(0)


def _heterogeneous_batch(args, rank, world, cpu_leg, B):
    import torch
    import taco_b200 as tb
    from taco_b200 import adjoint as adj
    rng = np.random.default_rng(args.seed + 400 + 1000 * rank)
    dims = rng.choice([2, 3, 4, 6, 8], B)
    Ns = 1 << rng.integers(14, 19, B)
    alpha = np.exp(rng.uniform(np.log(0.01), np.log(0.2), B))
    wc = rng.uniform(1.0, 20.0, B)
    beta = np.exp(rng.uniform(np.log(0.2), np.log(5.0), B))
    systems, gammas, tids, dts, As = [], [], [], [], []
    t0 = time.perf_counter()
    for b in range(B):
        s, A = gue_system(int(dims[b]), rng)
        dt = 10.0 / (Ns[b] * wc[b])
        C = adj.bcf_device([dict(alpha=alpha[b], omega_c=wc[b], beta=beta[b], N=int(Ns[b]), dt=dt)], int(Ns[b]) + 1)[0]
        gammas.append(tb.gamma_trapz_device(C, dt, s.omegas))
        systems.append(s)
        As.append(A)
        tids.append(np.arange(0, int(Ns[b]), 8, dtype=np.uint32))
        dts.append(dt)
    inputs_s = time.perf_counter() - t0
    inst = [(systems[b], gammas[b], dts[b], tids[b]) for b in range(B)]
    builds = int(sum(t.size for t in tids))
    # FP64 subset: evenly spaced instances
    nref = min(B, args.c4_ref_instances)
    ref_ids = sorted(set(int(round(k * (B - 1) / max(1, nref - 1))) for k in range(nref)))
    out = {"instances_per_gpu": B, "work_budget_gib": args.c4_budget_gib or "automatic",
           "dims": np.bincount(dims, minlength=9)[[2, 3, 4, 6, 8]].tolist(),
           "builds_per_step": builds, "input_build_seconds": round(inputs_s, 2)}
    t0 = time.perf_counter()
    plan = tb.Tcl4Plan(inst, precision="fp32")
    prep = time.perf_counter() - t0
    guard = tb.fp32_guard_stats()
    plan.run()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    plan.run()
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    out["fp32"] = {"value": world * builds / (ms / 1e3), "unit": "builds/s", "ms_per_step": ms,
                   "plan_prepare_seconds": round(prep, 2), "precision_guard": guard}
    res32 = {b: plan.results[b].to(torch.complex128) for b in ref_ids}
    plan.close()
    ref_inst = [inst[b] for b in ref_ids]
    ref_builds = int(sum(tids[b].size for b in ref_ids))
    t0 = time.perf_counter()
    plan64 = tb.Tcl4Plan(ref_inst, precision="fp64")
    prep64 = time.perf_counter() - t0
    plan64.run()
    torch.cuda.synchronize()
    ev0.record()
    plan64.run()
    ev1.record()
    torch.cuda.synchronize()
    ms64 = ev0.elapsed_time(ev1)
    out["fp64_subset"] = {"instances": len(ref_ids), "value": world * ref_builds / (ms64 / 1e3), "unit": "builds/s",
                          "ms_per_step": ms64, "plan_prepare_seconds": round(prep64, 2)}
    res64 = {b: r for b, r in zip(ref_ids, plan64.results)}
    # the times below 2048 and below 256 from FP64 builds of those times alone (short causal
    # FFTs): the full-length FP64 transform's round-off exceeds the FP32 form's guard at the
    # first, tiny L4 values of long series
    for b in ref_ids:
        r = res64[b].clone()
        for bound in (2048, 256):
            early = np.nonzero(tids[b] < bound)[0]
            if early.size:
                r[early] = tb.build_TCL4_generator_batch(systems[b], gammas[b], dts[b], tids[b][early], precision="fp64")
        res64[b] = r
    per, werr = [], []
    for b in ref_ids:
        a = res32[b].cpu().numpy().reshape(tids[b].size, -1)
        r = res64[b].cpu().numpy().reshape(tids[b].size, -1)
        g = float(np.linalg.norm(a - r) / np.linalg.norm(r))
        wl, w = max(window_errors(a, r, tids[b]), key=lambda x: x[1])
        per.append([b, int(dims[b]), int(np.log2(Ns[b])), round(float(wc[b]), 3), g, w, int(wl)])
        werr.append(w)
    out["l4_fp32_rel_err_vs_fp64_max"] = max(p[4] for p in per)
    out["l4_fp32_window_rel_err_max"] = max(werr)
    out["per_instance"] = per
    out["per_instance_columns"] = ["instance", "d", "log2 N", "wc", "whole-series err", "max dyadic-window err",
                                   "that window's first time"]
    # <A(t)> under L2 + L4 (RK4 at the sampled times, stride 8 dt) for the first subset
    # instance of each dimension
    expect = {}
    for d in sorted(set(int(dims[b]) for b in ref_ids)):
        b = next(x for x in ref_ids if dims[x] == d)
        s = systems[b]
        L2 = tb.tcl2_generator_series(s, gammas[b], tids[b])
        U = s.U
        rho0 = np.zeros((d, d), np.complex128)
        rho0[0, 0] = 1.0
        r0 = torch.from_numpy((U.conj().T @ rho0 @ U).reshape(-1, order="F")).cuda()
        ob = torch.from_numpy((U.conj().T @ As[b] @ U).T.reshape(-1, order="F")).cuda()
        tr = {}
        for name, L4 in (("fp32", res32[b]), ("fp64", res64[b])):
            _, _, o = tb.propagate_rk4_dense(L2, r0, dts[b] * 8, L_add=L4, sample_every=16, obs=ob)
            tr[name] = o.real.cpu().numpy()
        expect[str(d)] = {"instance": b, "rel_err": float(np.linalg.norm(tr["fp32"] - tr["fp64"]) / np.linalg.norm(tr["fp64"]))}
        del L2
    out["expect_A_fp32_rel_err_vs_fp64"] = expect
    if cpu_leg:
        # the oracle on the smallest subset instance of each dimension: F/C/R over the first
        # 2049 steps, L4 at four of the sampled times in that window
        import oracle
        chk = {}
        for d in sorted(set(int(dims[b]) for b in ref_ids)):
            b = min((k for k in ref_ids if dims[k] == d), key=lambda k: Ns[k])
            s = systems[b]
            pos = [16, 64, 128, 256]
            Gh = np.ascontiguousarray(gammas[b][:, :2049].cpu().numpy())
            p2f = np.ascontiguousarray(s.pair_to_freq.T, np.int32)
            ops = np.ascontiguousarray(np.stack([Ae.T for Ae in s.A_eig]))
            ref = oracle.tcl4_build_batch(s.N, s.nf, s.omegas, s.mirror, p2f, ops, Gh, dts[b], tidx=tids[b][pos])
            g64 = res64[b][pos].cpu().numpy()
            g32 = res32[b][pos].cpu().numpy()
            chk[str(d)] = {"instance": int(b), "times": tids[b][pos].tolist(),
                           "fp64_rel_err": float(np.linalg.norm(g64 - ref) / np.linalg.norm(ref)),
                           "fp32_rel_err": float(np.linalg.norm(g32 - ref) / np.linalg.norm(ref))}
        out["oracle_check"] = chk
    plan64.close()
    del res32, res64
    torch.cuda.empty_cache()
    return out


def differentiation(args, rank, world, cpu_leg):
    """The differentiation form: loss = mean_t (<sz(t)> - target)^2 per spin-boson instance,
    gradient in (eps, Delta, alpha, wc, beta) by the hand-written adjoint (FP64 and with the
    FP32 L4 build), timed end to end; on the CPU leg, central differences (h = 1e-6) of the
    FP64 oracle chain for one instance."""
    import torch
    from taco_b200 import adjoint as adj
    B = args.grad_instances
    rng = np.random.default_rng(args.seed + 77 + 1000 * rank)
    params = np.stack([rng.uniform(0.5, 2.0, B), rng.uniform(0.5, 2.0, B),
                       np.exp(rng.uniform(np.log(0.01), np.log(0.2), B)), rng.uniform(1.0, 20.0, B),
                       np.exp(rng.uniform(np.log(0.2), np.log(5.0), B))], axis=1)
    out = {"instances_per_gpu": B, "N": args.grad_N, "dt": args.grad_dt, "rk4_steps": args.grad_steps,
           "loss": "mean over 4097 samples of (<sz(t)> - target(t))^2, seeded damped-cosine target"}
    t = np.arange(args.grad_steps + 1) * args.grad_dt
    tgt = (0.6 * np.cos(rng.uniform(0.5, 2.0, (B, 1)) * t[None, :]) * np.exp(-0.1 * t[None, :]))
    for prec in ("fp64", "fp32"):
        cfg = adj.SpinBosonConfig(N=args.grad_N, dt=args.grad_dt, steps=args.grad_steps, precision=prec)
        adj.mse_loss_and_grad(params, tgt, cfg)  # warm-up (workspaces, tables)
        ph = adj.Phases()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss, grads = adj.mse_loss_and_grad(params, tgt, cfg, phases=ph)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3
        out[prec] = {"value": world * B / (ms / 1e3), "unit": "loss+gradient evaluations/s", "ms_per_step": ms,
                     "phases_ms": {k: round(v, 3) for k, v in ph.ms.items()}}
        if prec == "fp64":
            g64 = grads
        else:
            out["fp32_grad_rel_diff_vs_fp64"] = float(np.linalg.norm(grads - g64) / np.linalg.norm(g64))
    if cpu_leg:
        import oracle
        h = 1e-6
        fd = np.zeros(5)
        t0 = time.perf_counter()
        for k in range(5):
            pp, pm = params[0].copy(), params[0].copy()
            pp[k] += h
            pm[k] -= h
            lp = np.mean((oracle.spin_boson_trajectory(pp, args.grad_N, args.grad_dt, args.grad_steps) - tgt[0]) ** 2)
            lm = np.mean((oracle.spin_boson_trajectory(pm, args.grad_N, args.grad_dt, args.grad_steps) - tgt[0]) ** 2)
            fd[k] = (lp - lm) / (2 * h)
        out["oracle_fd_check"] = {"instance": 0, "params": params[0].tolist(), "grad": g64[0].tolist(),
                                  "fd": fd.tolist(),
                                  "rel_err": float(np.linalg.norm(g64[0] - fd) / np.linalg.norm(fd)),
                                  "max_component_rel_err": float(np.max(np.abs(g64[0] - fd) / np.abs(fd))),
                                  "oracle_seconds": round(time.perf_counter() - t0, 2)}
    return out


def c2_rk4_leg(args, systems, gammas, outs32, outs64, tidx):
    """The config's RK4 leg: rho(t) over all tmax steps under L = L2(t) + L4(t) on the device
    (FP64 state), one call per trajectory, with the FP32 form's and the FP64 path's L4;
    <sz(t)> in the lab frame sampled every 10 steps."""
    import torch
    import taco_b200 as tb
    P = min(args.rk4_instances, len(outs64))
    if P <= 0:
        return None
    T = tidx.size
    times, errs = [], []
    # one untimed call first: the kernels' first launch in a process loads them
    s0 = systems[0]
    L2w = tb.tcl2_generator_series(s0, gammas[0], tidx)
    r0w = torch.zeros(16, dtype=torch.complex128, device=L2w.device)
    r0w[0] = 1.0
    tb.propagate_rk4_dense(L2w, r0w, args.dt, L_add=outs64[0].view(T, 4, 4).transpose(1, 2).to(torch.complex128),
                           sample_every=10, obs=r0w)
    torch.cuda.synchronize()
    del L2w
    with tb.profile() as prof:
        for k in range(P):
            s, g = systems[k], gammas[k]
            L2 = tb.tcl2_generator_series(s, g, tidx)
            U = s.U
            rho0 = np.zeros((2, 2), np.complex128)
            rho0[0, 0] = 1.0
            r0 = torch.from_numpy((U.conj().T @ rho0 @ U).reshape(-1, order="F")).cuda()
            ob = torch.from_numpy((U.conj().T @ SZ @ U).T.reshape(-1, order="F")).cuda()
            traj = {}
            for name, L4 in (("fp32", outs32[k]), ("fp64", outs64[k])):
                L4v = L4.view(T, 4, 4).transpose(1, 2).to(torch.complex128)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                _, _, o = tb.propagate_rk4_dense(L2, r0, args.dt, L_add=L4v, sample_every=10, obs=ob)
                e1.record()
                torch.cuda.synchronize()
                times.append(e0.elapsed_time(e1))
                traj[name] = o.real.cpu().numpy()
            errs.append(float(np.linalg.norm(traj["fp32"] - traj["fp64"]) / np.linalg.norm(traj["fp64"])))
    steps = T - 1
    ms = statistics.median(times)
    # bytes of the step-matrix scheme per trajectory (D = 4, 16-byte entries): the L2 and L4
    # series read once to form the step matrices ("rk4_warp": the matrix kernel), the
    # matrices written there and read once by the sequential chain ("rk4_chain")
    D2 = 16 * 16
    kernel_bytes = {"rk4_warp": (steps + 1) * D2 * 2 + steps * D2, "rk4_chain": steps * D2}
    bytes_traj = sum(kernel_bytes.values())
    peaks, _ = measured_peaks()
    rk4 = {}
    for name, (n, tot) in prof.entries.items():
        ent = {"launches": n, "total_ms": round(tot, 4)}
        if name in kernel_bytes and n and tot > 0:
            gbs = kernel_bytes[name] / (tot / n / 1e3) / 1e9
            ent["gbs"] = round(gbs, 1)
            ent["frac_of_measured_hbm"] = round(gbs / peaks["hbm_gbs"], 4)
        rk4[name] = ent
    return {"trajectories": P, "steps": steps, "ms_per_trajectory": ms,
            "trajectories_per_s": 1e3 / ms, "gbs_per_trajectory_call": round(bytes_traj / (ms / 1e3) / 1e9, 2),
            "expect_sz_fp32_rel_err_vs_fp64_max": max(errs), "kernels": rk4,
            "note": "latency-bound (one matrix-vector product per sequential step); bytes: L2+L4 series "
                    "read once, step matrices written and read once"}


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
    from taco_b200 import workloads
    from taco_b200.workloads import spin_boson_batch

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    tb._capi.check(tb._capi.lib().taco_set_device(local))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=device)

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        return workloads.max_over_ranks(dist, x, device)

    B = args.instances
    params, systems, gammas = spin_boson_batch(torch, B, args.N, args.dt, seed=workloads.rank_seed(args.seed, rank),
                                               device=device)
    T = args.tmax + 1
    tidx = np.arange(T, dtype=np.uint32)
    N2 = 4
    outs32 = [torch.empty((T, N2 * N2), dtype=torch.complex64, device=device) for _ in range(B)]
    inst = [(s, g, args.dt, tidx) for s, g in zip(systems, gammas)]
    torch.cuda.synchronize()

    # ---- headline: the batching form (FP32 pass + precision guard), prepared once and
    # replayed as one CUDA graph ----
    plan32 = tb.Tcl4Plan(inst, precision="fp32", outs=outs32)
    guard = dict(tb.fp32_guard_stats(), tolerance=tb.fp32_guard())
    for _ in range(args.warmup):
        plan32.run()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    launches0 = tb.kernel_launches()
    torch.cuda.profiler.start()  # a profiler started with profiling off sees the timed steps alone
    with ClockSampler(local) as clk:
        ev0.record()
        for _ in range(args.steps):
            plan32.run()
        ev1.record()
        torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    launches = tb.kernel_launches() - launches0
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps)
    value = workloads.aggregate_rate(world, B * T, ms)

    # the FP32 pass alone (guard off), for the guard's share of the step
    tb.set_fp32_guard(0.0)
    outs32r = [torch.empty_like(o) for o in outs32]
    plan32r = tb.Tcl4Plan(inst, precision="fp32", outs=outs32r)
    tb.set_fp32_guard(guard["tolerance"])
    ms_pass = max_over_ranks(timed(torch, plan32r.run, 5))
    plan32r.close()
    del outs32r

    # per-kernel device time of one more step (the same launches, not graph-captured)
    with tb.profile() as prof:
        tb.build_instances(inst, precision="fp32", outs=outs32)
    direct32_ms = max_over_ranks(timed(torch, lambda: tb.build_instances(inst, precision="fp32", outs=outs32), 2))
    plan32.run()

    # ---- plain FP64 path: one instance per call (replayed plan, and the direct call) ----
    P = min(args.plain_instances, B)
    Pe = min(max(args.err_instances, P), B)
    outs64 = [torch.empty((T, N2 * N2), dtype=torch.complex128, device=device) for _ in range(Pe)]
    plans64 = [tb.Tcl4Plan([inst[k]], precision="fp64", outs=[outs64[k]]) for k in range(P)]
    ms64 = max_over_ranks(timed(torch, lambda: [p.run() for p in plans64], 3) / P)
    ms64_direct = max_over_ranks(timed(torch, lambda: [tb.build_TCL4_generator_batch(
        systems[k], gammas[k], args.dt, tidx, precision="fp64", out=outs64[k]) for k in range(P)], 2) / P)
    plain_value = T / (ms64 / 1e3)
    # FP32 form against FP64 on Pe instances: whole series and every dyadic window (FP64 for
    # the times below 2048 and below 256 from builds of those times alone: short causal FFTs)
    tb.build_instances(inst[P:Pe], precision="fp64", outs=outs64[P:Pe])
    torch.cuda.synchronize()
    errs_g, errs_w = [], []
    for k in range(Pe):
        a = outs32[k].to(torch.complex128).cpu().numpy()
        b = outs64[k].cpu().numpy().copy()
        for bound in (2048, 256):
            early = tidx[tidx < bound]
            b[: early.size] = tb.build_TCL4_generator_batch(systems[k], gammas[k], args.dt, early, precision="fp64"
                                                            ).transpose(1, 2).reshape(early.size, -1).cpu().numpy()
        errs_g.append(float(np.linalg.norm(a - b) / np.linalg.norm(b)))
        errs_w.append(max(e for _, e in window_errors(a, b, tidx)))
    err32 = max(errs_g)

    # ---- the same work with the reference's FFT length (2^19 from Nt), labelled separately ----
    Bf = min(B, 64)
    outs32f = [torch.empty((T, N2 * N2), dtype=torch.complex64, device=device) for _ in range(Bf)]
    plan32f = tb.Tcl4Plan(inst[:Bf], precision="fp32", outs=outs32f, full_length=True)
    ms_full = max_over_ranks(timed(torch, plan32f.run, 2))
    outs64f = torch.empty((T, N2 * N2), dtype=torch.complex128, device=device)
    plan64f = tb.Tcl4Plan([inst[0]], precision="fp64", outs=[outs64f], full_length=True)
    ms64_full = max_over_ranks(timed(torch, plan64f.run, 3))
    torch.cuda.synchronize()
    full_err = float(torch.linalg.vector_norm(outs32f[0].to(torch.complex128) - outs64[0])
                     / torch.linalg.vector_norm(outs64[0]))
    del outs32f
    plan32f.close()

    # ---- end to end through the C-ABI with pinned host buffers (H2D of Gamma, D2H of L4) ----
    host_g = [g.cpu().pin_memory() for g in gammas]
    host_out = [torch.empty((T, N2 * N2), dtype=torch.complex64).pin_memory() for _ in range(B)]
    inst_h = [(s, hg.numpy(), args.dt, tidx) for s, hg in zip(systems, host_g)]
    outs_h = [o.numpy() for o in host_out]
    for _ in range(max(3, args.warmup)):  # the first call checks the heads, the second prepares them
        tb.build_instances(inst_h, precision="fp32", outs=outs_h)
    barrier()
    e2e_times = []
    for _ in range(args.e2e_steps):
        t0 = time.perf_counter()
        tb.build_instances(inst_h, precision="fp32", outs=outs_h)
        e2e_times.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = max_over_ranks(sum(e2e_times) / len(e2e_times))
    h2d = sum(g.shape[0] * T * 16 for g in gammas)  # the consumed samples t <= tmax of every bucket
    d2h = B * T * N2 * N2 * 8
    e2e_value = world * B * T / (e2e_ms / 1e3)
    err_e2e = float(np.abs(outs_h[0] - outs32[0].cpu().numpy()).max())

    # ---- roofline of the dominant kernel (FP32 pass kernels: the byte model's shapes) ----
    peaks, peak_kind = measured_peaks()
    nfft = tb.fft_length(T, "fp32")[0]  # causal rule: 2 (tmax+1) - 1 rounded up to 2^k, 3*2^k or 5*2^k
    shape = (T, nfft, T, T, 3, 16)
    units_total = {"triple": B * 27, "spectrum": B * 6, "instance": B}
    tot_all = sum(v[1] for v in prof.entries.values()) or 1.0
    kernels = {}
    for name, (n, tot) in prof.entries.items():
        per_unit, unit = kernel_model_bytes(name, shape) if name.endswith("f32") else (None, None)
        ent = {"launches": n, "total_ms": round(tot, 4), "share": round(tot / tot_all, 4)}
        if per_unit:
            gbs = per_unit * units_total[unit] / (tot / 1e3) / 1e9
            ent["gbs"] = round(gbs, 1)
            ent["frac_of_measured_hbm"] = round(gbs / peaks["hbm_gbs"], 4)
        elif name.endswith("f64"):
            ent["note"] = "FP64 head of the precision guard"
        kernels[name] = ent
    roofline = None
    ranked = sorted(prof.entries.items(), key=lambda kv: -kv[1][1])
    for name, (n, tot) in ranked:
        per_unit, unit = kernel_model_bytes(name, shape) if name.endswith("f32") else (None, None)
        if not per_unit:
            continue
        per_launch = per_unit * units_total[unit] / n
        achieved = per_launch / (tot / n / 1e3) / 1e9
        tr = ncu_traffic().get(name)
        roofline = {"kernel": name, "bound": "hbm", "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"],
                    "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4), "peak_source": peak_kind,
                    "algorithmic_bytes_per_launch": per_launch, "avg_launch_ms": round(tot / n, 4),
                    "share_of_step": round(tot / tot_all, 4),
                    "traffic": (tr * units_total[unit] / n) if tr else None}
        break

    cpu = None
    fp64_parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle
        s0 = systems[0]
        G0 = gammas[0].cpu().numpy()
        p2f = np.ascontiguousarray(s0.pair_to_freq.T, np.int32)
        ops = np.ascontiguousarray(np.stack([A.T for A in s0.A_eig]))
        t0 = time.perf_counter()
        L4o = oracle.tcl4_build_batch(s0.N, s0.nf, s0.omegas, s0.mirror, p2f, ops, G0, args.dt, tidx=tidx)
        sec = time.perf_counter() - t0
        cpu = {"value": T / sec, "unit": "builds/s", "cores": oracle.max_threads(), "kind": "port",
               "sample": f"1 instance ({T} L4 builds, all 27 triples, FFT 2^19 as the reference) of the "
                         f"{B}-instance step"}
        # exact reference at t <= tmax: the Direct method on the causally truncated series
        L4d = oracle.tcl4_build_batch(s0.N, s0.nf, s0.omegas, s0.mirror, p2f, ops, np.ascontiguousarray(G0[:, :T]),
                                      args.dt, tidx=tidx, method=oracle.FCR_DIRECT)
        g64 = outs64[0].view(T, N2, N2).transpose(1, 2).cpu().numpy()
        g32 = outs32[0].view(T, N2, N2).transpose(1, 2).cpu().numpy()

        def re(a, b):
            return float(np.linalg.norm(a - b) / np.linalg.norm(b))

        fp64_parity = {"vs_oracle_convolution": re(g64, L4o), "vs_oracle_direct": re(g64, L4d),
                       "oracle_convolution_vs_direct": re(L4o, L4d), "fp32_vs_oracle_direct": re(g32, L4d),
                       "fp32_vs_oracle_direct_windows_max": max(e for _, e in window_errors(
                           g32.reshape(T, -1), L4d.reshape(T, -1), tidx))}

    # the other forms and configurations: one GPU only (the scaling runs time the headline)
    cpu_leg = rank == 0 and world == 1 and not args.no_cpu_baseline
    single = world == 1
    def section(fn, *a):
        # a secondary section that fails reports its error instead of losing the headline line
        t0s = time.perf_counter()
        try:
            res = fn(*a)
            if isinstance(res, dict):
                res["section_seconds"] = round(time.perf_counter() - t0s, 1)
            return res
        except Exception as exc:  # noqa: BLE001
            import traceback
            traceback.print_exc()
            try:
                tb.release_workspace()
                torch.cuda.empty_cache()
            except Exception:  # noqa: BLE001
                pass
            return {"error": f"{type(exc).__name__}: {exc}"}

    rk4 = section(c2_rk4_leg, args, systems, gammas, outs32, outs64, tidx) if single else None
    grad = section(differentiation, args, rank, world, cpu_leg) if single and args.grad_instances > 0 else None
    c3 = ([section(precision_random, args, int(d), cpu_leg) for d in args.c3_dims.split(",") if d.strip()]
          if single else None)
    c4 = section(heterogeneous_batch, args, rank, world, cpu_leg) if single and args.c4_instances > 0 else None

    if rank == 0:
        full_plain = T / (ms64_full / 1e3)
        line = {
            "metric": METRIC, "value": value, "unit": "builds/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": headline_config(args, world),
            "speedup_vs_plain_fp64": value / (world * plain_value),
            "fp32_rel_err_vs_fp64": err32,
            "fp32_window_rel_err_max": max(errs_w),
            "like_for_like": {"plain_fp64_full_length_builds_per_s": full_plain,
                              "vs_cpu_reference": (full_plain / cpu["value"]) if cpu else None,
                              "note": "one instance, FP64, FFT 2^19 from Nt: the reference's precision and "
                                      "algorithm length on the GPU against the CPU restatement"},
            "step": {"fft_length": nfft, "fp32_pass_ms": ms_pass, "guard_ms": ms - ms_pass,
                     "note": "one step = the FP32 pass over all instances, then the precision guard's "
                             "FP64 heads and row patch (heads chosen at plan creation)"},
            "precision_guard": guard,
            "plain_fp64": {"value": plain_value, "unit": "builds/s", "ms_per_instance": ms64,
                           "ms_per_instance_direct_call": ms64_direct, "instances": P},
            "fp32_errors": {"instances": Pe, "whole_series_max": err32, "dyadic_windows_max": max(errs_w),
                            "whole_series": [round(e, 10) for e in errs_g]},
            "fp64_parity": fp64_parity,
            "direct_call_ms_per_step": direct32_ms,
            "full_length_fft": {"note": "FFT length 2^19 from Nt as the reference; same results",
                                "value": world * Bf * T / (ms_full / 1e3), "instances": Bf, "ms_per_step": ms_full,
                                "plain_fp64_value": full_plain,
                                "speedup_vs_plain_fp64": (Bf * T / (ms_full / 1e3)) / full_plain,
                                "fp32_rel_err_vs_fp64": full_err},
            "e2e": {"value": e2e_value, "unit": "builds/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms, "steps": len(e2e_times), "ms_min": min(e2e_times),
                    "max_abs_diff_vs_device_run": err_e2e},
            "roofline": roofline, "kernels": kernels,
            "rk4_c2": rk4,
            "differentiation": grad,
            "precision_random": c3,
            "heterogeneous_batch": c4,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    for p in [plan32, plan64f, *plans64]:
        p.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
