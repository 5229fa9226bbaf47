"""Autotuner for the F/C/R launch schedules and FFT lengths.

Tiles: for one FFT length and precision it times the batched build of a representative
workload under each candidate schedule (column tile, row tile, Z/W chunk bytes, pruned
inverse-DFT rows), with CUDA events after warm-up, and keeps the fastest.
Radix: for a requested length the causal rule may use 2^k, 3 * 2^k or 5 * 2^k; the tuner
times the workload with each admissible length and turns off ("enabled": false) the mixed
lengths that lose to a longer one.
Results are persisted as JSON ({"<key>:<fp32|fp64>": {...}}) and applied with load(); the key
of an FFT length is log2 for powers of two, + 64 for 3 * 2^k and + 128 for 5 * 2^k
(taco_b200.fft_length).  Workloads: "c2" (spin-boson batch of the headline shape: the radix
choice for t_max = 10000 and the tiles of its lengths) and "c4" (batching-form lengths
2^15..2^19: one GUE instance of dimension 6 -- 31^3 frequency triples -- with N = 2^(L-1) and
every 8th time).  The FP32 form is
tuned with its precision guard off (the guard's FP64 heads are tuned as FP64 lengths).

    python -m taco_b200.autotune --workloads c2,c4 --out taco_b200/tuning.json   (needs a GPU)
"""
from __future__ import annotations

import ctypes as ct
import itertools
import json
import os

from . import _capi

DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")


def set_schedule(log2_nfft: int, precision: str, col_tile: int, row_tile: int, chunk_bytes: int,
                 inv_dft_rows: int, cluster_lm: int = 0) -> None:
    prec = _capi.TACO_PREC_FP32 if precision == "fp32" else _capi.TACO_PREC_FP64
    _capi.check(_capi.lib().taco_set_tuning(int(log2_nfft), prec, int(col_tile), int(row_tile), int(chunk_bytes),
                                            int(inv_dft_rows)))
    _capi.check(_capi.lib().taco_set_cluster_points(int(log2_nfft), prec, int(cluster_lm)))


def get_schedule(log2_nfft: int, precision: str) -> dict:
    prec = _capi.TACO_PREC_FP32 if precision == "fp32" else _capi.TACO_PREC_FP64
    c, r, d = ct.c_int(), ct.c_int(), ct.c_int()
    b = ct.c_size_t()
    _capi.check(_capi.lib().taco_get_tuning(int(log2_nfft), prec, ct.byref(c), ct.byref(r), ct.byref(b), ct.byref(d)))
    return {"col_tile": c.value, "row_tile": r.value, "chunk_bytes": b.value, "inv_dft_rows": d.value}


def set_length_enabled(key: int, precision: str, enabled: bool) -> None:
    prec = _capi.TACO_PREC_FP32 if precision == "fp32" else _capi.TACO_PREC_FP64
    _capi.check(_capi.lib().taco_set_fft_length_enabled(int(key), prec, 1 if enabled else 0))


def length_of(key: int) -> int:
    return (3 if 64 <= key < 128 else 5 if key >= 128 else 1) << (key & 63)


def load(path: str = DEFAULT_TABLE) -> int:
    """Apply a persisted table; returns the number of schedules applied (0 if absent)."""
    if not os.path.exists(path):
        return 0
    with open(path) as f:
        table = json.load(f)
    n = 0
    for key, sch in table.items():
        if key.startswith("_"):
            continue
        L, prec = key.split(":")
        if "col_tile" in sch:
            set_schedule(int(L), prec, sch["col_tile"], sch["row_tile"], sch["chunk_bytes"], sch["inv_dft_rows"],
                         sch.get("cluster_lm", 0))
        if int(L) >= 64 and "enabled" in sch:
            set_length_enabled(int(L), prec, bool(sch["enabled"]))
        n += 1
    return n


def candidates(precision: str):
    cols = [2048, 4096, 8192] if precision == "fp32" else [2048, 4096]
    rows = [1024, 2048, 4096]
    chunks = [24 << 20, 48 << 20, 96 << 20, 1 << 30]
    dft = [0, 16]
    return [dict(col_tile=c, row_tile=r, chunk_bytes=b, inv_dft_rows=d)
            for c, r, b, d in itertools.product(cols, rows, chunks, dft)]


def _time(log2_nfft, precision, sch, run, factory, reps, warmup, log, check=None):
    """Device time of one unit of work under schedule `sch` (inf when the schedule fails, or
    when `check` says the schedule changes the FFT length being tuned)."""
    import torch

    unit = None
    try:
        set_schedule(log2_nfft, precision, **sch)
        if check is not None and not check():
            if log:
                log(f"{precision} key {log2_nfft} {sch} -> changes the FFT length, skipped")
            return float("inf")
        unit = factory() if factory is not None else run
        for _ in range(warmup):
            unit()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            unit()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
    except _capi.TacoError as exc:  # e.g. a tile that does not fit shared memory
        ms = float("inf")
        if log:
            log(f"schedule {sch} failed: {exc}")
    finally:
        if unit is not None and hasattr(unit, "close"):
            unit.close()
    if log:
        log(f"{precision} key {log2_nfft} {sch} -> {ms:.3f} ms")
    return ms


def tune(run, log2_nfft: int, precision: str, cands=None, reps: int = 3, warmup: int = 1, log=None, factory=None,
         check=None):
    """Times one unit of work under every candidate schedule and keeps the fastest.

    run(): the unit (e.g. a batched build); or factory(): called after each schedule is
    set, returns the unit (e.g. a prepared plan's replay, with a close()).  Returns
    (best, results)."""
    results = []
    for sch in cands or candidates(precision):
        results.append((_time(log2_nfft, precision, sch, run, factory, reps, warmup, log, check), sch))
    results.sort(key=lambda x: x[0])
    best = dict(results[0][1])
    # phase 2: the thread-block-cluster path (points per CTA), with the best multi-pass tiles
    lm_max = 13 if precision == "fp32" else 12
    for lm in (11, 12, 13):
        if log2_nfft >= 64 or lm > lm_max or log2_nfft - lm > 3 or lm > log2_nfft:  # powers of two only
            continue
        sch = dict(best, cluster_lm=lm)
        results.append((_time(log2_nfft, precision, sch, run, factory, reps, warmup, log), sch))
    results.sort(key=lambda x: x[0])
    best = dict(results[0][1])
    best.setdefault("cluster_lm", 0)
    set_schedule(log2_nfft, precision, **best)
    return best, results


def save(entries: dict, path: str = DEFAULT_TABLE, note: str = "") -> None:
    table = {}
    if os.path.exists(path):
        with open(path) as f:
            table = json.load(f)
    table.update(entries)
    if note:
        table["_note"] = note
    with open(path, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)


class _Plans:
    """Replays of prepared plans as one unit of work."""

    def __init__(self, plans):
        self.plans = plans

    def __call__(self):
        for p in self.plans:
            p.run()

    def close(self):
        for p in self.plans:
            p.close()


def mixed_keys(n: int):
    """Schedule keys of the 3 * 2^k and 5 * 2^k lengths the causal rule could pick for n samples."""
    target = 2 * n - 1
    p2 = 1 << max(3, (target - 1).bit_length())
    keys = []
    for base, r in ((64, 3), (128, 5)):
        k = 3
        while (r << k) < target:
            k += 1
        if (r << k) < p2:
            keys.append(base + k)
    return keys


def small_candidates(precision: str):
    cols = [2048, 4096] if precision == "fp32" else [2048, 4096]
    return [dict(col_tile=c, row_tile=r, chunk_bytes=b, inv_dft_rows=d)
            for c, r, b, d in itertools.product(cols, [1024, 2048], [48 << 20, 1 << 30], [0, 16])]


def main():
    import argparse

    import numpy as np
    import torch

    import taco_b200 as tb
    from .workloads import spin_boson_batch

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--instances", type=int, default=32)
    ap.add_argument("--N", type=int, default=200000)
    ap.add_argument("--dt", type=float, default=5e-4)
    ap.add_argument("--tmax", type=int, default=10000)
    ap.add_argument("--precisions", default="fp32,fp64")
    ap.add_argument("--workloads", default="c2,c4")
    ap.add_argument("--c4-lengths", default="15,16,17,18,19")
    ap.add_argument("--c4-dim", type=int, default=6)
    args = ap.parse_args()
    load(args.out)
    guard = tb.fp32_guard()
    tb.set_fp32_guard(0.0)
    entries = {}

    def unit_factory(inst, prec, outs, full=False):
        if prec == "fp64":  # the plain path: one instance per plan
            return lambda: _Plans([tb.Tcl4Plan([inst[k]], precision="fp64", outs=[outs[k]], full_length=full)
                                   for k in range(min(4, len(inst)))])
        return lambda: _Plans([tb.Tcl4Plan(inst, precision=prec, outs=outs, full_length=full)])

    def time_unit(factory, reps=3):
        unit = factory()
        try:
            unit()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                unit()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps
        finally:
            unit.close()

    def tune_tiles(inst, tidx, n, prec, full=False, cands=None):
        nfft, L = tb.fft_length(n, prec, full_length=full)
        dtype = torch.complex64 if prec == "fp32" else torch.complex128
        outs = [torch.empty((tidx.size, x[0].N ** 4), dtype=dtype, device="cuda") for x in inst]

        def same_length(n=n, prec=prec, full=full, nfft=nfft):
            return tb.fft_length(n, prec, full_length=full)[0] == nfft

        best, res = tune(None, L, prec, cands=cands, log=print, factory=unit_factory(inst, prec, outs, full),
                         check=same_length)
        entries[f"{L}:{prec}"] = dict(entries.get(f"{L}:{prec}", {}), **best, ms=res[0][0])

    if "c2" in args.workloads:
        _, systems, gammas = spin_boson_batch(torch, args.instances, args.N, args.dt, seed=123)
        tidx = np.arange(args.tmax + 1, dtype=np.uint32)
        inst = [(s, g, args.dt, tidx) for s, g in zip(systems, gammas)]
        n = tidx.size
        for prec in args.precisions.split(","):
            # radix: each admissible length alone, the fastest kept
            keys = mixed_keys(n)
            dtype = torch.complex64 if prec == "fp32" else torch.complex128
            outs = [torch.empty((n, 16), dtype=dtype, device="cuda") for _ in inst]
            times = {}
            for choice in keys + [None]:
                for k in keys:
                    set_length_enabled(k, prec, k == choice)
                times[choice] = time_unit(unit_factory(inst, prec, outs))
                print(f"{prec} length {length_of(choice) if choice else 'pow2'}: {times[choice]:.3f} ms")
            best = min(times, key=times.get)
            # the rule picks the shortest enabled length: the shorter ones than the winner go
            for k in keys:
                on = best is not None and length_of(k) >= length_of(best)
                set_length_enabled(k, prec, on)
                entries[f"{k}:{prec}"] = dict(entries.get(f"{k}:{prec}", {}), enabled=on)
            tune_tiles(inst, tidx, n, prec)
            tune_tiles(inst, tidx, args.N + 1, prec, full=True)
    if "c4" in args.workloads:
        # one seeded GUE instance of dimension --c4-dim per length (its nf^3 triples dominate
        # the batching form's time): Ohmic bath, N = 2^(L-1), dt = 10 / (N wc), every 8th time
        from . import adjoint as adj
        from .workloads import gue_system
        s, _ = gue_system(args.c4_dim, np.random.default_rng(404))
        for L in [int(x) for x in args.c4_lengths.split(",") if x]:
            Nt = 1 << (L - 1)
            dt = 10.0 / (Nt * 5.0)
            C = adj.bcf_device([dict(alpha=0.05, omega_c=5.0, beta=1.0, N=Nt, dt=dt)], Nt + 1)[0]
            g = tb.gamma_trapz_device(C, dt, s.omegas)
            tidx = np.arange(0, Nt, 8, dtype=np.uint32)
            inst = [(s, g, dt, tidx)]
            for prec in args.precisions.split(","):
                # every output row is kept here, so the pruned inverse DFT never runs: keep the
                # choice an earlier workload measured for this length (0 if none)
                key = f"{tb.fft_length(int(tidx[-1]) + 1, prec)[1]}:{prec}"
                keep = entries.get(key, {}).get("inv_dft_rows", 0)
                cands = [c for c in small_candidates(prec) if c["inv_dft_rows"] == keep]
                tune_tiles(inst, tidx, int(tidx[-1]) + 1, prec, cands=cands)
            del g, C
            tb.release_workspace()
            torch.cuda.empty_cache()
    tb.set_fp32_guard(guard)
    save(entries, args.out, note="measured on B200 by taco_b200.autotune (workloads: " + args.workloads + ")")
    print(json.dumps(entries))


if __name__ == "__main__":
    main()
