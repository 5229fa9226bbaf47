"""Autotuner for the F/C/R launch schedules.

For one FFT length and precision it times the batched build of a representative
workload under each candidate schedule (column tile, row tile, Z/W chunk bytes, pruned
inverse-DFT rows), with CUDA events after warm-up, and keeps the fastest.  Results are
persisted as JSON ({"<key>:<fp32|fp64>": {...}}) and applied with load(); the key of an
FFT length is log2 for powers of two, + 64 for 3 * 2^k and + 128 for 5 * 2^k
(taco_b200.fft_length).

    python -m taco_b200.autotune --out taco_b200/tuning.json   (needs a GPU)
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
        set_schedule(int(L), prec, sch["col_tile"], sch["row_tile"], sch["chunk_bytes"], sch["inv_dft_rows"],
                     sch.get("cluster_lm", 0))
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
    args = ap.parse_args()
    _, systems, gammas = spin_boson_batch(torch, args.instances, args.N, args.dt, seed=123)
    tidx = np.arange(args.tmax + 1, dtype=np.uint32)
    T = tidx.size
    entries = {}
    for full in (False, True):
        # FFT length: next_pow2(2 n - 1) with n = tmax + 1 (default) or Nt (full length)
        n = (args.N + 1) if full else T
        for prec in args.precisions.split(","):
            nfft, L = tb.fft_length(n, prec, full_length=full)  # L: the schedule key of this length
            dtype = torch.complex64 if prec == "fp32" else torch.complex128
            outs = [torch.empty((T, 16), dtype=dtype, device="cuda") for _ in systems]
            inst = [(s, g, args.dt, tidx) for s, g in zip(systems, gammas)]
            if prec == "fp64":  # the plain path: one instance per plan
                def factory():
                    return _Plans([tb.Tcl4Plan([inst[k]], precision="fp64", outs=[outs[k]], full_length=full)
                                   for k in range(min(4, len(inst)))])
            else:  # the batched path: one plan over every instance
                def factory():
                    return _Plans([tb.Tcl4Plan(inst, precision=prec, outs=outs, full_length=full)])
            def same_length(n=n, prec=prec, full=full, nfft=nfft):
                return tb.fft_length(n, prec, full_length=full)[0] == nfft

            best, res = tune(None, L, prec, log=print, factory=factory, check=same_length)
            entries[f"{L}:{prec}"] = dict(best, ms=res[0][0])
    save(entries, args.out, note="measured on B200 by taco_b200.autotune (C2-shaped spin-boson batch)")
    print(json.dumps(entries))


if __name__ == "__main__":
    main()
