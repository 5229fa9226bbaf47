"""Autotuner for the F/C/R launch schedules.

For one FFT length and precision it times the batched build of a representative
workload under each candidate schedule (column tile, row tile, Z/W chunk bytes, pruned
inverse-DFT rows), with CUDA events after warm-up, and keeps the fastest.  Results are
persisted as JSON ({"<log2_nfft>:<fp32|fp64>": {...}}) and applied with load().

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


def tune(run, log2_nfft: int, precision: str, cands=None, reps: int = 3, warmup: int = 1, log=None):
    """run(): one timed unit of work (e.g. a batched build).  Returns (best, results)."""
    import torch

    results = []
    for sch in cands or candidates(precision):
        try:
            set_schedule(log2_nfft, precision, **sch)
            for _ in range(warmup):
                run()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                run()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
        except _capi.TacoError as exc:  # e.g. a tile that does not fit shared memory
            ms = float("inf")
            if log:
                log(f"schedule {sch} failed: {exc}")
        results.append((ms, sch))
        if log:
            log(f"{precision} 2^{log2_nfft} {sch} -> {ms:.3f} ms")
    results.sort(key=lambda x: x[0])
    best = dict(results[0][1])
    # phase 2: the thread-block-cluster path (points per CTA), with the best multi-pass tiles
    lm_max = 13 if precision == "fp32" else 12
    for lm in (11, 12, 13):
        if lm > lm_max or log2_nfft - lm > 3 or lm > log2_nfft:
            continue
        sch = dict(best, cluster_lm=lm)
        try:
            set_schedule(log2_nfft, precision, **sch)
            for _ in range(warmup):
                run()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                run()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
        except _capi.TacoError as exc:
            ms = float("inf")
            if log:
                log(f"schedule {sch} failed: {exc}")
        results.append((ms, sch))
        if log:
            log(f"{precision} 2^{log2_nfft} {sch} -> {ms:.3f} ms")
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
        L = (2 * n - 2).bit_length()
        for prec in args.precisions.split(","):
            dtype = torch.complex64 if prec == "fp32" else torch.complex128
            outs = [torch.empty((T, 16), dtype=dtype, device="cuda") for _ in systems]
            inst = [(s, g, args.dt, tidx) for s, g in zip(systems, gammas)]
            if prec == "fp64":  # the plain path runs one instance per call
                def run():
                    for k in range(min(4, len(inst))):
                        tb.build_TCL4_generator_batch(inst[k][0], inst[k][1], args.dt, tidx, precision="fp64",
                                                      out=outs[k], full_length=full)
            else:
                def run():
                    tb.build_instances(inst, precision=prec, outs=outs, full_length=full)
            best, res = tune(run, L, prec, log=print)
            entries[f"{L}:{prec}"] = dict(best, ms=res[0][0])
    save(entries, args.out, note="measured on B200 by taco_b200.autotune (C2-shaped spin-boson batch)")
    print(json.dumps(entries))


if __name__ == "__main__":
    main()
