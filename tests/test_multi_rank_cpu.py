"""Instance sharding across ranks (the multi-GPU scheme), run as two gloo ranks on CPU.
Every rank draws its own instance set, builds it with no data crossing ranks (here the CPU
oracle stands in for the device build), and the step time is the maximum over ranks."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    import oracle
    from taco_b200 import workloads

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        params, systems = workloads.spin_boson_systems(3, workloads.rank_seed(0, rank))
        builds = 0
        norms = []
        for prm, s in zip(params, systems):
            _, C = oracle.bcf_fft(400, 0.01, oracle.J_OHMIC, [prm["alpha"], prm["wc"]], prm["beta"])
            G = oracle.gamma_trapz(C, 0.01, s.omegas)
            p2f = np.ascontiguousarray(s.pair_to_freq.T, np.int32)
            ops = np.ascontiguousarray(np.stack([A.T for A in s.A_eig]))
            L4 = oracle.tcl4_build_batch(s.N, s.nf, s.omegas, s.mirror, p2f, ops, G, 0.01, tidx=np.arange(0, 401, 40))
            builds += L4.shape[0]
            norms.append(float(np.linalg.norm(L4)))
        ms = workloads.max_over_ranks(dist, 10.0 + 5.0 * rank, "cpu")
        rate = workloads.aggregate_rate(world, builds, ms)
        gathered = [None] * world
        dist.all_gather_object(gathered, (rank, [p["eps"] for p in params], norms, ms, rate))
        if rank == 0:
            np.save(out, np.array(gathered, dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def test_two_rank_instance_sharding(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "gathered.npy")
    mp.spawn(_worker, args=(2, _free_port(), out), nprocs=2, join=True)
    g = sorted(np.load(out, allow_pickle=True).tolist())
    (r0, eps0, n0, ms0, rate0), (r1, eps1, n1, ms1, rate1) = g
    assert (r0, r1) == (0, 1)
    assert not np.allclose(eps0, eps1)          # independent instance sets per rank
    assert not np.allclose(n0, n1)
    assert ms0 == ms1 == pytest.approx(15.0)    # the slowest rank sets the step time
    assert rate0 == rate1 == pytest.approx(2 * 3 * 11 / 0.015)
