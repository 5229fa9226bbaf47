"""Large systems and sliced builds: d = 6 and d = 8 random systems against the oracle, and
builds forced through triple slices (a small transient-memory budget) against the
unsliced build, for direct calls with host and device buffers and for replayed plans."""
import numpy as np
import pytest

import taco_b200 as tb
from cases import oracle_l4, random_case, relerr, spin_boson_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("d,Nt", [(6, 90), (8, 40)])
def test_large_random_systems_vs_oracle(d, Nt):
    osys, s, G = random_case(d, 1, Nt, 0.01, seed=30 + d)
    assert s.nf == d * d - d + 1
    tidx = np.array([0, 1, Nt // 2, Nt - 1])
    ref = oracle_l4(osys, G, 0.01, tidx)
    out = tb.build_TCL4_generator_batch(s, G, 0.01, tidx)
    assert relerr(out, ref) <= 1e-10
    out32 = tb.build_TCL4_generator_batch(s, G, 0.01, tidx, precision="fp32")
    assert relerr(out32, ref) <= 1e-6


def _cases():
    return [spin_boson_case(3000, 0.005), random_case(3, 2, 500, 0.01, seed=3), random_case(4, 1, 300, 0.01, seed=4)]


def test_sliced_builds_match_unsliced():
    import torch
    cases = _cases()
    refs = [tb.build_TCL4_generator_batch(s, G, 0.01, np.arange(0, G.shape[1], 3)) for _, s, G in cases]
    refs32 = [tb.build_TCL4_generator_batch(s, G, 0.01, np.arange(0, G.shape[1], 3), precision="fp32")
              for _, s, G in cases]
    tb.set_work_budget(3 << 20)
    try:
        for (_, s, G), ref, ref32 in zip(cases, refs, refs32):
            tidx = np.arange(0, G.shape[1], 3)
            host = tb.build_TCL4_generator_batch(s, G, 0.01, tidx)
            assert relerr(host, ref) <= 1e-13
            dev = tb.build_TCL4_generator_batch(s, torch.from_numpy(G).cuda(), 0.01, tidx)
            assert relerr(dev.cpu().numpy(), ref) <= 1e-13
            h32 = tb.build_TCL4_generator_batch(s, G, 0.01, tidx, precision="fp32")
            assert relerr(h32, ref32) <= 1e-6
        inst = [(s, torch.from_numpy(G).cuda(), 0.01, np.arange(0, G.shape[1], 3)) for _, s, G in cases]
        plan = tb.Tcl4Plan(inst, precision="fp64")
        res = plan.run()
        torch.cuda.synchronize()
        for r, ref in zip(res, refs):
            assert relerr(r.cpu().numpy(), ref) <= 1e-13
        res = plan.run()  # replays accumulate into freshly overwritten outputs
        torch.cuda.synchronize()
        for r, ref in zip(res, refs):
            assert relerr(r.cpu().numpy(), ref) <= 1e-13
        plan.close()
    finally:
        tb.set_work_budget(0)
