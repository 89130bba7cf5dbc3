"""Batched mode: every graph of a batch gets exactly the single-graph result
(oracle and GPU), independent of the number of concurrent workers."""
import numpy as np
import pytest
import torch

from thegraphpartitioning_b200 import graphs

pytestmark = pytest.mark.gpu


def _batch(device, count=14, seed=5):
    specs = graphs.batch_specs(count, seed=seed, nmin=300, nmax=12000)
    return specs, [graphs.batch_graph(s, device=device) for s in specs]


def test_batch_matches_oracle_and_single(oracle_mod, gp, cuda):
    specs, gs = _batch(cuda)
    ks = [s["k"] for s in specs]
    seeds = [s["seed"] for s in specs]
    parts, stats = gp.partition_batch(gs, ks, 0.03, seeds, workers=6)
    for s, (rp, ci), p, st in zip(specs, gs, parts, stats):
        ref, rst, _ = oracle_mod.partition(rp.cpu().numpy(), ci.cpu().numpy(), s["k"], 0.03, s["seed"])
        assert np.array_equal(p.cpu().numpy(), ref), s
        assert st["cut"] == rst["cut"]
        single, _, _ = gp.partition(rp, ci, s["k"], 0.03, s["seed"])
        assert torch.equal(single, p)


def test_batch_worker_count_invariance(gp, cuda):
    specs, gs = _batch(cuda, count=24, seed=9)
    ks = [s["k"] for s in specs]
    seeds = [s["seed"] for s in specs]
    a, _ = gp.partition_batch(gs, ks, 0.03, seeds, workers=1)
    b, _ = gp.partition_batch(gs, ks, 0.03, seeds, workers=12)
    assert all(torch.equal(x, y) for x, y in zip(a, b))


def test_batch_reports_invalid_graph(gp, cuda):
    rp, ci = graphs.grid2d(10, 10)
    bad_ci = ci.clone()
    bad_ci[5] = 1000
    gs = [(rp.to(cuda), ci.to(cuda)), (rp.to(cuda), bad_ci.to(cuda))]
    with pytest.raises(gp.GPError) as ei:
        gp.partition_batch(gs, [2, 2])
    assert ei.value.code == -1
