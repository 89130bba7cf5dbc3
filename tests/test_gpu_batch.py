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


def test_autotune_picks_a_config_with_identical_results(gp, cuda):
    """The autotuner times launch-shape candidates on a sample; whatever it
    picks, every partition equals the default call's."""
    from thegraphpartitioning_b200.autotune import autotune_batch, autotune_graph
    specs, gs = _batch(cuda, count=12, seed=3)
    ks = [s["k"] for s in specs]
    seeds = [s["seed"] for s in specs]
    best = autotune_batch(gs, ks, 0.03, seeds, sample=6, workers=(1, 4), small_level_n=(0, 2048),
                          ctas_per_sm=(2, 8))
    assert len(best["table"]) == 8 and best["sample"] == 6
    ref, _ = gp.partition_batch(gs, ks, 0.03, seeds)
    got, _ = gp.partition_batch(gs, ks, 0.03, seeds, options=best["options"], workers=best["workers"])
    assert all(torch.equal(x, y) for x, y in zip(ref, got))
    rp, ci = gs[0]
    one = autotune_graph(rp, ci, ks[0], seed=seeds[0], ctas_per_sm=(2, 16), small_level_n=(0, 4096))
    assert len(one["table"]) == 4
    p1, _, _ = gp.partition(rp, ci, ks[0], 0.03, seeds[0], options=one["options"])
    assert torch.equal(p1, ref[0])
