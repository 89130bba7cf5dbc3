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
    one = autotune_graph(rp, ci, ks[0], seed=seeds[0], ctas_per_sm=(2, 16), small_level_n=(0, 4096),
                         heavy_deg=(64, 2048), item_len=(256,))
    assert len(one["table"]) == 8
    p1, _, _ = gp.partition(rp, ci, ks[0], 0.03, seeds[0], options=one["options"])
    assert torch.equal(p1, ref[0])


def test_batch_stages_match_single_calls(gp, cuda):
    """Graphs whose levels are all small (refined entirely by the persistent
    one-block kernel), graphs whose finer levels are large (handed back to the
    multi-kernel loop), a hub whose input level has rows over 2048 entries, and
    a weighted graph: each result, cut and refinement-step count equals the
    single-graph call's."""
    from helpers import star_plus_grid, weighted
    specs = graphs.batch_specs(10, seed=11, nmin=2000, nmax=60000)
    gs = [graphs.batch_graph(s, device=cuda) for s in specs]
    ks = [s["k"] for s in specs]
    seeds = [s["seed"] for s in specs]
    rp, ci = star_plus_grid(leaves=5000, side=30)
    gs.append((rp.to(cuda), ci.to(cuda))); ks.append(6); seeds.append(4)
    rp, ci = graphs.grid2d(90, 110)
    ew, vw = weighted(rp.numpy(), ci.numpy(), seed=2)
    gs.append((rp.to(cuda), ci.to(cuda), torch.from_numpy(vw).to(cuda), torch.from_numpy(ew).to(cuda)))
    ks.append(9); seeds.append(1)
    parts, stats = gp.partition_batch(gs, ks, 0.03, seeds, workers=5)
    for g, k, sd, p, st in zip(gs, ks, seeds, parts, stats):
        vw_ = g[2] if len(g) > 2 else None
        ew_ = g[3] if len(g) > 3 else None
        single, sst, _ = gp.partition(g[0], g[1], k, 0.03, sd, vwgt=vw_, ewgt=ew_)
        assert torch.equal(single, p)
        for key in ("cut", "max_part_weight", "levels", "coarsest_n", "refine_iters"):
            assert st[key] == sst[key], (key, st[key], sst[key])
