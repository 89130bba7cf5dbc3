"""Batched mode across ranks: the LPT shard assignment is deterministic,
disjoint, complete and balanced; two gloo ranks on the CPU agree on it."""
import os

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from thegraphpartitioning_b200 import graphs, shard_graphs


def test_shards_cover_and_balance():
    specs = graphs.batch_specs(512, seed=3)
    costs = [s["n"] * 6 for s in specs]
    for world in (1, 2, 3, 8):
        shards = shard_graphs(costs, world)
        flat = sorted(i for sh in shards for i in sh)
        assert flat == list(range(len(specs)))
        loads = [sum(costs[i] for i in sh) for sh in shards]
        assert max(loads) - min(loads) <= max(costs)


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    specs = graphs.batch_specs(256, seed=11)
    shards = shard_graphs([s["n"] for s in specs], world)
    mine = torch.tensor(shards[rank] + [-1] * (256 - len(shards[rank])))
    gathered = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(gathered, mine)
    got = sorted(int(x) for t in gathered for x in t if x >= 0)
    out[rank] = int(got == list(range(256)))
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_shards():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == 1 and out[1] == 1


def test_autotune_sample_keeps_size_mix():
    """The tuner's sample: distinct indices, every step-th graph of the batch in
    decreasing cost order, so large and small graphs are both represented."""
    from thegraphpartitioning_b200.autotune import _sample
    costs = [(i * 7919) % 1000 + 1 for i in range(1000)]
    idx = _sample(len(costs), costs, 100)
    assert len(idx) == 100 and len(set(idx)) == 100
    order = sorted(range(1000), key=lambda i: (-costs[i], i))
    assert idx[0] == order[0]                      # the largest graph is in
    assert [costs[i] for i in idx] == sorted((costs[i] for i in idx), reverse=True)
    ranks = [order.index(i) for i in idx]
    assert max(ranks) >= 900                       # and the small end too
    assert _sample(5, [3, 1, 2, 5, 4], 10) == [3, 4, 0, 2, 1]   # sample larger than the batch: all, by cost
