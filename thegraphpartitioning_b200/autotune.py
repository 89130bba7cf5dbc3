"""Autotuner for the launch-shape knobs of the partitioner.

Every knob tuned here changes only how work is laid out on the device, never
the result: the partition of every graph is identical for every setting (the
parity tests run the same graphs under several settings).  So the tuner may
simply time candidates on a sample of the caller's own workload and keep the
fastest.

Knobs:
  * ``workers``        -- concurrent V-cycles (host threads / CUDA streams) of
                          a batched call;
  * ``small_level_n``  -- levels up to this many vertices refined by one
                          thread block per level (0: off);
  * ``ctas_per_sm``    -- grid of the neighbour-scan kernels (matching rounds,
                          connectivity pass, afterburner), in CTAs per SM;
  * ``heavy_deg``      -- degree-bucket threshold above which a row is scanned
                          by a whole CTA (8 warps per vertex) instead of one
                          warp or a lane group;
  * ``item_len``       -- tile size: entries of one CTA's piece of such a row.

    best = autotune_batch(graphs, ks)            # on a sample of a batch
    parts, stats = partition_batch(graphs, ks, options=best["options"], workers=best["workers"])

    best = autotune_graph(rowptr, colidx, k)     # one large graph
    part, stats, _ = partition(rowptr, colidx, k, options=best["options"])
"""
from __future__ import annotations

import itertools
import os
import time

from . import partition, partition_batch
from ._abi import make_options


def _sample(n_graphs: int, costs, size: int):
    """Indices of a sample that keeps the size mix: every step-th graph of the
    batch in decreasing cost order."""
    order = sorted(range(n_graphs), key=lambda i: (-int(costs[i]), i))
    if size >= n_graphs:
        return order
    step = n_graphs / float(size)
    return [order[int(j * step)] for j in range(size)]


def autotune_batch(graphs, ks, imbalances=0.03, seeds=0, sample: int = 256, reps: int = 1,
                   workers=None, small_level_n=(0, 2048), ctas_per_sm=(8, 64), heavy_deg=(4096,),
                   item_len=(32768,), log=None):
    """Time every (workers, small_level_n, ctas_per_sm, heavy_deg, item_len)
    combination on a sample of the batch (after one warm-up call each) and
    return the fastest: {"workers", "options", "seconds", "table"}.  The sample
    keeps the batch's size mix (every step-th graph in decreasing n + m)."""
    import torch
    G = len(graphs)
    per = lambda x: list(x) if isinstance(x, (list, tuple)) else [x] * G
    ks, imbs, sds = per(ks), per(imbalances), per(seeds)
    costs = [g[0].numel() + g[1].numel() for g in graphs]
    idx = _sample(G, costs, sample)
    gs = [graphs[i] for i in idx]
    kk, ii, ss = [ks[i] for i in idx], [imbs[i] for i in idx], [sds[i] for i in idx]
    if workers is None:
        cpus = os.cpu_count() or 16
        workers = sorted({max(1, cpus // 2), cpus, 2 * cpus})
    outs = [torch.empty(g[0].numel() - 1, dtype=torch.int32, device=g[0].device) for g in gs]
    table = []
    best = None
    for w, sl, cps, hd, il in itertools.product(workers, small_level_n, ctas_per_sm, heavy_deg, item_len):
        opt = make_options(small_level_n=sl, ctas_per_sm=cps, heavy_deg=hd, item_len=max(il, hd))
        partition_batch(gs, kk, ii, ss, options=opt, workers=w, outs=outs)
        torch.cuda.synchronize()
        t = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            partition_batch(gs, kk, ii, ss, options=opt, workers=w, outs=outs)
            torch.cuda.synchronize()
            t = min(t, time.perf_counter() - t0)
        row = {"workers": w, "small_level_n": sl, "ctas_per_sm": cps, "heavy_deg": hd, "item_len": max(il, hd),
               "seconds": t}
        table.append(row)
        if log:
            log(row)
        if best is None or t < best["seconds"]:
            best = row
    return {"workers": best["workers"],
            "options": make_options(small_level_n=best["small_level_n"], ctas_per_sm=best["ctas_per_sm"],
                                    heavy_deg=best["heavy_deg"], item_len=best["item_len"]),
            "seconds": best["seconds"], "sample": len(gs), "table": table}


def autotune_graph(rowptr, colidx, k: int, imbalance: float = 0.03, seed: int = 0, vwgt=None, ewgt=None,
                   ctas_per_sm=(16, 32, 64, 96), small_level_n=(0,), heavy_deg=(2048, 4096, 8192),
                   item_len=(16384, 32768, 65536), reps: int = 1, log=None):
    """Time full partitions of one graph (CUDA tensors) for every combination
    of the grid knobs, by the device time the library reports, and return the
    fastest: {"options", "ms", "table"}."""
    table = []
    best = None
    for cps, sl, hd, il in itertools.product(ctas_per_sm, small_level_n, heavy_deg, item_len):
        opt = make_options(ctas_per_sm=cps, small_level_n=sl, heavy_deg=hd, item_len=max(il, hd))
        partition(rowptr, colidx, k, imbalance, seed, vwgt=vwgt, ewgt=ewgt, options=opt)
        ms = min(partition(rowptr, colidx, k, imbalance, seed, vwgt=vwgt, ewgt=ewgt, options=opt)[1]["ms_total"]
                 for _ in range(reps))
        row = {"ctas_per_sm": cps, "small_level_n": sl, "heavy_deg": hd, "item_len": max(il, hd), "ms": ms}
        table.append(row)
        if log:
            log(row)
        if best is None or ms < best["ms"]:
            best = row
    return {"options": make_options(ctas_per_sm=best["ctas_per_sm"], small_level_n=best["small_level_n"],
                                    heavy_deg=best["heavy_deg"], item_len=best["item_len"]),
            "ms": best["ms"], "table": table}
