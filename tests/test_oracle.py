"""CPU tests of the oracle (the checker) and of the METIS baseline harness.

The reference ships no tests or golden vectors (its only worked example is the
5-vertex CSR preview in README.md), so the oracle is pinned by known answers:
paths (optimum k-1), rings (optimum k), disjoint cliques (0), two cliques joined by one edge (1),
grids (optimum min(R, C) for a bisection), plus exact invariants on every run.
"""
import numpy as np
import pytest
import torch

from thegraphpartitioning_b200 import graphs
from helpers import check_csr, to_np, weighted, star_plus_grid


def _check_result(oracle, rp, ci, part, st, k, imb=0.03, ew=None, vw=None):
    part = np.asarray(part)
    assert part.shape == (len(rp) - 1,)
    assert part.min() >= 0 and part.max() < k
    cut, pw = oracle.edge_cut(rp, ci, part, k, ewgt=ew, vwgt=vw)
    assert cut == st["cut"]
    assert pw.max() == st["max_part_weight"]
    assert pw.sum() == st["total_weight"]
    assert st["max_allowed"] == oracle.lmax(pw.sum(), k, imb)
    return cut, pw


@pytest.mark.parametrize("n,k", [(1000, 2), (1000, 4), (5000, 8), (3000, 7)])
def test_path_optimum(oracle_mod, n, k):
    rp, ci = to_np(*graphs.path(n))
    part, st, _ = oracle_mod.partition(rp, ci, k, 0.03, seed=0)
    cut, pw = _check_result(oracle_mod, rp, ci, part, st, k)
    assert cut == k - 1
    assert pw.max() <= st["max_allowed"]


def _ring(n):
    rows = [sorted({(v - 1) % n, (v + 1) % n}) for v in range(n)]
    rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int64)
    return rp, np.array([u for r in rows for u in r], dtype=np.int32)


@pytest.mark.parametrize("n,k,slack", [(100, 4, 0), (999, 7, 0), (1000, 8, 0), (4096, 64, 2)])
def test_ring_optimum(oracle_mod, n, k, slack):
    """A cycle cut into k arcs has the optimal cut k; small k reach it exactly
    on every seed, k = 64 on 4096 vertices within two extra edges."""
    rp, ci = _ring(n)
    for seed in range(3):
        part, st, _ = oracle_mod.partition(rp, ci, k, 0.03, seed=seed)
        cut, pw = _check_result(oracle_mod, rp, ci, part, st, k)
        assert k <= cut <= k + slack
        assert pw.max() <= st["max_allowed"]


@pytest.mark.parametrize("count,size", [(8, 20), (4, 50), (16, 12)])
def test_disjoint_cliques_zero_cut(oracle_mod, count, size):
    rp, ci = to_np(*graphs.cliques(count, size))
    part, st, _ = oracle_mod.partition(rp, ci, count, 0.0, seed=3)
    cut, pw = _check_result(oracle_mod, rp, ci, part, st, count, imb=0.0)
    assert cut == 0
    assert np.all(pw == size)


def test_two_cliques_one_bridge(oracle_mod):
    rp, ci = graphs.cliques(2, 30)
    s = np.repeat(np.arange(60), np.diff(rp.numpy()))
    d = ci.numpy().astype(np.int64)
    s = np.concatenate([s, [29, 30]]); d = np.concatenate([d, [30, 29]])
    rp2, ci2, _ = graphs.csr_from_edges(torch.from_numpy(s), torch.from_numpy(d), 60)
    rp2, ci2 = to_np(rp2, ci2)
    part, st, _ = oracle_mod.partition(rp2, ci2, 2, 0.0, seed=0)
    cut, _ = _check_result(oracle_mod, rp2, ci2, part, st, 2, imb=0.0)
    assert cut == 1


@pytest.mark.parametrize("rows,cols,k,bound", [(8, 8, 4, 16), (32, 64, 2, 32), (64, 64, 4, 128)])
def test_grid_near_optimum(oracle_mod, rows, cols, k, bound):
    rp, ci = to_np(*graphs.grid2d(rows, cols))
    part, st, _ = oracle_mod.partition(rp, ci, k, 0.03, seed=0)
    cut, pw = _check_result(oracle_mod, rp, ci, part, st, k)
    assert bound <= cut <= int(1.6 * bound)
    assert pw.max() <= st["max_allowed"]


def test_metis_harness_probe(oracle_mod):
    """METIS from the CUDA toolkit on an 8x8 grid, k=4: cut 16, sizes 16."""
    rp, ci = to_np(*graphs.grid2d(8, 8))
    part, cut, _ = oracle_mod.metis(rp, ci, 4)
    assert cut == 16
    assert np.all(np.bincount(part, minlength=4) == 16)


def test_quality_vs_metis_small(oracle_mod):
    for name, (rp, ci), k in [("grid", graphs.grid2d(96, 96), 8), ("rmat", graphs.rmat(13)[:2], 16),
                              ("cl", graphs.chung_lu(20000, 70000, seed=1), 16)]:
        rp, ci = to_np(rp, ci)
        part, st, _ = oracle_mod.partition(rp, ci, k, 0.03, seed=0)
        _check_result(oracle_mod, rp, ci, part, st, k)
        _, mcut, _ = oracle_mod.metis(rp, ci, k)
        assert st["cut"] <= 1.35 * mcut, (name, st["cut"], mcut)
        assert st["max_part_weight"] <= st["max_allowed"], name


def test_weighted_invariants(oracle_mod):
    rp, ci = to_np(*graphs.grid2d(40, 50))
    ew, vw = weighted(rp, ci, seed=2)
    part, st, ev = oracle_mod.partition(rp, ci, 6, 0.05, seed=5, vwgt=vw, ewgt=ew, trace=True)
    _check_result(oracle_mod, rp, ci, part, st, 6, imb=0.05, ew=ew, vw=vw)
    # coarse graphs conserve vertex weight and are symmetric without self-loops
    total = int(vw.sum())
    for e in ev:
        if e["kind"] == 2:
            check_csr(e["rowptr"], e["colidx"])
            assert int(e["vwgt"].sum()) == total


def test_determinism_and_seed(oracle_mod):
    rp, ci = to_np(*graphs.rmat(12, seed=4)[:2])
    a, sa, _ = oracle_mod.partition(rp, ci, 8, 0.03, seed=7)
    b, sb, _ = oracle_mod.partition(rp, ci, 8, 0.03, seed=7)
    c, _, _ = oracle_mod.partition(rp, ci, 8, 0.03, seed=8)
    assert np.array_equal(a, b) and sa == sb
    assert not np.array_equal(a, c)


def test_heavy_rows_and_trace_structure(oracle_mod):
    rp, ci = to_np(*star_plus_grid())
    part, st, ev = oracle_mod.partition(rp, ci, 4, 0.03, seed=1, trace=True,
                                        options={"coarsen_to": 200})
    _check_result(oracle_mod, rp, ci, part, st, 4)
    kinds = [e["kind"] for e in ev]
    assert kinds[0] == 1 and 3 in kinds and kinds[-1] == 5
    # match arrays are involutions
    for e in ev:
        if e["kind"] == 1:
            m = e["a0"]
            idx = np.nonzero(m >= 0)[0]
            assert np.array_equal(m[m[idx]], idx)


def test_k1_and_k_equals_n(oracle_mod):
    rp, ci = to_np(*graphs.grid2d(5, 5))
    part, st, _ = oracle_mod.partition(rp, ci, 1)
    assert np.all(part == 0) and st["cut"] == 0
    part, st, _ = oracle_mod.partition(rp, ci, 25, 0.0)
    assert sorted(part.tolist()) == list(range(25))
    assert st["cut"] == ci.size // 2


@pytest.mark.parametrize("case", ["k0", "kbig", "imb", "self", "range", "rowptr", "weight", "asym"])
def test_invalid_inputs(oracle_mod, case):
    rp, ci = to_np(*graphs.grid2d(4, 4))
    k, imb, ew, opts = 2, 0.03, None, None
    if case == "k0":
        k = 0
    elif case == "kbig":
        k = 17
    elif case == "imb":
        imb = -0.1
    elif case == "self":
        ci = ci.copy(); ci[0] = 0
    elif case == "range":
        ci = ci.copy(); ci[3] = 99
    elif case == "rowptr":
        rp = rp.copy(); rp[5] = rp[7]
    elif case == "weight":
        ew = np.ones(len(ci), np.int32); ew[2] = 0
    elif case == "asym":
        rp = np.array([0, 2, 4, 4, 5, 6]); ci = np.array([1, 2, 0, 3, 4, 2], np.int32)
        opts = {"check_input": 2}
    with pytest.raises(oracle_mod.OracleError) as ei:
        oracle_mod.partition(rp, ci, k, imb, ewgt=ew, options=opts)
    assert ei.value.code == -1


def test_rule_helpers(oracle_mod):
    # log-scale loss buckets are monotone and stay in 10 bits
    xs = sorted(set([-(2 ** 31) + 1, -70000, -100, -64, -63, -1, 0, 1, 63, 64, 65, 1000, 2 ** 20, 2 ** 31 - 1]))
    bs = [oracle_mod.loss_bucket(x) for x in xs]
    assert bs == sorted(bs) and 0 < min(bs) and max(bs) < 1024
    # edge hash is symmetric in its endpoints
    assert oracle_mod.edge_hash(5, 2, 10, 77) == oracle_mod.edge_hash(5, 2, 77, 10)


def test_priority_hook_with_edge_weights_is_plain(oracle_mod):
    """The learned mode's matching-priority hook, given each level's own edge
    weights as priorities, must reproduce the plain V-cycle event for event
    (the priority replaces exactly the edge weight's place in the key)."""
    from thegraphpartitioning_b200 import graphs
    from helpers import to_np, weighted
    from thegraphpartitioning_b200._abi import GP_TR_CONTRACT
    for g, k, w in ((graphs.rmat(12, seed=4)[:2], 16, False), (graphs.grid2d(40, 45), 5, True)):
        rp, ci = to_np(*g)
        ew = vw = None
        if w:
            ew, vw = weighted(rp, ci, seed=3)
        p0, s0, ev0 = oracle_mod.partition(rp, ci, k, 0.03, 6, vwgt=vw, ewgt=ew, trace=True)
        prio = {0: ew if ew is not None else np.ones(len(ci), np.int32)}
        for e in ev0:
            if e["kind"] == GP_TR_CONTRACT:
                prio[e["level"] + 1] = e["ewgt"]
        p1, s1, ev1 = oracle_mod.partition(rp, ci, k, 0.03, 6, vwgt=vw, ewgt=ew, trace=True, prio_levels=prio)
        assert np.array_equal(p0, p1) and s0["cut"] == s1["cut"]
        assert len(ev0) == len(ev1)
        for a, b in zip(ev0, ev1):
            assert a["kind"] == b["kind"] and a["level"] == b["level"] and a["iter"] == b["iter"]
            if "a0" in a:
                assert np.array_equal(a["a0"], b["a0"])
