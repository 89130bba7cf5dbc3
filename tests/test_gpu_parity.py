"""GPU parity: the sm_100a library against the CPU oracle, bit-exact.

Every case runs the full V-cycle on both sides with tracing on and compares,
event by event: the matching of every level, the fine->coarse map and coarse
CSR (ids, weights, vertex weights), the kept initial-partition trial, each
refinement iteration's proposals (destination, gain), its resulting partition
and the cut/heaviest-part before it, and the partition after each level.
"""
import numpy as np
import pytest
import torch

from thegraphpartitioning_b200 import graphs
from helpers import compare_traces, multi_star_grid, star_plus_grid, to_np, weighted

pytestmark = pytest.mark.gpu


def _cases():
    yield "grid64_k4", graphs.grid2d(64, 64), 4, 0.03, None, {}
    yield "grid48x80_k7", graphs.grid2d(48, 80), 7, 0.05, None, {}
    yield "rmat12_k16", graphs.rmat(12, seed=1)[:2], 16, 0.03, None, {}
    yield "chunglu_k8", graphs.chung_lu(12000, 40000, seed=2), 8, 0.03, None, {}
    yield "grid3d_k32", graphs.grid3d(16, 16, 16), 32, 0.03, None, {}
    yield "weighted_k5", graphs.grid2d(40, 50), 5, 0.05, "w", {}
    yield "star_heavy_k4", star_plus_grid(), 4, 0.03, None, {"coarsen_to": 200}
    # a hub of 40000 leaves: rows split over several CTAs, longest contraction tier
    yield "megahub_k8", star_plus_grid(leaves=40000, side=64), 8, 0.03, None, {}
    yield "megahub_w_k3", star_plus_grid(leaves=36000, side=40), 3, 0.05, "w", {"coarsen_to": 300}
    # a 150000-leaf hub: its coarse row is contracted by several CTAs sharing one table
    yield "gigahub_k4", star_plus_grid(leaves=150000, side=32), 4, 0.03, None, {}
    # hubs of 700 to 90,000 leaves: coarse rows in every contraction tier (C1, C, C2, C3, D)
    yield "multistar_k8", multi_star_grid(), 8, 0.03, None, {}
    yield "multistar_w_k5", multi_star_grid(seed=1), 5, 0.05, "w", {}
    yield "rmat11_k64_tight", graphs.rmat(11, seed=3)[:2], 64, 0.0, None, {}
    yield "er_k3_nohop", graphs.erdos_renyi(3000, 3.0, seed=5), 3, 0.02, None, {"two_hop": -1}
    yield "rgg_k2", graphs.random_geometric(4000, 8.0, seed=6), 2, 0.03, None, {"init_trials": 8}
    # the same workloads with every level refined by the multi-kernel loop, or
    # with a mix of both paths (small_level_n: levels above it multi-kernel)
    yield "rmat12_k16_multikernel", graphs.rmat(12, seed=1)[:2], 16, 0.03, None, {"small_level_n": -1}
    yield "grid3d_k32_multikernel", graphs.grid3d(16, 16, 16), 32, 0.03, None, {"small_level_n": -1}
    yield "weighted_k5_mixed", graphs.grid2d(40, 50), 5, 0.05, "w", {"small_level_n": 1200}
    yield "chunglu_k8_mixed", graphs.chung_lu(12000, 40000, seed=2), 8, 0.03, None, {"small_level_n": 3000}
    yield "er_k64_cta", graphs.erdos_renyi(16000, 8.0, seed=8), 64, 0.03, None, {"small_level_n": 16384}
    yield "rmat12_k16_ctas2", graphs.rmat(12, seed=1)[:2], 16, 0.03, None, {"ctas_per_sm": 2}
    # degree-bucket threshold and CTA piece length (autotuner knobs): most rows
    # scanned by whole CTAs, long rows split into many pieces
    yield "rmat12_k16_heavy64", graphs.rmat(12, seed=1)[:2], 16, 0.03, None, {"heavy_deg": 64, "item_len": 96}
    yield "weighted_k5_heavy64", graphs.grid2d(40, 50), 5, 0.05, "w", {"heavy_deg": 64, "small_level_n": 1200}
    # a longer refinement patience (more label-propagation / rebalancing cycles per level),
    # in the multi-kernel loop and in the one-block level loop
    yield "rmat12_k16_patience12", graphs.rmat(12, seed=1)[:2], 16, 0.03, None, {"refine_patience": 12}
    yield "er_k64_cta_patience12", graphs.erdos_renyi(16000, 8.0, seed=8), 64, 0.03, None, \
        {"small_level_n": 16384, "refine_patience": 12}
    # many parts: histograms of k bins, rebalancing over hundreds of parts
    yield "chunglu_k512", graphs.chung_lu(20000, 70000, seed=12), 512, 0.03, None, {}
    yield "grid120_k1000_w", graphs.grid2d(120, 120), 1000, 0.05, "w", {}
    yield "rmat13_k1024_cta", graphs.rmat(13, seed=13)[:2], 1024, 0.03, None, {"small_level_n": 16384}
    # exact balance on 50k-60k vertices: rebalance steps with more candidates
    # than one thread block sorts (radix-sorted multi-kernel path), weak and strong
    yield "rgg50k_k2_bigrb", graphs.random_geometric(50000, 8.0, seed=9), 2, 0.0, None, {}
    yield "er60k_k3_bigrb", graphs.erdos_renyi(60000, 10.0, seed=3), 3, 0.0, None, {}


CASES = list(_cases())


@pytest.mark.parametrize("name,g,k,imb,w,opts", CASES, ids=[c[0] for c in CASES])
def test_trace_parity(oracle_mod, gp, cuda, name, g, k, imb, w, opts):
    rp, ci = to_np(*g)
    ew = vw = None
    if w:
        ew, vw = weighted(rp, ci, seed=9)
    seed = 11
    p_ref, s_ref, ev_ref = oracle_mod.partition(rp, ci, k, imb, seed, vwgt=vw, ewgt=ew, options=opts, trace=True)
    # device entry point through torch CUDA tensors
    d = lambda a: None if a is None else torch.from_numpy(a).to(cuda)
    p_gpu, s_gpu, ev_gpu = gp.partition(d(rp), d(ci), k, imb, seed, vwgt=d(vw), ewgt=d(ew), options=opts, trace=True)
    compare_traces(ev_ref, ev_gpu)
    assert np.array_equal(p_ref, p_gpu.cpu().numpy())
    for key in ("cut", "max_part_weight", "total_weight", "max_allowed", "levels", "coarsest_n",
                "best_trial", "refine_iters"):
        assert s_ref[key] == s_gpu[key], (key, s_ref[key], s_gpu[key])


def test_host_entry_point_matches_oracle(oracle_mod, gp, cuda):
    rp, ci = to_np(*graphs.rmat(13, seed=2)[:2])
    p_ref, s_ref, _ = oracle_mod.partition(rp, ci, 32, 0.03, 5)
    p_gpu, s_gpu, _ = gp.partition(rp, ci, 32, 0.03, 5)
    assert np.array_equal(p_ref, p_gpu)
    assert s_ref["cut"] == s_gpu["cut"]


def test_edge_cut_device(oracle_mod, gp, cuda):
    rp, ci = to_np(*graphs.chung_lu(30000, 100000, seed=4))
    ew, vw = weighted(rp, ci, seed=1)
    k = 13
    part = (np.arange(len(rp) - 1) * 7919 % k).astype(np.int32)
    cut_ref, pw_ref = oracle_mod.edge_cut(rp, ci, part, k, ewgt=ew, vwgt=vw)
    d = lambda a: torch.from_numpy(a).to(cuda)
    cut, pw = gp.edge_cut(d(rp), d(ci), d(part), k, ewgt=d(ew), vwgt=d(vw))
    assert cut == cut_ref
    assert np.array_equal(pw, pw_ref)


def test_determinism_repeated_calls(gp, cuda):
    rp, ci = graphs.rmat(14, seed=7)[:2]
    rp, ci = rp.to(cuda), ci.to(cuda)
    outs = [gp.partition(rp, ci, 64, 0.03, 3)[0].cpu().numpy() for _ in range(3)]
    assert all(np.array_equal(outs[0], o) for o in outs[1:])


@pytest.mark.parametrize("case", ["self", "range", "rowptr", "weight", "asym", "k0", "kbig"])
def test_device_rejects_invalid(gp, cuda, case):
    rp, ci = to_np(*graphs.grid2d(6, 6))
    k, ew, opts = 2, None, None
    if case == "self":
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
    elif case == "k0":
        k = 0
    elif case == "kbig":
        k = 37
    d = lambda a: None if a is None else torch.from_numpy(np.asarray(a)).to(cuda)
    with pytest.raises(gp.GPError) as ei:
        gp.partition(d(rp.astype(np.int64)), d(ci.astype(np.int32)), k, 0.03, ewgt=d(ew), options=opts)
    assert ei.value.code == -1
    # the context is still usable afterwards
    rp2, ci2 = graphs.grid2d(8, 8)
    p, st, _ = gp.partition(rp2.to(cuda), ci2.to(cuda), 4)
    assert st["cut"] >= 16


def test_full_size_grid_config(oracle_mod, gp, cuda):
    """512x512 grid, k=4, 3%: identical to the oracle at full size."""
    rp, ci = to_np(*graphs.grid2d(512, 512))
    p_ref, s_ref, _ = oracle_mod.partition(rp, ci, 4, 0.03, 0)
    p_gpu, s_gpu, _ = gp.partition(torch.from_numpy(rp).to(cuda), torch.from_numpy(ci).to(cuda), 4, 0.03, 0)
    assert np.array_equal(p_ref, p_gpu.cpu().numpy())
    assert s_gpu["max_part_weight"] <= s_gpu["max_allowed"]


def _edge_cases():
    # two vertices, two parts
    yield "pair_k2", (np.array([0, 1, 2], np.int64), np.array([1, 0], np.int32)), 2, 0.0, None
    # one part per vertex
    rp, ci = to_np(*graphs.grid2d(5, 6))
    yield "grid_k_eq_n", (rp, ci), 30, 0.03, None
    # a clique
    yield "clique50_k7", to_np(*graphs.cliques(1, 50)), 7, 0.03, None
    # many components (2000 disjoint 4-cliques)
    yield "components_k16", to_np(*graphs.cliques(2000, 4)), 16, 0.03, None
    # a path (diameter = n - 1)
    yield "path3000_k9", to_np(*graphs.path(3000)), 9, 0.03, None
    # isolated vertices mixed in (Erdos-Renyi with mean degree 1)
    yield "sparse_er_k5", to_np(*graphs.erdos_renyi(6000, 1.0, seed=3)), 5, 0.03, None
    # heavy weights whose totals come close to the int32 limit
    rp, ci = to_np(*graphs.grid2d(30, 30))
    n = len(rp) - 1
    ew = np.full(len(ci), 2 * 10**5, np.int32)
    vw = np.full(n, 2 * 10**6, np.int32)
    yield "heavy_weights_k6", (rp, ci), 6, 0.03, (ew, vw)


ECASES = list(_edge_cases())


@pytest.mark.parametrize("name,g,k,imb,w", ECASES, ids=[c[0] for c in ECASES])
def test_edge_case_parity(oracle_mod, gp, cuda, name, g, k, imb, w):
    rp, ci = g
    ew, vw = (w if w is not None else (None, None))
    p_ref, s_ref, ev_ref = oracle_mod.partition(rp, ci, k, imb, 3, vwgt=vw, ewgt=ew, trace=True)
    d = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    p_gpu, s_gpu, ev_gpu = gp.partition(d(rp), d(ci), k, imb, 3, vwgt=d(vw), ewgt=d(ew), trace=True)
    compare_traces(ev_ref, ev_gpu)
    assert np.array_equal(p_ref, p_gpu.cpu().numpy())
    assert s_ref["cut"] == s_gpu["cut"] and s_ref["max_part_weight"] == s_gpu["max_part_weight"]
    cut, pw = gp.edge_cut(d(rp), d(ci), p_gpu, k, ewgt=d(ew), vwgt=d(vw))
    assert cut == s_gpu["cut"] and int(pw.max()) == s_gpu["max_part_weight"]


# ---- the co-purchase-shaped configuration at its full size: Chung-Lu graph
# drawn on 262,111 vertices with ~900k undirected edges (degree exponent 2.5,
# maximum expected degree 420); the 7,236 vertices left isolated are dropped,
# as the reference's preprocessing does, leaving 254,875.  k swept over 2..64,
# unit weights, 3 % imbalance.  k = 64 compares every trace event; the other
# k compare the final partition and statistics.
CL_KS = (2, 4, 8, 16, 32, 64)


@pytest.fixture(scope="module")
def chunglu_config():
    rp, ci = to_np(*graphs.chung_lu())
    assert len(rp) - 1 == 254875 and len(ci) // 2 == 899727
    return rp, ci


@pytest.mark.parametrize("k", CL_KS)
def test_chunglu_config_k_sweep(oracle_mod, gp, cuda, chunglu_config, k):
    rp, ci = chunglu_config
    trace = k == 64
    p_ref, s_ref, ev_ref = oracle_mod.partition(rp, ci, k, 0.03, 0, trace=trace)
    p_gpu, s_gpu, ev_gpu = gp.partition(torch.from_numpy(rp).to(cuda), torch.from_numpy(ci).to(cuda), k, 0.03, 0,
                                        trace=trace)
    if trace:
        compare_traces(ev_ref, ev_gpu)
    assert np.array_equal(p_ref, p_gpu.cpu().numpy())
    for key in ("cut", "max_part_weight", "max_allowed", "levels", "coarsest_n", "best_trial", "refine_iters"):
        assert s_ref[key] == s_gpu[key], (key, s_ref[key], s_gpu[key])
    assert s_gpu["max_part_weight"] <= s_gpu["max_allowed"]


def test_rmat20_k64_matches_oracle(oracle_mod, gp, cuda):
    """R-MAT scale 20 (646k vertices, 15.7M undirected edges), k = 64: the
    largest R-MAT the oracle finishes in about half a minute, bit-exact."""
    rp, ci = graphs.rmat(20, 16, seed=0)[:2]
    p_ref, s_ref, _ = oracle_mod.partition(rp.numpy(), ci.numpy(), 64, 0.03, 0)
    p_gpu, s_gpu, _ = gp.partition(rp.to(cuda), ci.to(cuda), 64, 0.03, 0)
    assert np.array_equal(p_ref, p_gpu.cpu().numpy())
    for key in ("cut", "max_part_weight", "levels", "coarsest_n", "refine_iters"):
        assert s_ref[key] == s_gpu[key], (key, s_ref[key], s_gpu[key])


def test_headline_config_matches_full_fixture(gp, cuda):
    """R-MAT scale 24, k = 64 (the benchmark workload, 260M undirected edges):
    the graph generated on the device and the partition of it are the ones
    the oracle recorded in tests/golden/rmat24_ef16_k64_full.json (SHA-256 of
    the CSR and of the part array, cut, heaviest part, levels)."""
    import hashlib
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rmat24_ef16_k64_full.json")
    with open(path) as f:
        fx = json.load(f)
    rp, ci, _ = graphs.rmat(24, 16, seed=0, device=cuda)
    def sha(*ts):
        h = hashlib.sha256()
        for t in ts:
            h.update(t.cpu().numpy().view(np.uint8).data)
        return h.hexdigest()
    assert sha(rp, ci) == fx["graph"]["sha256_rowptr_colidx"]
    part, st, _ = gp.partition(rp, ci, 64, 0.03, 0)
    orc = fx["oracle"]
    assert (st["cut"], st["max_part_weight"], st["levels"], st["coarsest_n"]) == \
        (orc["cut"], orc["max_part_weight"], orc["levels"], orc["coarsest_n"])
    assert sha(part) == orc["sha256_part"]
