"""GPU checks of the learned matching priorities.

* forward: the kernels' logits against oracle/gnn_ref.py (float64, same
  BF16-rounded parameters), tolerance 2e-4 + 2e-4*|t| per entry;
* backward: the kernels' gradient against the float64 chain rule, relative
  error of every parameter block below 2e-3 (FP32 accumulation);
* the learned V-cycle is bit-exact against the oracle fed the same per-level
  priorities (every trace event compared);
* training on the GPU reduces the loss; the fallback mode never returns a cut
  above the plain one, and returns exactly the plain partition when it
  rejects the learned one.
"""
import os

import numpy as np
import pytest
import torch

from thegraphpartitioning_b200 import graphs
from thegraphpartitioning_b200 import learned
from thegraphpartitioning_b200._abi import GP_TR_PRIO, GP_TR_MOVE_PRIO
from helpers import compare_traces, to_np, weighted

pytestmark = pytest.mark.gpu

ATOL, RTOL = 2e-4, 2e-4


def _params(seed):
    p = learned.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    p[learned.O_B1:learned.O_P] = rng.normal(0, 0.3, learned.H)
    p[learned.O_B2:learned.O_Z] = rng.normal(0, 0.3, learned.H)
    p[learned.O_BETA + 1] = 0.4   # gamma
    p[learned.O_BETA + 2] = -0.2  # delta
    p[learned.O_ETA] = 0.7        # common-neighbour coefficient
    return p


def _graph_cases():
    rp, ci = to_np(*graphs.grid2d(30, 33))
    ew, vw = weighted(rp, ci, seed=3)
    yield "grid_w", rp, ci, vw, ew, 2
    rp, ci = to_np(*graphs.chung_lu(6000, 20000, seed=8))
    yield "chunglu", rp, ci, None, None, 0
    rp, ci = to_np(*graphs.rmat(11, seed=4)[:2])
    ew, vw = weighted(rp, ci, seed=5)
    yield "rmat_w", rp, ci, vw, ew, 5


GCASES = list(_graph_cases())


def _dev(a, cuda):
    return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


@pytest.mark.parametrize("name,rp,ci,vw,ew,level", GCASES, ids=[c[0] for c in GCASES])
def test_forward_matches_reference(gp, cuda, name, rp, ci, vw, ew, level):
    from oracle import gnn_ref
    p = _params(1)
    model = gp.GNN(p)
    prio, logit = model.forward(_dev(rp, cuda), _dev(ci, cuda), _dev(vw, cuda), _dev(ew, cuda), level)
    t_ref = gnn_ref.forward(gnn_ref.bf16_round(p), rp, ci, vw, ew, level)
    t = logit.cpu().numpy().astype(np.float64)
    err = np.abs(t - t_ref)
    assert np.all(err <= ATOL + RTOL * np.abs(t_ref)), (name, err.max())
    # the priority is the quantised logit; symmetric entries carry the same value
    pr = prio.cpu().numpy()
    assert np.all(np.abs(pr.astype(np.int64) - gnn_ref.priorities(t_ref).astype(np.int64))
                  <= 1 + 65536 * (ATOL + RTOL * np.abs(t_ref)))
    n = len(rp) - 1
    src = np.repeat(np.arange(n), np.diff(rp))
    key = src.astype(np.int64) * n + ci
    rkey = ci.astype(np.int64) * n + src
    order = np.argsort(key)
    pos = order[np.searchsorted(key[order], rkey)]
    assert np.array_equal(pr, pr[pos])


@pytest.mark.parametrize("name,rp,ci,vw,ew,level", GCASES, ids=[c[0] for c in GCASES])
def test_gradient_matches_reference(gp, cuda, name, rp, ci, vw, ew, level):
    from oracle import gnn_ref
    p = _params(2)
    n = len(rp) - 1
    part = (np.arange(n) * 5 // n).astype(np.int32)
    src = np.repeat(np.arange(n), np.diff(rp))
    label = (part[src] == part[ci]).astype(np.uint8)
    model = gp.GNN(p)
    loss, g = model.grad(_dev(rp, cuda), _dev(ci, cuda), _dev(label, cuda), _dev(vw, cuda), _dev(ew, cuda), level)
    loss_ref, g_ref = gnn_ref.loss_and_grad(gnn_ref.bf16_round(p), rp, ci, label, vw, ew, level)
    assert abs(loss - loss_ref) <= 1e-5 + 1e-5 * abs(loss_ref)
    blocks = [("W1", gnn_ref.O_W1, gnn_ref.O_B1), ("b1", gnn_ref.O_B1, gnn_ref.O_P), ("P", gnn_ref.O_P, gnn_ref.O_W2),
              ("W2", gnn_ref.O_W2, gnn_ref.O_B2), ("b2", gnn_ref.O_B2, gnn_ref.O_Z), ("Z", gnn_ref.O_Z, gnn_ref.O_A),
              ("edge", gnn_ref.O_A, gnn_ref.NPARAM)]
    for bname, lo, hi in blocks:
        ref = g_ref[lo:hi]
        rel = np.linalg.norm(g[lo:hi] - ref) / max(np.linalg.norm(ref), 1e-12)
        assert rel < 2e-3, (name, bname, rel)


def test_learned_vcycle_matches_oracle(oracle_mod, gp, cuda):
    """The integer path of the learned mode is the plain path with the
    priorities substituted: the oracle, given the GPU's per-level priorities,
    reproduces every event of the learned run."""
    for g, k, w, seed, max_level in ((graphs.rmat(13, seed=21)[:2], 16, False, 3, -1),
                                     (graphs.grid2d(70, 60), 6, True, 4, -1),
                                     (graphs.rmat(13, seed=22)[:2], 8, False, 5, 0)):
        rp, ci = to_np(*g)
        ew = vw = None
        if w:
            ew, vw = weighted(rp, ci, seed=7)
        model = gp.GNN(_params(3), prio_bits=10, max_level=max_level)
        part, st, rep, ev = gp.partition_learned(_dev(rp, cuda), _dev(ci, cuda), k, model, 0.03, seed,
                                                 vwgt=_dev(vw, cuda), ewgt=_dev(ew, cuda), fallback=False, trace=True)
        prio = {e["level"]: e["a0"] for e in ev if e["kind"] == GP_TR_PRIO}
        assert prio and rep["kept_learned"] == 1
        if max_level >= 0:
            assert set(prio) == set(range(max_level + 1))
        ev_gpu = [e for e in ev if e["kind"] != GP_TR_PRIO]
        p_ref, s_ref, ev_ref = oracle_mod.partition(rp, ci, k, 0.03, seed, vwgt=vw, ewgt=ew, trace=True,
                                                    prio_levels=prio)
        compare_traces(ev_ref, ev_gpu)
        assert np.array_equal(p_ref, part.cpu().numpy())
        assert s_ref["cut"] == st["cut"]


def test_training_reduces_loss(gp, cuda):
    samples = []
    for i in range(12):
        spec = learned.graph_spec(i, seed=5, nmin=2000, nmax=6000)
        rp, ci = learned.make_graph(spec, cuda)
        samples.extend(learned.level_samples(rp, ci, 8, seed=i))
    model = gp.GNN(learned.init_params(0))
    first = np.mean([model.grad(s[0], s[1], s[5], s[2], s[3], s[4])[0] for s in samples])
    learned.train(model, samples, epochs=6, batch=8, lr=3e-3)
    last = np.mean([model.grad(s[0], s[1], s[5], s[2], s[3], s[4])[0] for s in samples])
    assert last < 0.97 * first, (first, last)
    # trained weights round-trip through the host
    p = model.get_params()
    assert np.all(np.isfinite(p))
    m2 = gp.GNN(p)
    s = samples[0]
    assert torch.equal(model.forward(s[0], s[1], s[2], s[3], s[4])[0], m2.forward(s[0], s[1], s[2], s[3], s[4])[0])


def test_fallback_mode_never_worse(gp, cuda):
    rp, ci = graphs.rmat(14, seed=9)[:2]
    rp, ci = rp.to(cuda), ci.to(cuda)
    plain, sp, _ = gp.partition(rp, ci, 32, 0.03, 2)
    for seed in (0, 1):
        model = gp.GNN(learned.init_params(seed))
        part, st, rep, _ = gp.partition_learned(rp, ci, 32, model, 0.03, 2, fallback=True)
        assert rep["cut_plain"] == sp["cut"]
        assert st["cut"] <= sp["cut"]
        assert st["cut"] == gp.edge_cut(rp, ci, part, 32)[0]
        if rep["kept_learned"]:
            assert st["cut"] == rep["cut_learned"]
        else:
            assert torch.equal(part, plain)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(learned.__file__), "gnn_weights.npz")),
                    reason="no trained weights")
def test_trained_model_against_plain(gp, cuda):
    """What the trained scorer gains over plain heavy-edge matching on graphs
    it was not trained on (k=32): the result with the plain fallback is never worse, and the
    scorer's own inference costs at most a fifth of the plain V-cycle's device
    time (plus 10 ms of launch latency on these small graphs).  The whole
    learned V-cycle's time also depends on the hierarchy it builds; that ratio
    is measured on the full-size evaluation graphs by learned.evaluate."""
    model = gp.default_gnn()
    rows = []
    for name, g in (("rmat16", graphs.rmat(16, seed=777)[:2]), ("grid3d_48", graphs.grid3d(48, 48, 48)),
                    ("chunglu_50k", graphs.chung_lu(50000, 170000, seed=778))):
        rp, ci = g[0].to(cuda), g[1].to(cuda)
        r = learned.evaluate(model, rp, ci, 32, reps=2)
        _, st, rep, _ = gp.partition_learned(rp, ci, 32, model, fallback=True)
        assert st["cut"] <= r["cut_plain"]
        assert r["ms_gnn"] <= 0.2 * r["ms_plain"] + 10.0, r
        rows.append((name, r["cut_plain"], r["cut_learned"], round(r["cut_ratio"], 4), round(r["time_ratio"], 3)))
    print("\nlearned vs plain (k=32):", rows)


def test_learned_api_rejects_invalid(gp, cuda):
    """Invalid arguments return GP_EINVAL with a message; the context stays usable."""
    import ctypes as C
    from thegraphpartitioning_b200._abi import GP_EINVAL
    L = gp.lib()
    model = gp.GNN(learned.init_params(0))
    with pytest.raises(gp.GPError) as e:
        model.set_params(np.zeros(10, dtype=np.float32))
    assert e.value.code == GP_EINVAL
    with pytest.raises(gp.GPError):
        model.prio_bits = 17
    with pytest.raises(gp.GPError):
        model.max_level = -2
    assert model.prio_bits == 16 and model.max_level == -1
    rp, ci = graphs.grid2d(20, 20)
    rp, ci = rp.to(cuda), ci.to(cuda)
    part = torch.empty(rp.numel() - 1, dtype=torch.int32, device=cuda)
    rc = L.gp_partition_learned_device(rp.numel() - 1, C.c_void_p(rp.data_ptr()), C.c_void_p(ci.data_ptr()), None,
                                       None, 4, 0.03, 0, C.c_void_p(part.data_ptr()), None, None, None, None, 1, None,
                                       None, None)
    assert rc == GP_EINVAL and b"model" in L.gp_last_error()
    with pytest.raises(gp.GPError):
        gp.partition_learned(rp, ci, 0, model)
    # still usable
    p, st, rep, _ = gp.partition_learned(rp, ci, 4, model, fallback=True)
    assert st["cut"] == gp.edge_cut(rp, ci, p, 4)[0]


def test_move_head_matches_reference(gp, cuda):
    """Move-order head: the device features, scores, priorities and gradient
    against the float64 reference (same BF16-rounded parameters), and Adam
    steps on the device lower the loss."""
    from oracle import gnn_ref
    rng = np.random.default_rng(11)
    n = 6000
    rp = np.concatenate([[0], np.cumsum(rng.integers(0, 300, n))]).astype(np.int64)
    dest = rng.integers(-1, 8, n).astype(np.int32)
    gain = rng.integers(-3000, 3000, n).astype(np.int32)
    vw = rng.integers(1, 60, n).astype(np.int32)
    feat = gp.GNN.move_features(_dev(rp, cuda), _dev(dest, cuda), _dev(gain, cuda), _dev(vw, cuda), level=3)
    fref = gnn_ref.move_features(gain, np.diff(rp), vw, 3)
    fref[dest < 0] = 0.0
    f = feat.cpu().numpy().astype(np.float64)
    assert np.all(np.abs(f - fref) <= 1e-6 + 1e-6 * np.abs(fref))
    p = (gnn_ref.move_init_params(4) + rng.normal(0, 0.3, gnn_ref.MNPARAM)).astype(np.float32)
    model = gp.GNN(learned.init_params(0))
    model.set_move_params(p)
    assert np.array_equal(model.get_move_params(), p)
    score, prio = model.move_scores(feat)
    sref, _ = gnn_ref.move_forward(gnn_ref.bf16_round(p), f)
    sc = score.cpu().numpy().astype(np.float64)
    assert np.all(np.abs(sc - sref) <= ATOL + RTOL * np.abs(sref))
    assert np.all(np.abs(prio.cpu().numpy().astype(np.int64) - gnn_ref.move_priorities(sref))
                  <= 1 + 4096 * (ATOL + RTOL * np.abs(sref)))
    label = (rng.random(n) < 1 / (1 + np.exp(-f[:, 0] * 8))).astype(np.uint8)
    loss, g = model.move_grad(feat, _dev(label, cuda))
    loss_ref, g_ref = gnn_ref.move_loss_and_grad(gnn_ref.bf16_round(p), f, label)
    assert abs(loss - loss_ref) <= 1e-5 + 1e-5 * abs(loss_ref)
    assert np.linalg.norm(g - g_ref) <= 2e-3 * np.linalg.norm(g_ref)
    for _ in range(60):
        model.move_train_step(feat, _dev(label, cuda), lr=1e-2)
    assert model.move_grad(feat, _dev(label, cuda))[0] < loss
    model.set_move_params(None)
    assert model.get_move_params() is None


def test_learned_vcycle_with_move_head_matches_oracle(oracle_mod, gp, cuda):
    """With a move-order head the afterburner orders candidates by the head's
    priorities; the oracle, given the GPU's matching and move priorities,
    reproduces every event of the learned run."""
    from oracle import gnn_ref
    rng = np.random.default_rng(5)
    for g, k, seed in ((graphs.rmat(13, seed=23)[:2], 16, 3), (graphs.grid2d(70, 60), 6, 4)):
        rp, ci = to_np(*g)
        model = gp.GNN(_params(3), prio_bits=10)
        model.set_move_params(gnn_ref.move_init_params(5) + rng.normal(0, 0.3, gnn_ref.MNPARAM).astype(np.float32))
        part, st, rep, ev = gp.partition_learned(_dev(rp, cuda), _dev(ci, cuda), k, model, 0.03, seed,
                                                 fallback=False, trace=True)
        prio = {e["level"]: e["a0"] for e in ev if e["kind"] == GP_TR_PRIO}
        mprio = {(e["level"], e["iter"]): e["a0"] for e in ev if e["kind"] == GP_TR_MOVE_PRIO}
        assert prio and mprio and rep["kept_learned"] == 1
        ev_gpu = [e for e in ev if e["kind"] not in (GP_TR_PRIO, GP_TR_MOVE_PRIO)]
        p_ref, s_ref, ev_ref = oracle_mod.partition(rp, ci, k, 0.03, seed, trace=True, prio_levels=prio,
                                                    move_prio=mprio)
        compare_traces(ev_ref, ev_gpu)
        assert np.array_equal(p_ref, part.cpu().numpy())
        assert s_ref["cut"] == st["cut"]
