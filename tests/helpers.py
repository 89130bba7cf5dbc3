"""Shared helpers of the test suite (graph builders and trace comparison)."""
import numpy as np
import torch

from thegraphpartitioning_b200 import graphs


def to_np(rp, ci):
    return rp.cpu().numpy().astype(np.int64), ci.cpu().numpy().astype(np.int32)


def check_csr(rp, ci, n=None, symmetric=True):
    rp = np.asarray(rp); ci = np.asarray(ci)
    n = len(rp) - 1 if n is None else n
    assert rp[0] == 0 and np.all(np.diff(rp) >= 0) and rp[-1] == len(ci)
    src = np.repeat(np.arange(n), np.diff(rp))
    assert np.all((ci >= 0) & (ci < n))
    assert not np.any(src == ci), "self-loop"
    if symmetric:
        a = np.sort(src.astype(np.int64) * n + ci)
        b = np.sort(ci.astype(np.int64) * n + src)
        assert np.array_equal(a, b), "not symmetric"


def star_plus_grid(leaves=3000, side=24):
    """A hub with `leaves` leaves (degree above the CTA-per-row threshold)
    attached to a grid, so that heavy-row code paths run."""
    rp, ci = graphs.grid2d(side, side)
    g = side * side
    src = [np.repeat(np.arange(g), np.diff(rp.numpy())), ]
    dst = [ci.numpy().astype(np.int64)]
    hub = g
    leaf = np.arange(g + 1, g + 1 + leaves)
    src += [np.full(leaves, hub), leaf, np.array([hub]), np.array([0])]
    dst += [leaf, np.full(leaves, hub), np.array([0]), np.array([hub])]
    # chain a few leaves so they are not all identical
    src += [leaf[:-1:7], leaf[1::7]]
    dst += [leaf[1::7], leaf[:-1:7]]
    s = torch.from_numpy(np.concatenate(src))
    d = torch.from_numpy(np.concatenate(dst))
    rp2, ci2, _ = graphs.csr_from_edges(s, d, g + 1 + leaves)
    return rp2, ci2


def multi_star_grid(hub_leaves=(700, 3000, 9000, 30000, 90000), side=32, shared=0.2, seed=0):
    """Hubs of the given leaf counts on a grid, so that the first coarse level
    has rows in every contraction tier (walks of about 700, 3,000, 9,000,
    30,000 and 90,000 entries); each hub also links to a `shared` fraction of
    the previous hub's leaves, so that coarse walks hold repeated neighbours."""
    rng = np.random.default_rng(seed)
    rp, ci = graphs.grid2d(side, side)
    g = side * side
    src = [np.repeat(np.arange(g), np.diff(rp.numpy()))]
    dst = [ci.numpy().astype(np.int64)]
    nxt = g
    prev = None
    for i, nl in enumerate(hub_leaves):
        hub = nxt
        leaf = np.arange(hub + 1, hub + 1 + nl)
        nxt = hub + 1 + nl
        att = np.array([i % g])
        src += [np.full(nl, hub), leaf, np.array([hub]), att]
        dst += [leaf, np.full(nl, hub), att, np.array([hub])]
        src += [leaf[:-1:5], leaf[1::5]]          # chains among the leaves
        dst += [leaf[1::5], leaf[:-1:5]]
        if prev is not None:
            extra = rng.choice(prev, size=int(shared * len(prev)), replace=False)
            src += [np.full(len(extra), hub), extra]
            dst += [extra, np.full(len(extra), hub)]
        prev = leaf
    s = torch.from_numpy(np.concatenate(src).astype(np.int64))
    d = torch.from_numpy(np.concatenate(dst).astype(np.int64))
    rp2, ci2, _ = graphs.csr_from_edges(s, d, nxt)
    return rp2, ci2


def weighted(rp, ci, seed=0, wmax=9):
    """Symmetric random integer edge weights in [1, wmax] and vertex weights in [1, 4]."""
    rp = np.asarray(rp); ci = np.asarray(ci)
    n = len(rp) - 1
    src = np.repeat(np.arange(n), np.diff(rp)).astype(np.int64)
    lo = np.minimum(src, ci); hi = np.maximum(src, ci)
    h = graphs.mix64(torch.from_numpy(lo * n + hi) ^ graphs.stream_salt(seed, 11)).numpy()
    ew = (np.abs(h) % wmax + 1).astype(np.int32)
    hv = graphs.mix64(torch.arange(n) ^ graphs.stream_salt(seed, 12)).numpy()
    vw = (np.abs(hv) % 4 + 1).astype(np.int32)
    return ew, vw


def compare_traces(ev_ref, ev_gpu):
    """Bit-exact comparison of two trace event lists (oracle vs GPU)."""
    assert len(ev_ref) == len(ev_gpu), (len(ev_ref), len(ev_gpu),
                                        [(e["kind"], e["level"], e["iter"]) for e in ev_ref[-5:]],
                                        [(e["kind"], e["level"], e["iter"]) for e in ev_gpu[-5:]])
    for i, (a, b) in enumerate(zip(ev_ref, ev_gpu)):
        where = f"event {i} kind={a['kind']} level={a['level']} iter={a['iter']}"
        for key in ("kind", "level", "iter", "mode", "n", "m", "cut", "maxpw", "count"):
            assert a[key] == b[key], f"{where}: {key} oracle={a[key]} gpu={b[key]}"
        for key in ("a0", "a1", "a2", "rowptr", "colidx", "ewgt", "vwgt"):
            if key in a or key in b:
                x, y = a.get(key), b.get(key)
                assert x is not None and y is not None, f"{where}: {key} missing"
                if not np.array_equal(x, y):
                    bad = np.nonzero(x != y)[0] if x.shape == y.shape else None
                    raise AssertionError(f"{where}: {key} differs (shape {x.shape} vs {y.shape}); "
                                         f"first mismatches {bad[:10] if bad is not None else ''}")
