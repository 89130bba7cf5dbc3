"""Generators: contract of conversion.py's output (symmetric, no self-loops,
no isolated vertices where promised) and device-independent hashing."""
import numpy as np
import torch

from thegraphpartitioning_b200 import graphs
from helpers import check_csr, to_np


def test_mix64_matches_oracle(oracle_mod):
    xs = torch.tensor([0, 1, 2, 3, 2 ** 40 + 17, -1, -(2 ** 63)], dtype=torch.int64)
    hs = graphs.mix64(xs).tolist()
    for x, h in zip(xs.tolist(), hs):
        assert (h & (2 ** 64 - 1)) == oracle_mod.mix64(x & (2 ** 64 - 1))


def test_grid_shapes():
    rp, ci = to_np(*graphs.grid2d(512, 512))
    assert len(rp) - 1 == 262144 and len(ci) // 2 == 523264
    check_csr(rp, ci)
    rp, ci = to_np(*graphs.grid3d(8, 9, 10))
    assert len(ci) // 2 == 3 * 8 * 9 * 10 - (9 * 10 + 8 * 10 + 8 * 9)
    check_csr(rp, ci)


def test_rmat_contract():
    rp, ci, n_all = graphs.rmat(12, seed=1)
    rp, ci = to_np(rp, ci)
    check_csr(rp, ci)
    assert n_all == 4096 and np.all(np.diff(rp) > 0)   # isolated vertices removed
    rp2, ci2, _ = graphs.rmat(12, seed=1)
    assert np.array_equal(rp, rp2.numpy()) and np.array_equal(ci, ci2.numpy())


def test_chung_lu_shape():
    rp, ci = to_np(*graphs.chung_lu())
    check_csr(rp, ci)
    n, m = len(rp) - 1, len(ci) // 2
    assert 240000 < n <= 262111 and 850000 < m < 950000
    deg = np.diff(rp)
    assert deg.min() >= 1 and 200 < deg.max() < 800


def test_er_rgg_contract():
    for rp, ci in (graphs.erdos_renyi(5000, 10.0, seed=2), graphs.random_geometric(5000, 8.0, seed=3)):
        rp, ci = to_np(rp, ci)
        check_csr(rp, ci)
        assert 6 < len(ci) / (len(rp) - 1) < 12
