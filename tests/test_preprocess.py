"""CPU checks of the preprocessing restatement (thegraphpartitioning_b200.preprocess,
after the reference's preprocess/conversion.py:30-110): self-loops dropped,
edges made bidirectional and de-duplicated, isolated vertices removed with the
rest renumbered in id order, and the five output files in their formats."""
import os

import numpy as np
import pytest

from thegraphpartitioning_b200 import preprocess


def _expected(edges, n):
    adj = {v: set() for v in range(n)}
    for a, b in edges:
        if a != b:
            adj[a].add(b)
            adj[b].add(a)
    alive = [v for v in range(n) if adj[v]]
    new = {v: i for i, v in enumerate(alive)}
    rows = [sorted(new[u] for u in adj[v]) for v in alive]
    rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int64)
    ci = np.array([u for r in rows for u in r], dtype=np.int32)
    return rp, ci


EDGES = [(0, 1), (1, 0), (1, 2), (2, 2), (4, 5), (5, 7), (7, 4), (4, 5), (9, 9), (3, 1)]


def test_to_csr_matches_definition():
    src = np.array([a for a, _ in EDGES]); dst = np.array([b for _, b in EDGES])
    rp, ci = preprocess.to_csr(src, dst)
    erp, eci = _expected(EDGES, 10)
    assert np.array_equal(rp, erp) and np.array_equal(ci, eci)


@pytest.mark.parametrize("ext", [".tsv", ".txt", ".tsv_1", ".mtx"])
def test_files(tmp_path, ext):
    path = str(tmp_path / ("g" + ext))
    if ext == ".mtx":
        import scipy.sparse as sp
        from scipy.io import mmwrite
        # entry (row, col) is the edge col -> row
        rows = [b for _, b in EDGES]; cols = [a for a, _ in EDGES]
        mmwrite(path, sp.coo_matrix((np.ones(len(EDGES)), (rows, cols)), shape=(10, 10)))
    else:
        head = {".tsv": 0, ".txt": 4, ".tsv_1": 1}[ext]
        with open(path, "w") as f:
            for i in range(head):
                f.write(f"# header {i}\n")
            for a, b in EDGES:
                f.write(f"{a}\t{b}" + ("\t1" if ext == ".tsv" else "") + "\n")
    out = str(tmp_path / "out")
    assert preprocess.main([path, out]) == 0
    erp, eci = _expected(EDGES, 10)
    rp = np.loadtxt(os.path.join(out, "row.txt"), dtype=np.int64)
    ci = np.loadtxt(os.path.join(out, "column.txt"), dtype=np.int64)
    w = np.loadtxt(os.path.join(out, "weight.txt"), dtype=np.int64)
    assert np.array_equal(rp, erp) and np.array_equal(ci, eci) and np.all(w == 1) and len(w) == len(ci)
    n, m = len(erp) - 1, len(eci)
    lines = open(os.path.join(out, "temp.graph")).read().splitlines()
    assert lines[0] == f"{n} {m // 2} 1"
    for v in range(n):
        toks = [int(t) for t in lines[1 + v].split()]
        assert toks[0::2] == [int(u) + 1 for u in eci[erp[v]:erp[v + 1]]] and all(t == 1 for t in toks[1::2])
    csr = open(os.path.join(out, "output_output.csr")).read().split("\n")
    assert csr[0] == f"{n} {m} {n + 1} {m}"
    assert [int(t) for t in csr[1].split()] == erp.tolist()
    assert [int(t) for t in csr[2].split()] == eci.tolist()
