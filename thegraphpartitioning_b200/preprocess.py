"""Edge list / Matrix Market file -> the CSR text files the CLI reads.

Restates preprocess/conversion.py of the reference (lines 30-110) without dgl:

  * inputs by extension: ``.mtx`` / ``.mmio`` (Matrix Market; an entry
    (row, col) becomes the edge col -> row, as the reference builds its graph
    from (col, row)), ``.tsv`` (tab-separated source, destination, data),
    ``.txt`` (tab-separated source, destination after four header lines, the
    SNAP layout), ``.tsv_1`` (tab-separated, one header line);
  * the graph has max id + 1 vertices; self-loops are dropped, every edge is
    made bidirectional and duplicates removed, isolated vertices are removed
    and the rest renumbered in id order; rows list neighbours in ascending id;
  * outputs in the current (or given) directory: ``row.txt`` (n + 1 row
    pointers), ``column.txt`` (column ids), ``weight.txt`` (a 1 per entry),
    ``output_output.csr`` ("n m len(rowptr) len(colidx)" then the two arrays
    on one line each) and ``temp.graph`` (METIS format, 1-based, unit edge
    weights, m/2 edges in the header).

    python -m thegraphpartitioning_b200.preprocess graph.tsv [outdir]
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np
import torch

from .graphs import csr_from_edges


def load_edges(path: str):
    """(src, dst) int64 arrays of the edge file, by extension."""
    ext = os.path.splitext(path)[1]
    if ext in (".mtx", ".mmio"):
        from scipy.io import mmread
        try:
            mat = mmread(path, spmatrix=False)   # sparse array (newer scipy)
        except TypeError:
            mat = mmread(path)
        coo = mat.tocoo()
        return np.asarray(coo.col, dtype=np.int64), np.asarray(coo.row, dtype=np.int64)
    skip = {".tsv": 0, ".txt": 4, ".tsv_1": 1}
    if ext not in skip:
        raise ValueError(f"unsupported file type {ext!r}: supported .tsv, .txt, .tsv_1, .mtx, .mmio")
    import pandas as pd
    df = pd.read_csv(path, delimiter="\t", header=None, skiprows=skip[ext], usecols=[0, 1], low_memory=False)
    return df[0].to_numpy(dtype=np.int64), df[1].to_numpy(dtype=np.int64)


def to_csr(src, dst):
    """Symmetric CSR without self-loops, duplicates or isolated vertices
    (renumbered in id order).  Returns (rowptr int64, colidx int32)."""
    # own writable copies: readers (pandas, mmread) may hand out read-only arrays
    s = torch.from_numpy(np.array(src, dtype=np.int64))
    d = torch.from_numpy(np.array(dst, dtype=np.int64))
    n = int(max(int(s.max()), int(d.max())) + 1) if s.numel() else 0
    rowptr, colidx, _ = csr_from_edges(s, d, n, drop_isolated=True)
    return rowptr.numpy(), colidx.numpy()


def _write_lines(path, arr):
    with open(path, "w") as f:
        step = 1 << 22
        for i in range(0, len(arr), step):
            f.write("\n".join(map(str, arr[i:i + step].tolist())))
            f.write("\n")


def write_outputs(rowptr, colidx, outdir="."):
    os.makedirs(outdir, exist_ok=True)
    n, m = len(rowptr) - 1, len(colidx)
    _write_lines(os.path.join(outdir, "row.txt"), rowptr)
    _write_lines(os.path.join(outdir, "column.txt"), colidx)
    with open(os.path.join(outdir, "weight.txt"), "w") as f:
        f.write("1\n" * m)
    with open(os.path.join(outdir, "output_output.csr"), "w") as f:
        f.write(f"{n} {m} {len(rowptr)} {len(colidx)}\n")
        f.write(" ".join(map(str, rowptr.tolist())) + " \n")
        f.write(" ".join(map(str, colidx.tolist())) + " ")
    with open(os.path.join(outdir, "temp.graph"), "w") as f:
        f.write(f"{n} {m // 2} 1\n")
        for v in range(n):
            nb = colidx[rowptr[v]:rowptr[v + 1]] + 1
            f.write(" ".join(f"{u} 1" for u in nb.tolist()) + "\n")


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if not argv:
        print(__doc__)
        return 1
    t0 = time.time()
    src, dst = load_edges(argv[0])
    print(f"Graph loaded: {len(src)} entries, {time.time() - t0:.3f}s")
    t1 = time.time()
    rowptr, colidx = to_csr(src, dst)
    print(f"Nodes: {len(rowptr) - 1}, Edges: {len(colidx)}")
    print(f"CSR size: row_ptr={len(rowptr)}, col_idx={len(colidx)}; built in {time.time() - t1:.3f}s")
    write_outputs(rowptr, colidx, argv[1] if len(argv) > 1 else ".")
    return 0


if __name__ == "__main__":
    sys.exit(main())
