"""The drop-in CLI in both command lines the reference has (src/gpu_part.cu:880-888
and README.md:130-138): finalpartition.txt in the reference's format, every
vertex listed once, the same partition as the library call, exit code 1 on bad
arguments."""
import os
import subprocess

import numpy as np
import pytest

from thegraphpartitioning_b200 import graphs
from helpers import to_np, weighted

pytestmark = pytest.mark.gpu


def _write(dirpath, rp, ci, ew=None):
    np.savetxt(os.path.join(dirpath, "row.txt"), rp, fmt="%d")
    np.savetxt(os.path.join(dirpath, "column.txt"), ci, fmt="%d")
    if ew is not None:
        np.savetxt(os.path.join(dirpath, "weight.txt"), ew, fmt="%d")


def _read_final(path, n, k):
    part = np.full(n, -1, dtype=np.int64)
    lines = open(path).read().strip().splitlines()
    assert len(lines) == k
    for q, line in enumerate(lines):
        head, _, rest = line.partition(":")
        assert head == f"Partition {q}"
        ids = [int(x) for x in rest.strip().split(",") if x.strip()]
        assert ids == sorted(ids)
        assert np.all(part[ids] == -1)
        part[ids] = q
    assert np.all(part >= 0)
    return part


def test_cli_both_forms_match_library(gp, cuda, tmp_path):
    rp, ci = to_np(*graphs.rmat(12, seed=3)[:2])
    ew, _ = weighted(rp, ci, seed=2)
    n, k = len(rp) - 1, 6
    d1 = tmp_path / "weighted"
    d1.mkdir()
    _write(str(d1), rp, ci, ew)
    out1 = tmp_path / "final1.txt"
    r = subprocess.run([gp.CLI_PATH, str(d1) + "/", str(n), str(len(ci)), str(k), "--out", str(out1)],
                       capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    ref, st, _ = gp.partition(rp, ci, k, 0.03, 0, ewgt=ew)
    assert np.array_equal(_read_final(str(out1), n, k), ref)
    assert str(st["cut"]) in r.stdout
    # README form, unit weights (no weight.txt beside column.txt)
    d2 = tmp_path / "unit"
    d2.mkdir()
    _write(str(d2), rp, ci)
    r = subprocess.run([gp.CLI_PATH, str(d2 / "row.txt"), str(d2 / "column.txt"), str(k)],
                       capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    ref2, _, _ = gp.partition(rp, ci, k, 0.03, 0)
    assert np.array_equal(_read_final(str(tmp_path / "finalpartition.txt"), n, k), ref2)


def test_cli_bad_arguments_exit_1(gp, tmp_path):
    r = subprocess.run([gp.CLI_PATH, "only-one-arg"], capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode == 1
