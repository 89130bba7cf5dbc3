"""CPU checks of the CLI's input reader (no device work: --parse-only): the
multi-threaded parser returns exactly the integers of row.txt / column.txt /
weight.txt in both command lines, and reports short or malformed files with
exit code 2, as the reference's readFile does (src/gpu_part.cu:786-800)."""
import os
import subprocess

import numpy as np
import pytest

import thegraphpartitioning_b200 as gp

FNV_OFFSET, FNV_PRIME, MASK = 1469598103934665603, 1099511628211, (1 << 64) - 1


def fnv(*arrays):
    h = FNV_OFFSET
    for a in arrays:
        for x in a.tolist():
            h = ((h ^ (x & MASK)) * FNV_PRIME) & MASK
    return f"{h:016x}"


def _graph(n, m, seed):
    rng = np.random.default_rng(seed)
    deg = rng.multinomial(m, np.ones(n) / n)
    rp = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    ci = rng.integers(0, n, size=m).astype(np.int64)
    ew = rng.integers(1, 1000, size=m).astype(np.int64)
    return rp, ci, ew


def _write(d, rp, ci, ew=None, sep="\n"):
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "row.txt"), "w") as f:
        f.write(sep.join(map(str, rp.tolist())) + "\n")
    with open(os.path.join(d, "column.txt"), "w") as f:
        f.write(" ".join(map(str, ci.tolist())) + "\n")
    if ew is not None:
        with open(os.path.join(d, "weight.txt"), "w") as f:
            f.write("\n".join(map(str, ew.tolist())) + "\n")


def _run(args, cwd):
    return subprocess.run([gp.CLI_PATH] + args + ["--parse-only"], capture_output=True, text=True, cwd=cwd)


@pytest.mark.parametrize("n,m", [(50, 300), (60000, 400000)])
def test_parse_both_forms(tmp_path, n, m):
    rp, ci, ew = _graph(n, m, seed=n)
    d = str(tmp_path / "g")
    _write(d, rp, ci, ew)
    r = _run([d, str(n), str(m), "4"], str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert f"n={n} m={m} weights=1 checksum={fnv(rp, ci, ew)}" in r.stdout
    os.remove(os.path.join(d, "weight.txt"))
    r = _run([os.path.join(d, "row.txt"), os.path.join(d, "column.txt"), "4"], str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert f"n={n} m={m} weights=0 checksum={fnv(rp, ci)}" in r.stdout


def test_parse_errors(tmp_path):
    rp, ci, ew = _graph(100, 500, seed=1)
    d = str(tmp_path / "short")
    _write(d, rp, ci[:-5], ew)
    r = _run([d, "100", "500", "4"], str(tmp_path))
    assert r.returncode == 2 and "column.txt" in r.stderr
    d = str(tmp_path / "bad")
    _write(d, rp, ci, ew)
    with open(os.path.join(d, "column.txt"), "w") as f:
        f.write(" ".join(map(str, ci[:10].tolist())) + " x7 " + " ".join(map(str, ci[11:].tolist())))
    r = _run([d, "100", "500", "4"], str(tmp_path))
    assert r.returncode == 2 and "not an integer at element 10" in r.stderr


def test_preprocess_output_feeds_the_cli(tmp_path):
    """Ranks 3-4 of the pipeline together: an edge list turned into row.txt /
    column.txt / weight.txt by the preprocessing restatement is read back by
    the CLI exactly, in both command lines (the reference's users run
    conversion.py and then gpu_part on its output)."""
    from thegraphpartitioning_b200 import preprocess
    rng = np.random.default_rng(5)
    src = rng.integers(0, 3000, size=20000)
    dst = rng.integers(0, 3000, size=20000)
    edges = str(tmp_path / "g.tsv")
    with open(edges, "w") as f:
        for a, b in zip(src.tolist(), dst.tolist()):
            f.write(f"{a}\t{b}\t1\n")
    out = str(tmp_path / "csr")
    assert preprocess.main([edges, out]) == 0
    rp, ci = preprocess.to_csr(src, dst)
    rp = rp.astype(np.int64); ci = ci.astype(np.int64)
    n, m = len(rp) - 1, len(ci)
    r = _run([out, str(n), str(m), "8"], str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert f"n={n} m={m} weights=1 checksum={fnv(rp, ci, np.ones(m, dtype=np.int64))}" in r.stdout
    r = _run([os.path.join(out, "row.txt"), os.path.join(out, "column.txt"), "8"], str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert f"n={n} m={m} weights=1" in r.stdout   # weight.txt beside row.txt is picked up
