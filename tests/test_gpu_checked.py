"""The bounds-checked build (libgp_b200_checked.so: the same sources compiled
with -DGP_CHECKED) run over graphs that reach every kernel family -- warp,
lane-group and CTA-item rows, every contraction tier, the one-block and the
multi-kernel refinement loops, the radix-sorted rebalancing, the batched
stages -- must count no out-of-range index and return the oracle's
partitions.  It runs in a child process, which loads the checked library in
place of the regular one."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import sys
import numpy as np
import torch
sys.path.insert(0, ROOT); sys.path.insert(0, ROOT + "/tests")
import oracle
import thegraphpartitioning_b200 as gp
from thegraphpartitioning_b200 import graphs
from helpers import multi_star_grid, star_plus_grid, to_np, weighted
assert gp.CHECKED and gp.LIB_PATH.endswith("libgp_b200_checked.so")
assert "bounds-checked" in gp.version()
dev = torch.device("cuda:0")
gp.checked_violations(clear=True)
cases = [
    (to_np(*graphs.rmat(14, seed=1)[:2]), 64, {}),
    (to_np(*graphs.chung_lu(30000, 100000, seed=2)), 8, {}),
    (to_np(*star_plus_grid(leaves=40000, side=64)), 4, {}),
    (to_np(*star_plus_grid(leaves=150000, side=32)), 3, {}),
    (to_np(*multi_star_grid()), 8, {}),
    (to_np(*graphs.grid3d(20, 20, 20)), 32, {"small_level_n": 16384}),
    (to_np(*graphs.random_geometric(50000, 8.0, seed=9)), 2, {}),
    (to_np(*graphs.rmat(12, seed=3)[:2]), 16, {"heavy_deg": 64, "item_len": 96}),
]
for (rp, ci), k, opts in cases:
    imb = 0.0 if k == 2 else 0.03
    ref, rst, _ = oracle.partition(rp, ci, k, imb, 5, options=opts)
    got, st, _ = gp.partition(torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev), k, imb, 5, options=opts)
    assert np.array_equal(ref, got.cpu().numpy()) and st["cut"] == rst["cut"], (len(rp), k)
rp, ci = to_np(*graphs.grid2d(60, 70))
ew, vw = weighted(rp, ci, seed=4)
d = lambda a: torch.from_numpy(a).to(dev)
ref, _, _ = oracle.partition(rp, ci, 7, 0.05, 2, vwgt=vw, ewgt=ew)
got, _, _ = gp.partition(d(rp), d(ci), 7, 0.05, 2, vwgt=d(vw), ewgt=d(ew))
assert np.array_equal(ref, got.cpu().numpy())
specs = graphs.batch_specs(12, seed=4, nmin=500, nmax=40000)
gs = [graphs.batch_graph(s, device=dev) for s in specs]
parts, _ = gp.partition_batch(gs, [s["k"] for s in specs], 0.03, [s["seed"] for s in specs], workers=4)
for s, (grp, gci), p in zip(specs, gs, parts):
    ref, _, _ = oracle.partition(grp.cpu().numpy(), gci.cpu().numpy(), s["k"], 0.03, s["seed"])
    assert np.array_equal(ref, p.cpu().numpy())
cnt, site = gp.checked_violations(clear=True)
print("violations", cnt, "first site", site)
assert cnt == 0, (cnt, site)
'''


def test_bounds_checked_build_counts_no_violation(gp, cuda, oracle_mod):
    lib = os.path.join(ROOT, "thegraphpartitioning_b200", "libgp_b200_checked.so")
    assert os.path.exists(lib), "build the checked library (make -C thegraphpartitioning_b200/csrc)"
    env = dict(os.environ, THEGRAPHPARTITIONING_CHECKED="1")
    out = subprocess.run([sys.executable, "-c", CHILD.replace("ROOT", repr(ROOT))], env=env, capture_output=True,
                         text=True, timeout=900)
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    assert "violations 0" in out.stdout


def test_regular_build_reports_it_is_not_checked(gp, cuda):
    import ctypes as C
    if gp.CHECKED:
        pytest.skip("this process runs the checked build")
    cnt, site = C.c_int64(0), C.c_int32(0)
    assert gp.lib().gp_checked_violations(C.byref(cnt), C.byref(site), 0) == -1
    assert "not the bounds-checked build" in gp.lib().gp_last_error().decode()
