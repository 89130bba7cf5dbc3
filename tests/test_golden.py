"""Golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py).

CPU: the oracle still reproduces every fixture bit for bit (a change of the
deterministic rules shows up here first).  GPU: the library returns the
fixture's partition, cut, heaviest part, level count and coarsest size, through
the host entry point and the device entry point, twice in a row.
"""
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
IDS = [os.path.basename(f)[:-4] for f in FILES]


def _load(path):
    z = np.load(path)
    d = {key: z[key] for key in z.files}
    return d


def test_fixtures_present():
    assert len(FILES) >= 8


@pytest.mark.parametrize("path", FILES, ids=IDS)
def test_oracle_reproduces_golden(oracle_mod, path):
    d = _load(path)
    part, st, _ = oracle_mod.partition(d["rowptr"], d["colidx"], int(d["k"]), float(d["imbalance"]), int(d["seed"]),
                                       vwgt=d.get("vwgt"), ewgt=d.get("ewgt"))
    assert np.array_equal(part, d["part"])
    assert st["cut"] == int(d["cut"]) and st["max_part_weight"] == int(d["max_part_weight"])
    assert st["levels"] == int(d["levels"]) and st["coarsest_n"] == int(d["coarsest_n"])
    cut, pw = oracle_mod.edge_cut(d["rowptr"], d["colidx"], part, int(d["k"]), ewgt=d.get("ewgt"), vwgt=d.get("vwgt"))
    assert cut == int(d["cut"]) and pw.max() == int(d["max_part_weight"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=IDS)
def test_gpu_matches_golden(gp, cuda, path):
    import torch
    d = _load(path)
    args = (int(d["k"]), float(d["imbalance"]), int(d["seed"]))
    host, st, _ = gp.partition(d["rowptr"], d["colidx"], *args, vwgt=d.get("vwgt"), ewgt=d.get("ewgt"))
    assert np.array_equal(host, d["part"])
    t = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    for _ in range(2):
        dev, st2, _ = gp.partition(t(d["rowptr"]), t(d["colidx"]), *args, vwgt=t(d.get("vwgt")), ewgt=t(d.get("ewgt")))
        assert np.array_equal(dev.cpu().numpy(), d["part"])
        for s in (st, st2):
            assert s["cut"] == int(d["cut"]) and s["max_part_weight"] == int(d["max_part_weight"])
            assert s["levels"] == int(d["levels"]) and s["coarsest_n"] == int(d["coarsest_n"])
