"""Generate tests/golden/*.npz: seeded small workloads with the oracle's
partition and statistics.

The reference (iamrupamroyy/TheGraphPartitioning) ships no tests, fixtures or
recorded outputs, and its GPU program is non-deterministic and depends on an
external gpmetis binary, so it cannot produce golden outputs.  These files
freeze the oracle's results on fixed inputs instead: tests/test_golden.py
checks that the oracle still reproduces them (any change of the rules shows
up as a diff here) and that the GPU library matches them bit for bit.

Each file holds the CSR (rowptr int64, colidx int32, optional weights), the
arguments (k, imbalance, seed) and the expected part array, cut, heaviest
part, levels and coarsest size.  Known answers that do not depend on the
oracle are checked separately in tests/test_oracle.py.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))


def cases():
    from thegraphpartitioning_b200 import graphs
    from helpers import to_np, weighted, star_plus_grid
    yield "grid32_k4", to_np(*graphs.grid2d(32, 32)), 4, 0.03, 0, False
    yield "grid20x30_k5_w", to_np(*graphs.grid2d(20, 30)), 5, 0.05, 3, True
    yield "rmat11_k8", to_np(*graphs.rmat(11, seed=1)[:2]), 8, 0.03, 7, False
    yield "chunglu3000_k16", to_np(*graphs.chung_lu(3000, 10000, seed=4)), 16, 0.03, 1, False
    yield "grid3d12_k32", to_np(*graphs.grid3d(12, 12, 12)), 32, 0.03, 2, False
    yield "star_grid_k3", to_np(*star_plus_grid(leaves=2500, side=20)), 3, 0.03, 5, False
    yield "rgg2500_k2_tight", to_np(*graphs.random_geometric(2500, 8.0, seed=6)), 2, 0.0, 9, False
    yield "er2000_k64", to_np(*graphs.erdos_renyi(2000, 6.0, seed=2)), 64, 0.03, 4, False


def main():
    import oracle
    from helpers import weighted
    oracle.build()
    for name, (rp, ci), k, imb, seed, w in cases():
        ew = vw = None
        if w:
            ew, vw = weighted(rp, ci, seed=13)
        part, st, _ = oracle.partition(rp, ci, k, imb, seed, vwgt=vw, ewgt=ew)
        extra = {} if not w else {"ewgt": ew, "vwgt": vw}
        np.savez_compressed(os.path.join(HERE, name + ".npz"), rowptr=rp.astype(np.int64), colidx=ci.astype(np.int32),
                            k=np.int32(k), imbalance=np.float32(imb), seed=np.uint64(seed), part=part.astype(np.int32),
                            cut=np.int64(st["cut"]), max_part_weight=np.int64(st["max_part_weight"]),
                            levels=np.int32(st["levels"]), coarsest_n=np.int32(st["coarsest_n"]), **extra)
        print(name, "n", len(rp) - 1, "m", len(ci) // 2, "k", k, "cut", st["cut"])


if __name__ == "__main__":
    main()
