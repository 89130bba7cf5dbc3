"""Generate the full-size fixture of the benchmark workload:
tests/golden/rmat24_ef16_k64_full.json.

The benchmark partitions an R-MAT graph of scale 24 (edge factor 16,
a,b,c,d = 0.57,0.19,0.19,0.05, deduplicated, symmetrized, isolated vertices
dropped: 8,870,017 vertices, 260,377,570 undirected edges) into k = 64 parts
at 3 % imbalance, seed 0.  That size is far beyond what a test can run through
the oracle, so this script runs it once on the CPU and records:

  graph   SHA-256 of rowptr (int64) and colidx (int32), little-endian bytes,
          so a consumer can check that its graph is this one;
  oracle  the oracle's partition: SHA-256 of the part array (int32), cut,
          heaviest part, levels, coarsest size, refinement iterations and
          its single-core wall time;
  metis   METIS 5 PartGraphKway (CUDA toolkit's libmetis_static.a, default
          options: ufactor 30 = 3 %, seed 0) on the same graph: cut, heaviest
          part, imbalance and single-core wall time (the quality and speed
          baseline that replaces the reference's gpmetis call,
          src/gpu_part.cu:857).

bench.py compares its timed partition against the oracle record and reports
the METIS record beside its own cut and time.  The oracle takes about 13
minutes on one core; METIS keeps every level of its hierarchy in 64-bit
arrays and needs more than 60 GB of host memory on this graph, so the two
records can be made in separate runs on different hosts (each run keeps the
records already in the output file):

    python tests/golden/make_full_fixtures.py [--skip-oracle] [--skip-metis]
"""
import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

OUT = os.path.join(HERE, "rmat24_ef16_k64_full.json")


def sha256_of(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).view(np.uint8).data)
    return h.hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--k", type=int, default=64)
    ap.add_argument("--imbalance", type=float, default=0.03)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--skip-oracle", action="store_true")
    ap.add_argument("--skip-metis", action="store_true")
    ap.add_argument("--out", default=OUT)
    args = ap.parse_args()
    import oracle
    from thegraphpartitioning_b200 import graphs
    oracle.build()
    rec = {}
    if os.path.exists(args.out):
        with open(args.out) as f:
            rec = json.load(f)
    t = time.perf_counter()
    rp, ci, n_all = graphs.rmat(args.scale, 16, seed=args.seed, device="cpu")
    rp = rp.numpy().astype(np.int64)
    ci = ci.numpy().astype(np.int32)
    n, m = len(rp) - 1, len(ci) // 2
    print(f"graph: n={n} m={m} ({time.perf_counter() - t:.1f} s)", flush=True)
    rec["workload"] = f"rmat{args.scale}_ef16_k{args.k}"
    rec["graph"] = {"scale": args.scale, "edge_factor": 16, "seed": args.seed, "n": n, "n_before_isolated": n_all,
                    "m_undirected": m, "sha256_rowptr_colidx": sha256_of(rp, ci)}
    rec["args"] = {"k": args.k, "imbalance": args.imbalance, "seed": args.seed}
    W = n

    def save():
        with open(args.out, "w") as f:
            json.dump(rec, f, indent=1)
            f.write("\n")

    save()
    if not args.skip_oracle:
        t = time.perf_counter()
        part, st, _ = oracle.partition(rp, ci, args.k, args.imbalance, args.seed)
        dt = time.perf_counter() - t
        rec["oracle"] = {"sha256_part": sha256_of(part.astype(np.int32)), "cut": st["cut"],
                         "max_part_weight": st["max_part_weight"], "max_allowed": st["max_allowed"],
                         "levels": st["levels"], "coarsest_n": st["coarsest_n"],
                         "refine_iters": st["refine_iters"], "seconds": round(dt, 1), "cores": 1}
        print("oracle:", rec["oracle"], flush=True)
        save()
        del part
    if not args.skip_metis:
        mpart, mcut, t_metis = oracle.metis(rp, ci, args.k, seed=args.seed)
        pw = np.bincount(mpart, minlength=args.k)
        rec["metis"] = {"cut": mcut, "max_part_weight": int(pw.max()),
                        "imbalance": round(float(pw.max()) * args.k / W - 1, 5), "seconds": round(t_metis, 1),
                        "cores": 1, "library": "METIS 5 (CUDA toolkit libmetis_static.a), METIS_PartGraphKway, "
                                               "64-bit idx_t, default options (ufactor 30), seed 0"}
        print("metis:", rec["metis"], flush=True)
        save()


if __name__ == "__main__":
    main()
