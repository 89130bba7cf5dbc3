"""Training and evaluation of the learned matching priorities.

The reference has no code for this part (its run log names a
GNNcoarsening.cu, script/run.txt:5-6, that is not in the repository).

Data: the plain partitioner labels its own hierarchy.  For every level at
which it matched, the level graph (the input, or a coarse graph from the
CONTRACT trace) is one sample; an entry (v, u) is labelled 1 when v and u sit
in the same part after that level's refinement (the LEVEL_DONE trace).  The
network learns which edges stay inside parts; matching then contracts those
first instead of the heaviest ones.

Training runs entirely in the library's own kernels (gp_gnn_train_step_device:
forward, backward and Adam on the GPU).  The families follow the workloads of
the plain method: Chung-Lu power-law graphs, R-MAT, random geometric graphs
and Erdos-Renyi graphs, n log-uniform in [2k, 64k].

After training, the priority resolution (GNN.prio_bits) is chosen on a
validation set of larger graphs from the same families (other seeds): the
value with the lowest geometric-mean cut relative to the plain method.

Move-order head: the label-propagation candidates of the plain partitioner
(every LP step of every level, from the REFINE_ITER trace: proposed part and
integer gain) are labelled 1 when the candidate ends its level in the part it
proposed (LEVEL_DONE), i.e. the moves the plain method finally accepts.  The
head is trained on these rows with its own device kernels and kept only when
it lowers the geometric-mean cut on the validation set.

    python -m thegraphpartitioning_b200.learned train --graphs 2000 --out gnn_weights.npz
    python -m thegraphpartitioning_b200.learned train-move --init gnn_weights.npz --out gnn_weights.npz
    python -m thegraphpartitioning_b200.learned eval --weights gnn_weights.npz --seeds 0,1,2
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import GNN, partition, partition_learned, graphs as G
from ._abi import GP_TR_MATCH, GP_TR_CONTRACT, GP_TR_LEVEL_DONE, GP_TR_REFINE_ITER

H, F0, MSG, ZD = 64, 4, 8, 4
O_W1 = 0
O_B1 = O_W1 + H * 2 * F0
O_P = O_B1 + H
O_W2 = O_P + MSG * H
O_B2 = O_W2 + H * (H + MSG)
O_Z = O_B2 + H
O_A = O_Z + ZD * H
O_BETA = O_A + ZD
O_ETA = O_BETA + 3          # common-neighbour coefficient
NPARAM = O_BETA + 4
FAMILIES = ("chung_lu", "rmat", "rgg", "er")
# move-order head: W1[MH, MF] b1[MH] w2[MH] b2
MH, MF = 16, 4
MO_W1 = 0
MO_B1 = MO_W1 + MH * MF
MO_W2 = MO_B1 + MH
MO_B2 = MO_W2 + MH
MNPARAM = MO_B2 + 1


def init_params(seed: int = 0) -> np.ndarray:
    """He-scaled random weights, zero biases; the edge-weight coefficient
    starts at 1 so that an untrained model behaves like heavy-edge matching
    with noise."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, dtype=np.float32)
    p[O_W1:O_B1] = rng.normal(0, math.sqrt(2.0 / (2 * F0)), H * 2 * F0)
    p[O_P:O_W2] = rng.normal(0, math.sqrt(1.0 / H), MSG * H)
    p[O_W2:O_B2] = rng.normal(0, math.sqrt(2.0 / (H + MSG)), H * (H + MSG))
    p[O_Z:O_A] = rng.normal(0, math.sqrt(1.0 / H), ZD * H)
    p[O_A:O_BETA] = rng.normal(0, 0.1, ZD)
    p[O_BETA] = 1.0
    return p


def graph_spec(i: int, seed: int = 0, nmin: int = 2000, nmax: int = 64000):
    """Family, size, k and seed of training graph i (hash-derived)."""
    h = G._mix64_int(G.stream_salt(seed, 7000 + i) & ((1 << 64) - 1))
    u = (h >> 11) / float(1 << 53)
    n = int(round(math.exp(math.log(nmin) + u * (math.log(nmax) - math.log(nmin)))))
    fam = FAMILIES[i % len(FAMILIES)]
    k = (2, 4, 8, 16, 32, 64)[(h >> 5) % 6]
    return {"i": i, "family": fam, "n": n, "k": k, "seed": G._mix64_int(h ^ 0x2545F4914F6CDD1D)}


def make_graph(spec, device="cuda"):
    fam, n, sd = spec["family"], spec["n"], spec["seed"]
    if fam == "chung_lu":
        rp, ci = G.chung_lu(n, target_edges=int(3.43 * n), exponent=2.5, max_degree=max(20.0, 420.0 * n / 262111),
                            seed=sd, device=device)
    elif fam == "rmat":
        scale = max(10, int(round(math.log2(n))))
        rp, ci, _ = G.rmat(scale, 16, seed=sd, device=device)
    elif fam == "rgg":
        rp, ci = G.random_geometric(n, 8.0, seed=sd, device=device)
    else:
        rp, ci = G.erdos_renyi(n, 10.0, seed=sd, device=device)
    return rp, ci


def level_samples(rowptr, colidx, k: int, seed: int = 0, imbalance: float = 0.03):
    """[(rowptr, colidx, vwgt, ewgt, level, label)] CUDA tensors for every level
    the plain V-cycle matched at."""
    import torch
    dev = rowptr.device
    _, _, ev = partition(rowptr, colidx, k, imbalance=imbalance, seed=seed,
                         trace={GP_TR_MATCH, GP_TR_CONTRACT, GP_TR_LEVEL_DONE})
    graphs = {0: (rowptr, colidx, None, None)}
    parts, matched = {}, set()
    for e in ev:
        if e["kind"] == GP_TR_CONTRACT:
            t = lambda a, dt: torch.from_numpy(a).to(dev, dt)
            graphs[e["level"] + 1] = (t(e["rowptr"], torch.int64), t(e["colidx"], torch.int32),
                                      t(e["vwgt"], torch.int32), t(e["ewgt"], torch.int32))
        elif e["kind"] == GP_TR_LEVEL_DONE:
            parts[e["level"]] = e["a0"]
        elif e["kind"] == GP_TR_MATCH:
            matched.add(e["level"])
    out = []
    for lvl in sorted(matched):
        if lvl not in graphs or lvl not in parts:
            continue
        rp, ci, vw, ew = graphs[lvl]
        p = torch.from_numpy(parts[lvl]).to(dev)
        src = torch.repeat_interleave(torch.arange(rp.numel() - 1, device=dev), rp[1:] - rp[:-1])
        label = (p[src] == p[ci.long()]).to(torch.uint8)
        out.append((rp, ci, vw, ew, lvl, label))
    return out


def move_samples(rowptr, colidx, k: int, seed: int = 0, imbalance: float = 0.03):
    """(features float32[r, 4], labels uint8[r]) CUDA tensors: every
    label-propagation candidate of the plain V-cycle, labelled 1 when it ends
    its level in the part it proposed."""
    import torch
    dev = rowptr.device
    _, _, ev = partition(rowptr, colidx, k, imbalance=imbalance, seed=seed,
                         trace={GP_TR_CONTRACT, GP_TR_REFINE_ITER, GP_TR_LEVEL_DONE})
    graphs = {0: (rowptr, None)}
    steps, final = {}, {}
    for e in ev:
        if e["kind"] == GP_TR_CONTRACT:
            graphs[e["level"] + 1] = (torch.from_numpy(e["rowptr"]).to(dev), torch.from_numpy(e["vwgt"]).to(dev))
        elif e["kind"] == GP_TR_REFINE_ITER and e["mode"] == 0:
            steps.setdefault(e["level"], []).append((e["a0"], e["a1"]))
        elif e["kind"] == GP_TR_LEVEL_DONE:
            final[e["level"]] = e["a0"]
    feats, labels = [], []
    for lvl, lst in steps.items():
        rp, vw = graphs[lvl]
        fin = final[lvl]
        for dest, gain in lst:
            cand = np.nonzero(dest >= 0)[0]
            if len(cand) == 0:
                continue
            f = GNN.move_features(rp, torch.from_numpy(dest).to(dev), torch.from_numpy(gain).to(dev), vw, lvl)
            idx = torch.from_numpy(cand).to(dev)
            feats.append(f[idx])
            labels.append(torch.from_numpy((fin[cand] == dest[cand]).astype(np.uint8)).to(dev))
    if not feats:
        return torch.zeros((0, 4), device=dev), torch.zeros(0, dtype=torch.uint8, device=dev)
    return torch.cat(feats), torch.cat(labels)


def build_move_dataset(count: int, seed: int = 0, device="cuda", log=None):
    import torch
    feats, labels, t0 = [], [], time.time()
    for i in range(count):
        spec = graph_spec(i, seed)
        rp, ci = make_graph(spec, device)
        k = min(spec["k"], max(2, (rp.numel() - 1) // 64))
        f, y = move_samples(rp, ci, k, seed=spec["seed"])
        feats.append(f)
        labels.append(y)
        if log and (i + 1) % 100 == 0:
            log(f"graphs {i + 1}/{count}: {sum(x.shape[0] for x in feats)} candidates, {time.time() - t0:.1f}s")
    return torch.cat(feats), torch.cat(labels)


def train_move_head(model: GNN, feat, label, steps: int = 600, lr: float = 1e-2, log=None):
    """Full-batch Adam on the candidate rows, cosine-decayed step size; returns
    the loss before the first and after the last step."""
    first = model.move_grad(feat, label)[0]
    for t in range(steps):
        cur = lr * 0.5 * (1 + math.cos(math.pi * t / max(steps, 1)))
        loss = model.move_train_step(feat, label, lr=max(cur, lr * 0.02))
        if log and t % 100 == 0:
            log(f"move head step {t}: loss {loss:.4f}")
    return first, model.move_grad(feat, label)[0]


def move_init_params(seed: int = 0) -> np.ndarray:
    """Head that starts as the plain (gain) order: hidden unit 0 copies the
    signed log gain, the output is a positive multiple of it."""
    rng = np.random.default_rng(seed)
    p = np.zeros(MNPARAM, dtype=np.float32)
    p[MO_W1:MO_B1] = rng.normal(0, math.sqrt(2.0 / MF), MH * MF) * 0.1
    p[MO_W1 + 0] = 1.0
    p[MO_B1 + 0] = 0.5
    p[MO_W2 + 0] = 4.0
    return p


def build_dataset(count: int, seed: int = 0, device="cuda", log=None):
    samples, t0 = [], time.time()
    for i in range(count):
        spec = graph_spec(i, seed)
        rp, ci = make_graph(spec, device)
        n = rp.numel() - 1
        k = min(spec["k"], max(2, n // 64))
        samples.extend(level_samples(rp, ci, k, seed=spec["seed"]))
        if log and (i + 1) % 200 == 0:
            log(f"graphs {i + 1}/{count}: {len(samples)} level samples, {time.time() - t0:.1f}s")
    return samples


def train(model: GNN, samples, epochs: int = 4, batch: int = 32, lr: float = 3e-3, seed: int = 0, log=None):
    """Adam over shuffled mini-batches; cosine-decayed step size.  Returns the
    mean loss of each epoch."""
    rng = np.random.default_rng(seed)
    steps = epochs * ((len(samples) + batch - 1) // batch)
    step, hist = 0, []
    for ep in range(epochs):
        order = rng.permutation(len(samples))
        tot, cnt = 0.0, 0
        for b in range(0, len(order), batch):
            cur = lr * 0.5 * (1 + math.cos(math.pi * step / max(steps, 1)))
            loss = model.train_step([samples[j] for j in order[b:b + batch]], lr=max(cur, lr * 0.02))
            tot += loss
            cnt += 1
            step += 1
        hist.append(tot / max(cnt, 1))
        if log:
            log(f"epoch {ep}: mean loss {hist[-1]:.4f}")
    return hist


def validation_set(count_per_family: int = 2, seed: int = 1, n: int = 200_000, device="cuda"):
    """Larger graphs of the training families (other seeds) for choosing prio_bits."""
    out = []
    for j in range(count_per_family * len(FAMILIES)):
        spec = graph_spec(j, seed, nmin=n, nmax=n)
        spec["family"] = FAMILIES[j % len(FAMILIES)]
        out.append(make_graph(spec, device))
    return out


def tune_prio_bits(model: GNN, graphs, k: int = 32, candidates=(4, 6, 8, 10, 12, 16), levels=(0, 1, -1), log=None):
    """Set model.prio_bits and model.max_level to the candidate pair with the
    lowest geometric-mean learned/plain cut ratio over `graphs`; returns
    {(bits, max_level): ratio}."""
    plain = [partition(rp, ci, k)[1]["cut"] for rp, ci in graphs]
    res = {}
    for lv in levels:
        for b in candidates:
            model.prio_bits = b
            model.max_level = lv
            logs = [math.log(max(partition_learned(rp, ci, k, model, fallback=False)[1]["cut"], 1) / max(c, 1))
                    for (rp, ci), c in zip(graphs, plain)]
            res[(b, lv)] = math.exp(sum(logs) / len(logs))
            if log:
                log(f"prio_bits {b}, max_level {lv}: geometric-mean cut ratio {res[(b, lv)]:.4f}")
    b, lv = min(res, key=lambda t: (res[t], -t[0]))
    model.prio_bits, model.max_level = b, lv
    return res


def evaluate(model: GNN, rowptr, colidx, k: int, seed: int = 0, imbalance: float = 0.03, reps: int = 1):
    """Plain vs learned V-cycle on one graph: cuts, balance and device times
    (one untimed warm-up of each, then the fastest of `reps` runs)."""
    import torch
    partition(rowptr, colidx, k, imbalance=imbalance, seed=seed)
    partition_learned(rowptr, colidx, k, model, imbalance=imbalance, seed=seed, fallback=False)
    best = None
    for _ in range(reps):
        torch.cuda.synchronize()
        _, sp, _ = partition(rowptr, colidx, k, imbalance=imbalance, seed=seed)
        _, sl, rep, _ = partition_learned(rowptr, colidx, k, model, imbalance=imbalance, seed=seed, fallback=False)
        r = {"cut_plain": sp["cut"], "cut_learned": sl["cut"], "imb_plain": sp["imbalance"],
             "imb_learned": sl["imbalance"], "ms_plain": sp["ms_total"], "ms_learned": sl["ms_total"],
             "ms_gnn": rep["ms_gnn"], "balanced_learned": sl["max_part_weight"] <= sl["max_allowed"]}
        for key in ("ms_coarsen", "ms_initial", "ms_refine", "levels", "refine_iters"):
            r[key + "_plain"], r[key + "_learned"] = sp[key], sl[key]
        if best is None or r["ms_learned"] < best["ms_learned"]:
            best = r
    best["cut_ratio"] = best["cut_learned"] / max(best["cut_plain"], 1)
    best["time_ratio"] = best["ms_learned"] / max(best["ms_plain"], 1e-9)
    return best


def held_out(name: str, device="cuda"):
    """The evaluation graphs: R-MAT scale 22 and the 3D 7-point grid 256^3."""
    if name == "rmat22":
        rp, ci, _ = G.rmat(22, 16, seed=12345, device=device)
        return rp, ci
    if name == "grid3d256":
        return G.grid3d(256, 256, 256, device=device)
    raise KeyError(name)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--graphs", type=int, default=2000)
    t.add_argument("--epochs", type=int, default=4)
    t.add_argument("--batch", type=int, default=32)
    t.add_argument("--lr", type=float, default=3e-3)
    t.add_argument("--seed", type=int, default=0)
    t.add_argument("--out", default="gnn_weights.npz")
    t.add_argument("--init", default=None, help="start from these weights instead of a seeded init")
    t.add_argument("--tune-only", action="store_true", help="with --init: only re-tune prio_bits / max_level")
    tm = sub.add_parser("train-move")
    tm.add_argument("--init", required=True, help="model (edge scorer) to add the head to")
    tm.add_argument("--graphs", type=int, default=400)
    tm.add_argument("--steps", type=int, default=600)
    tm.add_argument("--lr", type=float, default=1e-2)
    tm.add_argument("--seed", type=int, default=0)
    tm.add_argument("--out", default="gnn_weights.npz")
    e = sub.add_parser("eval")
    e.add_argument("--weights", default=None)
    e.add_argument("--seeds", default="0", help="partition seeds; the table reports each and their spread")
    e.add_argument("--graphs", default="rmat22,grid3d256")
    e.add_argument("--k", type=int, default=32)
    e.add_argument("--reps", type=int, default=2)
    e.add_argument("--json", default=None)
    a = ap.parse_args(argv)
    log = lambda s: print(s, flush=True)
    import torch
    if a.cmd == "train":
        model = GNN.load(a.init) if a.init else GNN(init_params(a.seed))
        if not (a.tune_only and a.init):
            t0 = time.time()
            samples = build_dataset(a.graphs, a.seed, log=log)
            log(f"dataset: {len(samples)} samples, {sum(int(s[1].numel()) for s in samples)} entries, "
                f"{time.time() - t0:.1f}s")
            t1 = time.time()
            hist = train(model, samples, a.epochs, a.batch, a.lr, a.seed, log=log)
            log(f"training: {time.time() - t1:.1f}s, loss {hist[0]:.4f} -> {hist[-1]:.4f}")
            del samples
            torch.cuda.empty_cache()
        tune_prio_bits(model, validation_set(), log=log)
        log(f"prio_bits = {model.prio_bits}, max_level = {model.max_level}")
        model.save(a.out)
        log(f"saved {a.out}")
    elif a.cmd == "train-move":
        model = GNN.load(a.init)
        t0 = time.time()
        feat, label = build_move_dataset(a.graphs, a.seed, log=log)
        log(f"move dataset: {feat.shape[0]} candidates ({float(label.float().mean()):.3f} accepted), "
            f"{time.time() - t0:.1f}s")
        model.set_move_params(move_init_params(a.seed))
        l0, l1 = train_move_head(model, feat, label, a.steps, a.lr, log=log)
        log(f"move head loss {l0:.4f} -> {l1:.4f}")
        del feat, label
        torch.cuda.empty_cache()
        # keep the head only when it lowers the validation cut
        val = validation_set()
        k = 32
        ratios = {}
        for use in (False, True):
            saved = model.get_move_params()
            if not use:
                model.set_move_params(None)
            logs = [math.log(max(partition_learned(rp, ci, k, model, fallback=False)[1]["cut"], 1) /
                             max(partition(rp, ci, k)[1]["cut"], 1)) for rp, ci in val]
            ratios[use] = math.exp(sum(logs) / len(logs))
            if not use:
                model.set_move_params(saved)
        log(f"validation geometric-mean cut ratio vs plain: without head {ratios[False]:.4f}, "
            f"with head {ratios[True]:.4f}")
        if ratios[True] >= ratios[False]:
            model.set_move_params(None)
            log("head not kept")
        model.save(a.out)
        log(f"saved {a.out}")
    else:
        from . import default_gnn
        model = GNN.load(a.weights) if a.weights else default_gnn()
        res = {}
        seeds = [int(x) for x in a.seeds.split(",")]
        for name in a.graphs.split(","):
            rp, ci = held_out(name)
            rows = []
            for sd in seeds:
                r = evaluate(model, rp, ci, a.k, seed=sd, reps=a.reps)
                r.update({"graph": name, "seed": sd, "n": rp.numel() - 1, "undirected_edges": ci.numel() // 2,
                          "k": a.k, "move_head": model.get_move_params() is not None})
                log(json.dumps(r))
                rows.append(r)
            cr = [r["cut_ratio"] for r in rows]
            pl = [r["cut_plain"] for r in rows]
            res[name] = {"runs": rows, "cut_ratio_geomean": math.exp(sum(math.log(x) for x in cr) / len(cr)),
                         "cut_ratio_min": min(cr), "cut_ratio_max": max(cr),
                         "plain_seed_spread": max(pl) / max(min(pl), 1),
                         "time_ratio_max": max(r["time_ratio"] for r in rows)}
            log(json.dumps({k2: v for k2, v in res[name].items() if k2 != "runs"}))
            del rp, ci
            torch.cuda.empty_cache()
        if a.json:
            with open(a.json, "w") as f:
                json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
