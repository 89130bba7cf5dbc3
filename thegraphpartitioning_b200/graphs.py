"""Seeded synthetic graph generators (CSR, symmetric, no self-loops).

The reference's inputs are made by preprocess/conversion.py:60-74 (remove
self-loops, make bidirected, drop isolated vertices, CSR).  These generators
produce graphs with the same contract.  Randomness comes from a counter-based
splitmix64 hash evaluated with torch int64 ops, so a given seed yields the
same graph on the CPU and on a GPU (integer ops are exact on both); floating
point values that shape a distribution are computed on the CPU only.

Every generator returns (rowptr int64[n+1], colidx int32[E]) torch tensors on
`device`, rows sorted by neighbour id.
"""
from __future__ import annotations

import math

import torch

_M1 = 0xBF58476D1CE4E5B9 - (1 << 64)
_M2 = 0x94D049BB133111EB - (1 << 64)
_GOLD = 0x9E3779B97F4A7C15 - (1 << 64)


def _u64(x: int) -> int:
    """Python int -> the int64 with the same 64 bits."""
    x &= (1 << 64) - 1
    return x - (1 << 64) if x >= (1 << 63) else x


def mix64(x: torch.Tensor) -> torch.Tensor:
    """splitmix64 finalizer on int64 tensors (wrapping arithmetic)."""
    x = x ^ ((x >> 30) & ((1 << 34) - 1))
    x = x * _M1
    x = x ^ ((x >> 27) & ((1 << 37) - 1))
    x = x * _M2
    x = x ^ ((x >> 31) & ((1 << 33) - 1))
    return x


def _mix64_int(x: int) -> int:
    m = (1 << 64) - 1
    x &= m
    x ^= x >> 30
    x = (x * 0xBF58476D1CE4E5B9) & m
    x ^= x >> 27
    x = (x * 0x94D049BB133111EB) & m
    x ^= x >> 31
    return x


def stream_salt(seed: int, stream: int) -> int:
    """Independent int64 salt per (seed, stream)."""
    return _u64(_mix64_int((seed & ((1 << 64) - 1)) ^ _mix64_int(0x9E3779B97F4A7C15 * (stream + 1))))


def hash_bits(salt: int, idx: torch.Tensor) -> torch.Tensor:
    """64 random bits (as int64) per counter value."""
    return mix64(idx ^ salt)


def top_bits(h: torch.Tensor, nbits: int) -> torch.Tensor:
    """The top nbits bits of a 64-bit hash as a non-negative int64."""
    return (h >> (64 - nbits)) & ((1 << nbits) - 1)


# ------------------------------------------------------------------ CSR build
def csr_from_edges(src: torch.Tensor, dst: torch.Tensor, n: int, drop_isolated: bool = False,
                   relabel_salt: int | None = None):
    """Symmetrize, drop self-loops and duplicates, optionally drop isolated
    vertices (relabelling the rest by a hashed permutation when
    relabel_salt is given, else in id order).  Returns (rowptr, colidx, n)."""
    dev = src.device
    src = src.to(torch.int64)
    dst = dst.to(torch.int64)
    keep = src != dst
    src, dst = src[keep], dst[keep]
    key = torch.cat([src * n + dst, dst * n + src])
    del src, dst
    key = torch.unique(key)  # sorted
    u = torch.div(key, n, rounding_mode="floor")
    v = key - u * n
    del key
    if drop_isolated or relabel_salt is not None:
        deg = torch.bincount(u, minlength=n)
        alive = deg > 0 if drop_isolated else torch.ones(n, dtype=torch.bool, device=dev)
        ids = torch.nonzero(alive).flatten()
        if relabel_salt is not None:
            h = hash_bits(relabel_salt, ids)
            order = torch.argsort(h, stable=True)
            ids = ids[order]
        newid = torch.full((n,), -1, dtype=torch.int64, device=dev)
        newid[ids] = torch.arange(ids.numel(), device=dev)
        n = int(ids.numel())
        u = newid[u]
        v = newid[v]
        key = torch.sort(u * n + v).values
        u = torch.div(key, n, rounding_mode="floor")
        v = key - u * n
        del key
    counts = torch.bincount(u, minlength=n)
    rowptr = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    rowptr[1:] = torch.cumsum(counts, 0)
    return rowptr, v.to(torch.int32), n


# ------------------------------------------------------------------ families
def grid2d(rows: int, cols: int, device="cpu"):
    """5-point grid; vertex (r, c) has id r*cols + c."""
    n = rows * cols
    idx = torch.arange(n, device=device, dtype=torch.int64)
    r, c = idx // cols, idx % cols
    parts_s, parts_d = [], []
    for dr, dc in ((-1, 0), (0, -1), (0, 1), (1, 0)):  # ascending neighbour ids
        rr, cc = r + dr, c + dc
        ok = (rr >= 0) & (rr < rows) & (cc >= 0) & (cc < cols)
        parts_s.append(idx[ok])
        parts_d.append((rr * cols + cc)[ok])
    s = torch.cat(parts_s)
    d = torch.cat(parts_d)
    order = torch.argsort(s * n + d)
    s, d = s[order], d[order]
    counts = torch.bincount(s, minlength=n)
    rowptr = torch.zeros(n + 1, dtype=torch.int64, device=device)
    rowptr[1:] = torch.cumsum(counts, 0)
    return rowptr, d.to(torch.int32)


def grid3d(x: int, y: int, z: int, device="cpu"):
    """7-point grid; vertex (i, j, l) has id (i*y + j)*z + l."""
    n = x * y * z
    idx = torch.arange(n, device=device, dtype=torch.int64)
    i, rem = idx // (y * z), idx % (y * z)
    j, l = rem // z, rem % z
    parts_s, parts_d = [], []
    for di, dj, dl in ((-1, 0, 0), (0, -1, 0), (0, 0, -1), (0, 0, 1), (0, 1, 0), (1, 0, 0)):
        ii, jj, ll = i + di, j + dj, l + dl
        ok = (ii >= 0) & (ii < x) & (jj >= 0) & (jj < y) & (ll >= 0) & (ll < z)
        parts_s.append(idx[ok])
        parts_d.append(((ii * y + jj) * z + ll)[ok])
    s = torch.cat(parts_s)
    d = torch.cat(parts_d)
    del parts_s, parts_d
    # rows come out grouped by direction; a stable sort by source keeps the
    # direction order, which is ascending neighbour id
    order = torch.argsort(s, stable=True)
    d = d[order]
    counts = torch.bincount(s, minlength=n)
    rowptr = torch.zeros(n + 1, dtype=torch.int64, device=device)
    rowptr[1:] = torch.cumsum(counts, 0)
    return rowptr, d.to(torch.int32)


def path(n: int, device="cpu"):
    s = torch.arange(n - 1, device=device)
    return csr_from_edges(s, s + 1, n)[:2]


def cliques(count: int, size: int, device="cpu"):
    """`count` disjoint cliques of `size` vertices (ids grouped by clique)."""
    base = torch.arange(count, device=device).repeat_interleave(size * size) * size
    a = torch.arange(size, device=device).repeat_interleave(size).repeat(count)
    b = torch.arange(size, device=device).repeat(size * count)
    return csr_from_edges(base + a, base + b, count * size)[:2]


def rmat(scale: int, edge_factor: int = 16, a=0.57, b=0.19, c=0.19, seed: int = 0,
         device="cpu", chunk: int = 1 << 26):
    """R-MAT (Chakrabarti, Zhan, Faloutsos 2004) without noise.  Each of the
    edge_factor * 2**scale samples descends `scale` quadrant choices made from
    24-bit hash thresholds; the result is symmetrized, deduplicated, stripped
    of self-loops and isolated vertices, and relabelled by a hashed
    permutation.  Returns (rowptr, colidx, n_before_isolated_removal)."""
    n = 1 << scale
    m = edge_factor * n
    t_a = int(round(a * (1 << 24)))
    t_ab = int(round((a + b) * (1 << 24)))
    t_abc = int(round((a + b + c) * (1 << 24)))
    salt = stream_salt(seed, 1)
    srcs, dsts = [], []
    for start in range(0, m, chunk):
        cnt = min(chunk, m - start)
        e = torch.arange(start, start + cnt, device=device, dtype=torch.int64) * scale
        s = torch.zeros(cnt, dtype=torch.int64, device=device)
        d = torch.zeros(cnt, dtype=torch.int64, device=device)
        for lvl in range(scale):
            u = top_bits(hash_bits(salt, e + lvl), 24)
            sb = (u >= t_ab).to(torch.int64)
            db = ((u >= t_a) & (u < t_ab)) | (u >= t_abc)
            s = (s << 1) | sb
            d = (d << 1) | db.to(torch.int64)
            del u, sb, db
        srcs.append(s)
        dsts.append(d)
        del e
    src = torch.cat(srcs)
    dst = torch.cat(dsts)
    del srcs, dsts
    rowptr, colidx, n_alive = csr_from_edges(src, dst, n, drop_isolated=True,
                                             relabel_salt=stream_salt(seed, 2))
    return rowptr, colidx, n


def chung_lu(n: int = 262111, target_edges: int = 900_000, exponent: float = 2.5,
             max_degree: float = 420.0, seed: int = 0, device="cpu"):
    """Chung-Lu graph with expected degrees w_i = max_degree*((i+i0)/i0)^(-1/(exponent-1)),
    i0 chosen so that sum(w) = 2*target_edges.  Endpoints of target_edges samples
    are drawn proportionally to w by integer inverse-CDF on fixed-point weights
    (exact on every device); then symmetrized, deduplicated, self-loops and
    isolated vertices removed (in id order, as conversion.py:66-69 does).
    Returns (rowptr, colidx)."""
    beta = 1.0 / (exponent - 1.0)
    # solve sum_i max_degree*((i+i0)/i0)^-beta = 2*target_edges for i0 (bisection, on CPU)
    i = torch.arange(n, dtype=torch.float64)

    def total(i0):
        return float((max_degree * ((i + i0) / i0) ** (-beta)).sum())

    lo, hi = 1e-3, float(n)
    for _ in range(200):
        mid = math.sqrt(lo * hi)
        if total(mid) < 2 * target_edges:
            lo = mid
        else:
            hi = mid
    i0 = 0.5 * (lo + hi)
    w = max_degree * ((i + i0) / i0) ** (-beta)
    wfix = torch.round(w * 4096.0).to(torch.int64)
    cum = torch.cumsum(wfix, 0).to(device)
    tot = int(cum[-1])
    salt = stream_salt(seed, 3)
    e = torch.arange(2 * target_edges, device=device, dtype=torch.int64)
    r = top_bits(hash_bits(salt, e), 62) % tot
    ends = torch.searchsorted(cum, r, right=True)
    src, dst = ends[0::2], ends[1::2]
    rowptr, colidx, _ = csr_from_edges(src, dst, n, drop_isolated=True)
    return rowptr, colidx


def erdos_renyi(n: int, mean_degree: float, seed: int = 0, device="cpu"):
    """G(n, M) with M = n*mean_degree/2 uniform hashed edge samples."""
    m = int(round(n * mean_degree / 2))
    salt = stream_salt(seed, 4)
    e = torch.arange(2 * m, device=device, dtype=torch.int64)
    ends = top_bits(hash_bits(salt, e), 62) % n
    rowptr, colidx, _ = csr_from_edges(ends[0::2], ends[1::2], n)
    return rowptr, colidx


def random_geometric(n: int, mean_degree: float = 8.0, seed: int = 0, device="cpu"):
    """Points in the unit square on a 2^20 integer lattice (hashed); edge when
    squared lattice distance <= r^2 with r = sqrt(mean_degree/(pi*n)).
    Neighbour search over a cell grid of side >= r."""
    salt = stream_salt(seed, 5)
    idx = torch.arange(n, device=device, dtype=torch.int64)
    S = 1 << 20
    px = top_bits(hash_bits(salt, 2 * idx), 20)
    py = top_bits(hash_bits(salt, 2 * idx + 1), 20)
    r = math.sqrt(mean_degree / (math.pi * n))
    r_lat = int(r * S)
    r2 = r_lat * r_lat
    ncell = max(1, S // max(r_lat, 1))
    cs = (S + ncell - 1) // ncell
    cx, cy = px // cs, py // cs
    cell = cx * ncell + cy
    order = torch.argsort(cell * n + idx)
    cell_sorted = cell[order]
    starts = torch.searchsorted(cell_sorted, torch.arange(ncell * ncell + 1, device=device))
    srcs, dsts = [], []
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            ncx, ncy = cx + dx, cy + dy
            ok = (ncx >= 0) & (ncx < ncell) & (ncy >= 0) & (ncy < ncell)
            q = idx[ok]
            nc = (ncx * ncell + ncy)[ok]
            beg, end = starts[nc], starts[nc + 1]
            cnt = end - beg
            tot = int(cnt.sum())
            if tot == 0:
                continue
            rep_q = q.repeat_interleave(cnt)
            offs = torch.arange(tot, device=device) - torch.repeat_interleave(torch.cumsum(cnt, 0) - cnt, cnt)
            cand = order[beg.repeat_interleave(cnt) + offs]
            ddx = px[rep_q] - px[cand]
            ddy = py[rep_q] - py[cand]
            close = (ddx * ddx + ddy * ddy <= r2) & (rep_q < cand)
            srcs.append(rep_q[close])
            dsts.append(cand[close])
    src = torch.cat(srcs) if srcs else torch.zeros(0, dtype=torch.int64, device=device)
    dst = torch.cat(dsts) if dsts else torch.zeros(0, dtype=torch.int64, device=device)
    rowptr, colidx, _ = csr_from_edges(src, dst, n)
    return rowptr, colidx


def undirected_edges(rowptr) -> int:
    return int(rowptr[-1]) // 2


def batch_specs(count: int = 4096, seed: int = 0, nmin: int = 1000, nmax: int = 200_000,
                ks=(2, 4, 8, 16, 32)):
    """Specs of the batched workload: graph i has n log-uniform in [nmin, nmax],
    is a random geometric graph (mean degree 8) when i is even and an
    Erdos-Renyi graph (mean degree 10) when odd, k drawn from ks, and its own
    seed; all from hashes of (seed, i).  Returns a list of dicts."""
    specs = []
    for i in range(count):
        h = _mix64_int(stream_salt(seed, 1000 + i) & ((1 << 64) - 1))
        u = (h >> 11) / float(1 << 53)
        n = int(round(math.exp(math.log(nmin) + u * (math.log(nmax) - math.log(nmin)))))
        k = ks[(h >> 3) % len(ks)]
        specs.append({"i": i, "n": n, "k": k, "kind": "rgg" if i % 2 == 0 else "er",
                      "seed": _mix64_int(h ^ 0x5851F42D4C957F2D)})
    return specs


def batch_graph(spec, device="cpu"):
    """(rowptr, colidx) of one batch spec."""
    if spec["kind"] == "rgg":
        return random_geometric(spec["n"], 8.0, seed=spec["seed"], device=device)
    return erdos_renyi(spec["n"], 10.0, seed=spec["seed"], device=device)
