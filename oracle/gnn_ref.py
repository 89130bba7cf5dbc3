"""Float64 restatement of the learned edge scorer (forward, loss, gradients).

TEST INFRASTRUCTURE ONLY: the checker for the network kernels in
thegraphpartitioning_b200/csrc/gp_gnn.cu.  The reference has no code for
this part (its run log names a GNNcoarsening.cu, script/run.txt:5-6, that
is not in the repository), so this file is the specification the CUDA
kernels are held to.

Parameter layout (floats, row-major), H = 64 hidden, F0 = 4 input features,
MSG = 8 message floats, ZD = 4 edge-embedding floats:

    W1[H, 2*F0]  b1[H]  P[MSG, H]  W2[H, H+MSG]  b2[H]  Z[ZD, H]  A[ZD]
    beta  gamma  delta  eta

Per graph (CSR, weights None = 1):

    x_v  = [log2(1+deg)/8, log2(1+wdeg)/16, log2(1+vw)/16, level/16]
    a_v  = mean_{u in N(v)} x_u
    h1_v = relu(W1 [x_v; a_v] + b1),   m_v = P h1_v
    c_v  = mean_{u in N(v)} m_u
    h2_v = relu(W2 [h1_v; c_v] + b2),  z_v = Z h2_v
    t_vu = sum_j A_j z_v[j] z_u[j] + beta log2(1+w)/8 + gamma (w/wdeg_v + w/wdeg_u) + delta
           + eta log2(1 + cn_vu)/7
    cn_vu = popcount(sig_v & sig_u) without the bits of v and u, where the
            128-bit signature sig_x has bit b(y) = fmix32(y * 0x9E3779B1) >> 25
            (MurmurHash3's 32-bit finalizer) set for every neighbour y of x
    prio = clamp(rint(t * 2^bits) + 2^30, 0, 2^31 - 128)      (bits = 16 by default)
    loss = mean over directed entries of BCE-with-logits(t, label)

The kernels run with the parameters rounded to bfloat16; `bf16_round`
reproduces that rounding (round to nearest even) so that both sides use the
same numbers.  The backward pass here is the plain chain rule over every
directed entry (no use of symmetry), so it also checks the kernels'
symmetric-gather shortcut.
"""
from __future__ import annotations

import numpy as np

H, F0, MSG, ZD = 64, 4, 8, 4
O_W1 = 0
O_B1 = O_W1 + H * 2 * F0
O_P = O_B1 + H
O_W2 = O_P + MSG * H
O_B2 = O_W2 + H * (H + MSG)
O_Z = O_B2 + H
O_A = O_Z + ZD * H
O_BETA = O_A + ZD
O_GAMMA = O_BETA + 1
O_DELTA = O_GAMMA + 1
O_ETA = O_DELTA + 1
NPARAM = O_ETA + 1


def bf16_round(p: np.ndarray) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even) -> float64."""
    b = np.ascontiguousarray(p, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (b >> 16) & 1
    r = ((b + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return dict(
        W1=p[O_W1:O_B1].reshape(H, 2 * F0), b1=p[O_B1:O_P], P=p[O_P:O_W2].reshape(MSG, H),
        W2=p[O_W2:O_B2].reshape(H, H + MSG), b2=p[O_B2:O_Z], Z=p[O_Z:O_A].reshape(ZD, H),
        A=p[O_A:O_BETA], beta=p[O_BETA], gamma=p[O_GAMMA], delta=p[O_DELTA], eta=p[O_ETA])


def init_params(seed: int = 0) -> np.ndarray:
    """Seeded initial parameters: He-scaled weights, zero biases, the edge
    terms starting at heavy-edge behaviour (beta > 0)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, dtype=np.float32)
    p[O_W1:O_B1] = rng.normal(0, np.sqrt(2.0 / (2 * F0)), H * 2 * F0)
    p[O_P:O_W2] = rng.normal(0, np.sqrt(1.0 / H), MSG * H)
    p[O_W2:O_B2] = rng.normal(0, np.sqrt(2.0 / (H + MSG)), H * (H + MSG))
    p[O_Z:O_A] = rng.normal(0, np.sqrt(1.0 / H), ZD * H)
    p[O_A:O_BETA] = rng.normal(0, 0.1, ZD)
    p[O_BETA] = 1.0
    return p


def _fmix32(x):
    x = x & 0xFFFFFFFF
    x ^= x >> 16
    x = (x * 0x85EBCA6B) & 0xFFFFFFFF
    x ^= x >> 13
    x = (x * 0xC2B2AE35) & 0xFFFFFFFF
    x ^= x >> 16
    return x


def nb_bit(ids):
    """Signature bit (0..127) of each vertex id."""
    x = (np.asarray(ids, dtype=np.uint64) * np.uint64(0x9E3779B1)) & np.uint64(0xFFFFFFFF)
    return (_fmix32(x) >> np.uint64(25)).astype(np.int64)


def common_neighbours(rowptr, colidx):
    """Per directed entry (v, u): popcount of sig_v & sig_u without the bits of v and u."""
    rp, n, src = _rows(rowptr)
    col = np.asarray(colidx, dtype=np.int64)
    sig = np.zeros((n, 2), dtype=np.uint64)
    b = nb_bit(col)
    lo = b < 64
    one = np.uint64(1)
    np.bitwise_or.at(sig[:, 0], src[lo], one << b[lo].astype(np.uint64))
    np.bitwise_or.at(sig[:, 1], src[~lo], one << (b[~lo] - 64).astype(np.uint64))
    m = sig[src] & sig[col]
    for ends in (src, col):
        eb = nb_bit(ends)
        half = (eb >= 64).astype(np.int64)
        bit = one << (eb - 64 * half).astype(np.uint64)
        m[np.arange(len(m)), half] &= ~bit
    return np.bitwise_count(m).sum(1).astype(np.int64)


def _rows(rowptr):
    rp = np.asarray(rowptr, dtype=np.int64)
    n = len(rp) - 1
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp))
    return rp, n, src


def _mean(rp, src, col, val):
    n = len(rp) - 1
    deg = np.diff(rp).astype(np.float64)
    out = np.zeros((n, val.shape[1]))
    np.add.at(out, src, val[col])
    inv = np.where(deg > 0, 1.0 / np.maximum(deg, 1), 0.0)
    return out * inv[:, None], inv


def forward(params, rowptr, colidx, vwgt=None, ewgt=None, level=0, keep=False):
    """Logits per directed entry (and the activations when keep=True)."""
    q = unpack(params)
    rp, n, src = _rows(rowptr)
    col = np.asarray(colidx, dtype=np.int64)
    w = np.ones(len(col)) if ewgt is None else np.asarray(ewgt, dtype=np.float64)
    vw = np.ones(n) if vwgt is None else np.asarray(vwgt, dtype=np.float64)
    deg = np.diff(rp).astype(np.float64)
    wdeg = np.zeros(n)
    np.add.at(wdeg, src, w)
    x = np.stack([np.log2(1 + deg) / 8, np.log2(1 + wdeg) / 16, np.log2(1 + vw) / 16,
                  np.full(n, level / 16.0)], axis=1)
    a, inv = _mean(rp, src, col, x)
    xa = np.concatenate([x, a], axis=1)
    pre1 = xa @ q["W1"].T + q["b1"]
    h1 = np.maximum(pre1, 0)
    m = h1 @ q["P"].T
    c, _ = _mean(rp, src, col, m)
    hc = np.concatenate([h1, c], axis=1)
    pre2 = hc @ q["W2"].T + q["b2"]
    h2 = np.maximum(pre2, 0)
    z = h2 @ q["Z"].T
    ft = np.log2(1 + w) / 8
    fg = w / wdeg[src] + w / wdeg[col]
    fc = np.log2(1 + common_neighbours(rp, col)) / 7
    t = (q["A"][None, :] * z[src] * z[col]).sum(1) + q["beta"] * ft + q["gamma"] * fg + q["delta"] + q["eta"] * fc
    if not keep:
        return t
    return t, dict(src=src, col=col, inv=inv, xa=xa, pre1=pre1, h1=h1, hc=hc, pre2=pre2, h2=h2, z=z,
                   ft=ft, fg=fg, fc=fc, n=n)


def priorities(t, bits: int = 16):
    q = np.rint(np.asarray(t, dtype=np.float64) * float(1 << bits)) + 1073741824.0
    return np.clip(q, 0, 2147483520).astype(np.int32)


def loss_and_grad(params, rowptr, colidx, label, vwgt=None, ewgt=None, level=0):
    """Mean BCE over directed entries and its gradient (float64)."""
    q = unpack(params)
    t, S = forward(params, rowptr, colidx, vwgt, ewgt, level, keep=True)
    y = np.asarray(label, dtype=np.float64)
    E = max(len(t), 1)
    loss = (np.maximum(t, 0) - t * y + np.log1p(np.exp(-np.abs(t)))).sum() / E
    dt = (1 / (1 + np.exp(-t)) - y) / E
    src, col, z, n = S["src"], S["col"], S["z"], S["n"]
    g = np.zeros(NPARAM)
    g[O_A:O_BETA] = (dt[:, None] * z[src] * z[col]).sum(0)
    g[O_BETA] = (dt * S["ft"]).sum()
    g[O_GAMMA] = (dt * S["fg"]).sum()
    g[O_DELTA] = dt.sum()
    g[O_ETA] = (dt * S["fc"]).sum()
    dz = np.zeros((n, ZD))
    np.add.at(dz, src, dt[:, None] * q["A"][None, :] * z[col])
    np.add.at(dz, col, dt[:, None] * q["A"][None, :] * z[src])
    g[O_Z:O_A] = (dz.T @ S["h2"]).ravel()
    dpre2 = (dz @ q["Z"]) * (S["pre2"] > 0)
    g[O_W2:O_B2] = (dpre2.T @ S["hc"]).ravel()
    g[O_B2:O_Z] = dpre2.sum(0)
    dhc = dpre2 @ q["W2"]
    dh1 = dhc[:, :H].copy()
    dc = dhc[:, H:]
    # c_v = inv_v sum_{u in N(v)} m_u  ->  dm_u += inv_v dc_v for every entry (v, u)
    dm = np.zeros((n, MSG))
    np.add.at(dm, col, dc[src] * S["inv"][src][:, None])
    g[O_P:O_W2] = (dm.T @ S["h1"]).ravel()
    dh1 += dm @ q["P"]
    dpre1 = dh1 * (S["pre1"] > 0)
    g[O_W1:O_B1] = (dpre1.T @ S["xa"]).ravel()
    g[O_B1:O_P] = dpre1.sum(0)
    return float(loss), g


# ---------------------------------------------------------------- move-order head
# Parameters W1[MH, MF] b1[MH] w2[MH] b2; features of a label-propagation
# candidate with integer gain g, degree deg, vertex weight vw at `level`:
#   f = [sign(g) log2(1+|g|)/16, log2(1+deg)/8, log2(1+vw)/16, level/16]
#   s = w2 . relu(W1 f + b1) + b2,   move priority = clamp(rint(s * 2^12), -2^30, 2^30)
# trained by mean binary cross-entropy against "the candidate ends the level in
# its proposed part".
MH, MF = 16, 4
MO_W1 = 0
MO_B1 = MO_W1 + MH * MF
MO_W2 = MO_B1 + MH
MO_B2 = MO_W2 + MH
MNPARAM = MO_B2 + 1


def move_features(gain, deg, vw, level):
    g = np.asarray(gain, dtype=np.float64)
    mag = np.log2(1 + np.abs(g)) / 16
    return np.stack([np.where(g < 0, -mag, mag), np.log2(1 + np.asarray(deg, dtype=np.float64)) / 8,
                     np.log2(1 + np.asarray(vw, dtype=np.float64)) / 16,
                     np.full(len(g), level / 16.0)], axis=1)


def move_init_params(seed: int = 0) -> np.ndarray:
    """He-scaled first layer; the output starts as a positive multiple of the
    first hidden unit that copies the signed gain feature (the plain order)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(MNPARAM, dtype=np.float32)
    p[MO_W1:MO_B1] = rng.normal(0, np.sqrt(2.0 / MF), MH * MF) * 0.1
    p[MO_W1 + 0] = 1.0                   # unit 0 <- signed log gain
    p[MO_B1 + 0] = 0.5                   # kept positive over the gain range
    p[MO_W2 + 0] = 4.0
    return p


def move_forward(params, feat):
    p = np.asarray(params, dtype=np.float64)
    W1 = p[MO_W1:MO_B1].reshape(MH, MF)
    pre = feat @ W1.T + p[MO_B1:MO_W2]
    return np.maximum(pre, 0) @ p[MO_W2:MO_B2] + p[MO_B2], pre


def move_priorities(score):
    return np.clip(np.rint(np.asarray(score) * 4096.0), -(1 << 30), 1 << 30).astype(np.int32)


def move_loss_and_grad(params, feat, label):
    p = np.asarray(params, dtype=np.float64)
    s, pre = move_forward(p, feat)
    y = np.asarray(label, dtype=np.float64)
    N = max(len(s), 1)
    loss = (np.maximum(s, 0) - s * y + np.log1p(np.exp(-np.abs(s)))).sum() / N
    ds = (1 / (1 + np.exp(-s)) - y) / N
    h = np.maximum(pre, 0)
    g = np.zeros(MNPARAM)
    g[MO_B2] = ds.sum()
    g[MO_W2:MO_B2] = ds @ h
    dh = (ds[:, None] * p[MO_W2:MO_B2][None, :]) * (pre > 0)
    g[MO_B1:MO_W2] = dh.sum(0)
    g[MO_W1:MO_B1] = (dh.T @ feat).ravel()
    return float(loss), g
