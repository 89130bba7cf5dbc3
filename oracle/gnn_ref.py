"""Float64 restatement of the learned edge scorer (forward, loss, gradients).

TEST INFRASTRUCTURE ONLY: the checker for the network kernels in
thegraphpartitioning_b200/csrc/gp_gnn.cu.  The reference has no code for
this part (its run log names a GNNcoarsening.cu, script/run.txt:5-6, that
is not in the repository), so this file is the specification the CUDA
kernels are held to.

Parameter layout (floats, row-major), H = 64 hidden, F0 = 4 input features,
MSG = 8 message floats, ZD = 4 edge-embedding floats:

    W1[H, 2*F0]  b1[H]  P[MSG, H]  W2[H, H+MSG]  b2[H]  Z[ZD, H]  A[ZD]
    beta  gamma  delta

Per graph (CSR, weights None = 1):

    x_v  = [log2(1+deg)/8, log2(1+wdeg)/16, log2(1+vw)/16, level/16]
    a_v  = mean_{u in N(v)} x_u
    h1_v = relu(W1 [x_v; a_v] + b1),   m_v = P h1_v
    c_v  = mean_{u in N(v)} m_u
    h2_v = relu(W2 [h1_v; c_v] + b2),  z_v = Z h2_v
    t_vu = sum_j A_j z_v[j] z_u[j] + beta log2(1+w)/8 + gamma (w/wdeg_v + w/wdeg_u) + delta
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
NPARAM = O_DELTA + 1


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
        A=p[O_A:O_BETA], beta=p[O_BETA], gamma=p[O_GAMMA], delta=p[O_DELTA])


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
    t = (q["A"][None, :] * z[src] * z[col]).sum(1) + q["beta"] * ft + q["gamma"] * fg + q["delta"]
    if not keep:
        return t
    return t, dict(src=src, col=col, inv=inv, xa=xa, pre1=pre1, h1=h1, hc=hc, pre2=pre2, h2=h2, z=z,
                   ft=ft, fg=fg, n=n)


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
