"""CPU checks of the float64 learned-scorer reference (oracle/gnn_ref.py):
its analytic gradient against central finite differences, the BF16 rounding,
and the symmetry of the logits that the GPU backward pass relies on."""
import numpy as np

from oracle import gnn_ref as R
from thegraphpartitioning_b200 import graphs
from helpers import to_np, weighted


def _setup():
    rp, ci = to_np(*graphs.grid2d(6, 7))
    ew, vw = weighted(rp, ci, seed=2, wmax=5)
    n = len(rp) - 1
    p = R.init_params(3).astype(np.float64)
    rng = np.random.default_rng(1)
    p[R.O_B1:R.O_P] = rng.normal(0, 0.3, R.H)
    p[R.O_B2:R.O_Z] = rng.normal(0, 0.3, R.H)
    p[R.O_GAMMA], p[R.O_DELTA] = 0.4, -0.2
    src = np.repeat(np.arange(n), np.diff(rp))
    part = np.arange(n) * 3 // n
    return rp, ci, ew, vw, p, (part[src] == part[ci]).astype(np.uint8)


def test_gradient_finite_differences():
    rp, ci, ew, vw, p, lab = _setup()
    _, g = R.loss_and_grad(p, rp, ci, lab, vw, ew, level=2)
    eps, worst = 1e-6, 0.0
    for i in list(range(0, R.NPARAM, 61)) + list(range(R.O_A, R.NPARAM)):
        q = p.copy(); q[i] += eps
        lp, _ = R.loss_and_grad(q, rp, ci, lab, vw, ew, 2)
        q[i] -= 2 * eps
        lm, _ = R.loss_and_grad(q, rp, ci, lab, vw, ew, 2)
        fd = (lp - lm) / (2 * eps)
        worst = max(worst, abs(fd - g[i]) / (abs(fd) + 1e-6))
    assert worst < 1e-4


def test_logits_symmetric():
    rp, ci, ew, vw, p, _ = _setup()
    t = R.forward(p, rp, ci, vw, ew, 1)
    n = len(rp) - 1
    src = np.repeat(np.arange(n), np.diff(rp))
    d = {(int(a), int(b)): x for a, b, x in zip(src, ci, t)}
    assert all(abs(d[(b, a)] - x) < 1e-12 for (a, b), x in d.items())


def test_bf16_round():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0, 1e-30], dtype=np.float32)
    r = R.bf16_round(x)
    # bfloat16 keeps 8 significant bits: 1 + 2^-8 ties to even (1.0), 1 + 1.5*2^-8 rounds up
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-12
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)


def test_priority_quantisation():
    t = np.array([0.0, 1.0, -1.0, 1e9, -1e9])
    q = R.priorities(t)
    assert list(q[:3]) == [1 << 30, (1 << 30) + 65536, (1 << 30) - 65536]
    assert q[3] == 2147483520 and q[4] == 0


def test_move_head_gradient_central_differences():
    """The float64 move-order head: analytic gradient against central differences."""
    from oracle import gnn_ref as R
    rng = np.random.default_rng(3)
    n = 400
    feat = R.move_features(rng.integers(-300, 300, n), rng.integers(1, 200, n), rng.integers(1, 9, n), 3)
    label = (rng.random(n) < 0.4).astype(np.uint8)
    p = R.move_init_params(2).astype(np.float64) + rng.normal(0, 0.2, R.MNPARAM)
    _, g = R.move_loss_and_grad(p, feat, label)
    h = 1e-6
    for i in range(R.MNPARAM):
        q1, q2 = p.copy(), p.copy()
        q1[i] += h
        q2[i] -= h
        num = (R.move_loss_and_grad(q1, feat, label)[0] - R.move_loss_and_grad(q2, feat, label)[0]) / (2 * h)
        assert abs(num - g[i]) <= 1e-6 + 1e-4 * abs(num), (i, num, g[i])
