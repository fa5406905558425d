"""The gate's CPU reference: its gradient against finite differences (with the
BF16 roundings off, so the loss is smooth), and the BF16 rounding helper."""
import numpy as np

from oracle import gate_oracle as G


def _data(n=64, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.random((n, 6)).astype(np.float32)
    y = (rng.random(n) < 0.35).astype(np.float32)
    w = (0.5 + rng.random(n)).astype(np.float32)
    p = (rng.standard_normal(G.NPARAMS) * 0.3).astype(np.float32)
    return p, x, y, w


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.0e-3, 65504.0], dtype=np.float32)
    r = G.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0          # tie rounds to even
    assert r[2] == np.float32(1.0078125)         # above the tie rounds up
    bits = r.view(np.uint32)
    assert np.all((bits & 0xFFFF) == 0)


def test_gradient_matches_finite_differences():
    p, x, y, w = _data()
    _, g = G.loss_and_grad(p, x, y, w, rounding=False)
    rng = np.random.default_rng(1)
    idx = np.concatenate([rng.choice(384, 6, replace=False),            # W1
                          384 + rng.choice(64, 4, replace=False),       # b1
                          448 + rng.choice(4096, 8, replace=False),     # W2
                          4544 + rng.choice(64, 4, replace=False),      # b2
                          4608 + rng.choice(64, 4, replace=False), [4672]])
    pd = p.astype(np.float64)
    for i in idx:
        eps = 1e-3
        a = pd.copy(); a[i] += eps
        b = pd.copy(); b[i] -= eps
        la, _ = G.loss_and_grad(a.astype(np.float32), x, y, w, rounding=False)
        lb, _ = G.loss_and_grad(b.astype(np.float32), x, y, w, rounding=False)
        fd = (la - lb) / (2 * eps)
        assert abs(fd - g[i]) <= 2e-3 * max(1.0, abs(fd)), (i, fd, g[i])


def test_forward_is_a_probability():
    p, x, _, _ = _data()
    prob, _ = G.forward(p, x)
    assert prob.shape == (64,) and np.all((prob > 0) & (prob < 1))
