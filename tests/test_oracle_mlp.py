"""The MLP oracle's analytic gradients (including the second-order term of the
dE/dx loss) against central finite differences, in FP64."""
from __future__ import annotations

import numpy as np

from oracle import mlp as M


def _problem(seed=3, B=6, D=7, Dp=8, H=5):
    rng = np.random.default_rng(seed)
    p = M.Params.random(D, Dp, H, seed)
    X = np.zeros((B, Dp))
    X[:, :D] = rng.normal(size=(B, D))
    y = rng.normal(size=B)
    Gref = np.zeros((B, Dp))
    Gref[:, :D] = rng.normal(size=(B, D))
    return p, X, y, Gref, D


def test_input_gradient_is_dE_dx():
    p, X, _, _, D = _problem()
    E, G = M.forward(p, X)
    h = 1e-6
    for d in range(D):
        Xp, Xm = X.copy(), X.copy()
        Xp[:, d] += h
        Xm[:, d] -= h
        fd = (M.forward(p, Xp)[0] - M.forward(p, Xm)[0]) / (2 * h)
        assert np.allclose(fd, G[:, d], rtol=1e-6, atol=1e-8)


def test_weight_gradients_match_finite_differences():
    p, X, y, Gref, D = _problem()
    lam = 0.7
    _, g, _, _ = M.loss_and_grads(p, X, y, Gref, lam, D)
    h = 1e-6
    rng = np.random.default_rng(0)
    for name in ("W1", "b1", "W2", "b2", "w3", "b3"):
        w = getattr(p, name)
        if name == "b3":
            idx_list = [None]
        else:
            flat = np.arange(np.asarray(w).size)
            if name == "W1":   # only the live (d < D) columns carry gradient
                flat = [i for i in flat if i % w.shape[1] < D]
            idx_list = rng.choice(flat, size=min(8, len(flat)), replace=False)
        for idx in idx_list:
            def at(delta):
                q = M.Params(p.W1, p.b1, p.W2, p.b2, p.w3, p.b3)
                if name == "b3":
                    q.b3 = p.b3 + delta
                else:
                    arr = getattr(q, name).reshape(-1)
                    arr[idx] += delta
                return M.loss_only(q, X, y, Gref, lam, D)
            fd = (at(h) - at(-h)) / (2 * h)
            an = g[name] if name == "b3" else np.asarray(g[name]).reshape(-1)[idx]
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)), (name, idx, fd, an)


def test_padded_columns_stay_zero():
    p, X, y, Gref, D = _problem()
    _, g, _, _ = M.loss_and_grads(p, X, y, Gref, 1.0, D)
    assert np.all(g["W1"][:, D:] == 0.0)


def test_round_bf16_ties_to_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5e-3], np.float64)
    r = M.round_bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                 # tie, even mantissa kept
    assert r[2] == 1.0 + 2 ** -6       # tie, rounds up to even
    assert r[3] == 1.0
    assert abs(r[4] / x[4] - 1.0) < 2 ** -8
