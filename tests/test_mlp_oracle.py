"""The CPU oracle of the learned preconditioner (oracle/mlp_oracle.py) is
itself checked here, without a GPU: its analytic gradient equals central
finite differences of its loss (weights unrounded, so the loss is smooth),
and its BF16 rounding is round-to-nearest-even."""
import numpy as np

from oracle import mlp_oracle as M


def test_analytic_gradient_equals_finite_differences():
    F = M.feature_width()
    rng = np.random.default_rng(0)
    n = 60
    X = rng.normal(size=(n, F))
    r, u, t = rng.normal(size=n), rng.normal(size=n), rng.normal(size=n)
    den = -rng.uniform(0.1, 3.0, size=n)
    wt = rng.uniform(0.5, 2.0, size=n)
    w = M.init_weights(F, 1)
    w[-M.HID - 1:-1] *= 30.0
    _, g = M.loss_and_grad(w, F, X, r, den, u, t, wt, 0.5, 1e-12, rounding=False)
    h = 1e-6
    idx = np.concatenate([rng.choice(len(w), 60, replace=False), [len(w) - 1, len(w) - 2, 0]])
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (M.loss_and_grad(wp, F, X, r, den, u, t, wt, 0.5, 1e-12, rounding=False)[0]
              - M.loss_and_grad(wm, F, X, r, den, u, t, wt, 0.5, 1e-12, rounding=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-4 * max(abs(fd), 1e-6), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-41, 65504.0])
    y = M.bf16(x)
    assert y[0] == 1.0
    assert y[1] == 1.0          # tie, rounds to even
    assert y[2] == 1.0 + 2 ** -7
    assert y[3] == -2.5
    assert y[5] == 65536.0
