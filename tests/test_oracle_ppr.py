"""Pins the FP64 PPR oracle: exact solve vs Jacobi, and central finite
differences of the forward against the adjoint gradient.  CPU only."""
import numpy as np

from galois_b200 import assign_weights_f32, rmat
from oracle import ppr as oppr


def setup(scale=7, B=3, seed=3):
    g, _ = rmat(scale, 8, seed=seed, symmetrize=False)
    assign_weights_f32(g, seed=seed)
    rng = np.random.default_rng(seed)
    T = np.zeros((g.n, B))
    for b in range(B):
        idx = rng.choice(g.n, 5, replace=False)
        T[idx, b] = 1.0 / 5
    c = rng.standard_normal((g.n, B))
    return g, T, c, g.w_f32.astype(np.float64)


def test_exact_equals_jacobi():
    g, T, _, w = setup()
    xe = oppr.forward(g, T, w, exact=True)
    xj = oppr.forward(g, T, w, exact=False, tol=1e-15)
    assert np.abs(xe - xj).max() < 1e-12


def test_adjoint_gradient_matches_finite_differences():
    g, T, c, w = setup()
    alpha = 0.85
    x = oppr.forward(g, T, w, alpha)
    gT, gw = oppr.backward(g, x, c, w, alpha)
    loss = lambda T_, w_: float((c * oppr.forward(g, T_, w_, alpha)).sum())  # noqa: E731
    rng = np.random.default_rng(0)
    h = 1e-6
    for e in rng.choice(g.m, 12, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[e] += h
        wm[e] -= h
        fd = (loss(T, wp) - loss(T, wm)) / (2 * h)
        assert abs(fd - gw[e]) <= 1e-6 * max(1.0, abs(fd))
    for (i, b) in [(0, 0), (5, 1), (17, 2)]:
        Tp, Tm = T.copy(), T.copy()
        Tp[i, b] += h
        Tm[i, b] -= h
        fd = (loss(Tp, w) - loss(Tm, w)) / (2 * h)
        assert abs(fd - gT[i, b]) <= 1e-6 * max(1.0, abs(fd))
