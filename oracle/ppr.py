"""ORACLE -- test infrastructure only.

FP64 personalised PageRank and its gradient (numpy/scipy).  There is no
reference implementation of this path (it is an addition beside the PageRank
apps), so this oracle is pinned by its own algebra: an exact sparse solve
cross-checked against the Jacobi iteration, and finite differences of the FP64
forward against the FP64 adjoint gradient (tests/test_oracle_ppr.py).

Conventions (match include/gb.h): arcs j->i in CSR order with weight w[e];
s_j = sum of j's out-weights; W~_ij = w_ji / s_j;
x = (1-a) T + a W~ x;  lam = gx + a W~^T lam;
dL/dT = (1-a) lam;  dL/dw_ji = a/s_j * sum_b x_j^b (lam_i^b - mu_j^b),
mu_j = (lam_j - gx_j)/a.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def _rows(g) -> np.ndarray:
    return np.repeat(np.arange(g.n, dtype=np.int64), g.degrees())


def wtilde(g, w) -> sp.csr_matrix:
    """W~ as an n x n matrix, entry (i, j) = w_ji / s_j."""
    w = np.asarray(w, np.float64)
    src = _rows(g)
    s = np.bincount(src, weights=w, minlength=g.n)
    vals = np.where(s[src] > 0, w / np.where(s[src] > 0, s[src], 1.0), 0.0)
    return sp.csr_matrix((vals, (g.col.astype(np.int64), src)), shape=(g.n, g.n))


def forward(g, T, w, alpha=0.85, exact=True, tol=1e-14, max_iter=10000):
    """x solving (I - a W~) x = (1-a) T (exact sparse solve, or Jacobi)."""
    W = wtilde(g, w)
    T = np.asarray(T, np.float64)
    if exact:
        A = (sp.identity(g.n, format="csc") - alpha * W.tocsc())
        lu = spla.splu(A)
        return lu.solve((1 - alpha) * T)
    x = (1 - alpha) * T
    for _ in range(max_iter):
        y = (1 - alpha) * T + alpha * (W @ x)
        if np.abs(y - x).sum(axis=0).max() <= tol:
            return y
        x = y
    return x


def backward(g, x, gx, w, alpha=0.85):
    """(dL/dT, dL/dw) for L with dL/dx = gx, in FP64 (exact adjoint solve)."""
    W = wtilde(g, w)
    A = (sp.identity(g.n, format="csc") - alpha * W.T.tocsc())
    lam = spla.splu(A).solve(np.asarray(gx, np.float64))
    gT = (1 - alpha) * lam
    src = _rows(g)
    s = np.bincount(src, weights=np.asarray(w, np.float64), minlength=g.n)
    mu = (lam - gx) / alpha
    dots = np.einsum("eb,eb->e", x[src], lam[g.col.astype(np.int64)] - mu[src])
    gw = np.where(s[src] > 0, alpha / np.where(s[src] > 0, s[src], 1.0), 0.0) * dots
    return gT, gw
