"""Weighted Jacobi steps on the 2-D Poisson problem in NumPy FP64 -- test
infrastructure only.  Follows the reference's stencil app
(sandbox/apps/python/stencil/jacobi2D/polymage_jacobi.py:8-60,
polymage_common.py:16-75): interior [1, N]^2 updated, the boundary ring of
every step after the input unwritten (read as 0).  Parity unpinned: the
reference holds no output of this app; the restatement is checked against
a point-by-point evaluation of the DSL statement."""

import numpy as np


def jacobi2d(V, F, T=4):
    """V, F: float64 [N+2][N+2] -> the T-th step, float64 [N+2][N+2]."""
    V = np.asarray(V, np.float64)
    F = np.asarray(F, np.float64)
    N = V.shape[0] - 2
    h = 1.0 / (N + 1)
    invhh = 1.0 / (h * h)
    c = (4.0 / 5.0) * ((h * h) / 4.0)
    u = V
    for _ in range(T):
        w = np.zeros_like(u)
        i = slice(1, N + 1)
        w[i, i] = u[i, i] - c * ((u[i, i] * 4.0 - u[0:N, i] - u[2:N + 2, i] -
                                  u[i, 0:N] - u[i, 2:N + 2]) * invhh -
                                 F[i, i])
        u = w
    return u


def make_input(N, seed=0):
    rng = np.random.default_rng(seed)
    return rng.random((N + 2, N + 2)), rng.random((N + 2, N + 2))


def jacobi3d(V, F, T=2):
    """3-D variant (stencil/jacobi3D/polymage_jacobi.py:8-60): 7-point
    Laplacian, omega = 8/9, c = omega h^2 / 6."""
    V = np.asarray(V, np.float64)
    F = np.asarray(F, np.float64)
    N = V.shape[0] - 2
    h = 1.0 / (N + 1)
    invhh = 1.0 / (h * h)
    c = (8.0 / 9.0) * ((h * h) / 6.0)
    i = slice(1, N + 1)
    lo = slice(0, N)
    hi = slice(2, N + 2)
    u = V
    for _ in range(T):
        w = np.zeros_like(u)
        w[i, i, i] = u[i, i, i] - c * ((
            u[i, i, i] * 6.0 - u[lo, i, i] - u[hi, i, i] - u[i, lo, i] -
            u[i, hi, i] - u[i, i, lo] - u[i, i, hi]) * invhh - F[i, i, i])
        u = w
    return u
