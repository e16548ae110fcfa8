"""Multigrid V-cycle for the 2-D Poisson problem in NumPy FP64 -- test
infrastructure only.  Follows the reference's multigrid app
(sandbox/apps/python/multigrid/jacobi2D/polymage_vcycle.py:27-140 and the
smoother, defect, restrict and interpolate modules): weighted Jacobi with
omega 4/5, 5-point defect, full-weighting restriction, bilinear
interpolation with correction; boundary rings as the spec sets them.
Parity unpinned (no reference output exists); checked against a
point-by-point evaluation of the DSL statement."""

import numpy as np


def _consts(N):
    h = 1.0 / (N + 1)
    return 1.0 / (h * h), (4.0 / 5.0) * ((h * h) / 4.0)


def _lap(U, N):
    i = slice(1, N + 1)
    return (U[i, i] * 4.0 - U[0:N, i] - U[2:N + 2, i] - U[i, 0:N] -
            U[i, 2:N + 2])


def _ring(W, U, N, finest):
    """Boundary ring: the input's values at the finest level, else 0."""
    if finest:
        W[0, :] = U[0, :]
        W[N + 1, :] = U[N + 1, :]
        W[1:N + 1, 0] = U[1:N + 1, 0]
        W[1:N + 1, N + 1] = U[1:N + 1, N + 1]
    return W


def _smooth(U, F, N, finest):
    invhh, c = _consts(N)
    W = np.zeros((N + 2, N + 2))
    i = slice(1, N + 1)
    if U is None:
        W[i, i] = c * F[i, i]
    else:
        W[i, i] = U[i, i] - c * (_lap(U, N) * invhh - F[i, i])
    return _ring(W, U, N, finest) if U is not None else W


def _defect(U, F, N):
    invhh, _ = _consts(N)
    W = np.zeros((N + 2, N + 2))
    i = slice(1, N + 1)
    W[i, i] = F[i, i] - _lap(U, N) * invhh
    return W


def _restrict(U, Nc):
    W = np.zeros((Nc + 2, Nc + 2))
    y = np.arange(1, Nc + 1)[:, None]
    x = np.arange(1, Nc + 1)[None, :]
    W[1:Nc + 1, 1:Nc + 1] = (
        (U[2 * y - 1, 2 * x - 1] + U[2 * y - 1, 2 * x + 1] +
         U[2 * y + 1, 2 * x - 1] + U[2 * y + 1, 2 * x + 1]) * 0.0625 +
        (U[2 * y - 1, 2 * x] + U[2 * y + 1, 2 * x] + U[2 * y, 2 * x - 1] +
         U[2 * y, 2 * x + 1]) * 0.125 + U[2 * y, 2 * x] * 0.25)
    return W


def _interpolate(E, corr, N):
    y = np.arange(1, N + 1)[:, None]
    x = np.arange(1, N + 1)[None, :]
    hy, hx = y // 2, x // 2
    e00 = E[hy, hx]
    e01 = (E[hy, hx] + E[hy, hx + 1]) * 0.5
    e10 = (E[hy, hx] + E[hy + 1, hx]) * 0.5
    e11 = (E[hy, hx] + E[hy + 1, hx] + E[hy, hx + 1] + E[hy + 1, hx + 1]) * \
        0.25
    ey = (y % 2) == 0
    ex = (x % 2) == 0
    up = np.where(ey, np.where(ex, e00, e01), np.where(ex, e10, e11))
    W = np.zeros((N + 2, N + 2)) if corr is None else corr.copy()
    if corr is None:
        W[1:N + 1, 1:N + 1] = up
    else:
        W[1:N + 1, 1:N + 1] = corr[1:N + 1, 1:N + 1] + up
    return W


def v_cycle(V, F, n, L=2, nu1=1, nu2=1, nuc=1, gamma=1):
    """V, F: float64 [N_L+2]^2 with N_L = 2^L (n+1) - 1; ``gamma`` 2 is
    the W-cycle (polymage_wcycle.py:80-84: the coarse cycle twice, the
    second from the first's result)."""
    N = [n]
    for _ in range(L):
        N.append(2 * N[-1] + 1)

    def cycle(v, f, l):
        if l == 0:
            u = v
            for _ in range(nuc):
                u = _smooth(u, f, N[0], l == L)
            return u
        u = v
        for _ in range(nu1):
            u = _smooth(u, f, N[l], l == L)
        r = f if u is None else _defect(u, f, N[l])
        r2 = _restrict(r, N[l - 1])
        e = None
        for _ in range(gamma):
            e = cycle(e, r2, l - 1)
        ec = u if e is None else _interpolate(e, u, N[l])
        for _ in range(nu2):
            ec = _smooth(ec, f, N[l], l == L)
        return ec

    return cycle(np.asarray(V, np.float64), np.asarray(F, np.float64), L)


def make_input(n, L=2, seed=0):
    N = n
    for _ in range(L):
        N = 2 * N + 1
    rng = np.random.default_rng(seed)
    return rng.random((N + 2, N + 2)), rng.random((N + 2, N + 2))


# ---------------------------------------------------------------------------
# 3-D (multigrid/jacobi3D): 7-point operator, omega 8/9, 27-point
# restriction summed corners / edges / faces / centre, trilinear
# interpolation in the reference's summation order.

_ORDER3 = {(0, 0, 0): [(0, 0, 0)],
           (0, 0, 1): [(0, 0, 0), (0, 0, 1)],
           (0, 1, 0): [(0, 0, 0), (0, 1, 0)],
           (1, 0, 0): [(0, 0, 0), (1, 0, 0)],
           (0, 1, 1): [(0, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1)],
           (1, 0, 1): [(0, 0, 0), (1, 0, 0), (0, 0, 1), (1, 0, 1)],
           (1, 1, 0): [(0, 0, 0), (0, 1, 0), (1, 0, 0), (1, 1, 0)],
           (1, 1, 1): [(0, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1),
                       (1, 0, 0), (1, 1, 0), (1, 0, 1), (1, 1, 1)]}


def _sl(N, o):
    return slice(1 + o, N + 1 + o)


def _lap3(U, N):
    c = U[_sl(N, 0), _sl(N, 0), _sl(N, 0)] * 6.0
    for k in range(3):
        for o in (-1, 1):
            s = [_sl(N, 0)] * 3
            s[k] = _sl(N, o)
            c = c - U[tuple(s)]
    return c


def _ring3(W, U, N, finest):
    if finest:
        i = slice(1, N + 1)
        W[0], W[N + 1] = U[0], U[N + 1]
        W[i, 0, :], W[i, N + 1, :] = U[i, 0, :], U[i, N + 1, :]
        W[i, i, 0], W[i, i, N + 1] = U[i, i, 0], U[i, i, N + 1]
    return W


def _smooth3(U, F, N, finest):
    h = 1.0 / (N + 1)
    invhh, c = 1.0 / (h * h), (8.0 / 9.0) * ((h * h) / 6.0)
    W = np.zeros((N + 2,) * 3)
    i = (slice(1, N + 1),) * 3
    if U is None:
        W[i] = c * F[i]
        return W
    W[i] = U[i] - c * (_lap3(U, N) * invhh - F[i])
    return _ring3(W, U, N, finest)


def _defect3(U, F, N):
    h = 1.0 / (N + 1)
    W = np.zeros((N + 2,) * 3)
    i = (slice(1, N + 1),) * 3
    W[i] = F[i] - _lap3(U, N) * (1.0 / (h * h))
    return W


def _restrict3(U, Nc):
    import itertools
    z = np.arange(1, Nc + 1)[:, None, None]
    y = np.arange(1, Nc + 1)[None, :, None]
    x = np.arange(1, Nc + 1)[None, None, :]

    def pt(o):
        return U[2 * z + o[0], 2 * y + o[1], 2 * x + o[2]]
    offs = list(itertools.product((-1, 0, 1), repeat=3))
    groups = [([o for o in offs if sum(1 for t in o if t) == 3], 1 / 64.0),
              ([o for o in offs if sum(1 for t in o if t) == 2], 1 / 32.0),
              ([(-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1),
                (0, 0, 1)], 1 / 16.0),
              ([(0, 0, 0)], 1 / 8.0)]
    body = None
    for grp, w in groups:
        s = pt(grp[0])
        for o in grp[1:]:
            s = s + pt(o)
        body = s * w if body is None else body + s * w
    W = np.zeros((Nc + 2,) * 3)
    W[1:Nc + 1, 1:Nc + 1, 1:Nc + 1] = body
    return W


def _interpolate3(E, corr, N):
    z = np.arange(1, N + 1)[:, None, None]
    y = np.arange(1, N + 1)[None, :, None]
    x = np.arange(1, N + 1)[None, None, :]
    hz, hy, hx = z // 2, y // 2, x // 2
    up = np.zeros((N, N, N))
    for bits, pts in _ORDER3.items():
        e = None
        for d in pts:
            t = E[hz + d[0], hy + d[1], hx + d[2]]
            e = t if e is None else e + t
        if len(pts) > 1:
            e = e * (1.0 / len(pts))
        m = ((z % 2 == bits[0]) & (y % 2 == bits[1]) & (x % 2 == bits[2]))
        up = np.where(m, e, up)
    W = np.zeros((N + 2,) * 3) if corr is None else corr.copy()
    i = (slice(1, N + 1),) * 3
    W[i] = (0.0 if corr is None else corr[i]) + up
    return W


def v_cycle3d(V, F, n, L=2, nu1=1, nu2=1, nuc=1, gamma=1):
    """V, F: float64 [N_L+2]^3 with N_L = 2^L (n+1) - 1."""
    N = [n]
    for _ in range(L):
        N.append(2 * N[-1] + 1)

    def cycle(v, f, l):
        if l == 0:
            u = v
            for _ in range(nuc):
                u = _smooth3(u, f, N[0], l == L)
            return u
        u = v
        for _ in range(nu1):
            u = _smooth3(u, f, N[l], l == L)
        r = f if u is None else _defect3(u, f, N[l])
        r2 = _restrict3(r, N[l - 1])
        e = None
        for _ in range(gamma):
            e = cycle(e, r2, l - 1)
        ec = u if e is None else _interpolate3(e, u, N[l])
        for _ in range(nu2):
            ec = _smooth3(ec, f, N[l], l == L)
        return ec

    return cycle(np.asarray(V, np.float64), np.asarray(F, np.float64), L)


def make_input3d(n, L=2, seed=0):
    N = n
    for _ in range(L):
        N = 2 * N + 1
    rng = np.random.default_rng(seed)
    return rng.random((N + 2,) * 3), rng.random((N + 2,) * 3)
