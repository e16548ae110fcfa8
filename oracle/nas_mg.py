"""The NAS MG V-cycle (mg3P) in NumPy FP64 -- test infrastructure only.
Follows the reference's app (sandbox/apps/python/multigrid/
NAS-PB-MG-3.2/polymage_mg3p.py and its restrict, interp, residual and
solver modules; coefficients from init.py:68-92).  Parity unpinned (no
reference output is kept); checked against a point-by-point evaluation of
the DSL statement."""

import numpy as np

A_COEF = (-8.0 / 3.0, 0.0, 1.0 / 6.0, 1.0 / 12.0)


def c_coef(prob_class):
    if prob_class in ('S', 'W', 'A'):
        return (-3.0 / 8.0, 1.0 / 32.0, -1.0 / 64.0, 0.0)
    return (-3.0 / 17.0, 1.0 / 33.0, -1.0 / 61.0, 0.0)


def _sh(a, dz, dy, dx):
    """a[z+dz, y+dy, x+dx] over the interior 1..m (a is (m+2)^3)."""
    m = a.shape[0] - 2
    return a[1 + dz:m + 1 + dz, 1 + dy:m + 1 + dy, 1 + dx:m + 1 + dx]


def _interior(core):
    m = core.shape[0]
    out = np.zeros((m + 2,) * 3)
    out[1:m + 1, 1:m + 1, 1:m + 1] = core
    return out


def _residual(U, V, a):
    def u1(dx):
        return (_sh(U, 0, -1, dx) + _sh(U, 0, 1, dx) + _sh(U, -1, 0, dx) +
                _sh(U, 1, 0, dx))

    def u2(dx):
        return (_sh(U, -1, -1, dx) + _sh(U, -1, 1, dx) + _sh(U, 1, -1, dx) +
                _sh(U, 1, 1, dx))
    return _interior(_sh(V, 0, 0, 0) - a[0] * _sh(U, 0, 0, 0) -
                     a[2] * (u2(0) + u1(-1) + u1(1)) -
                     a[3] * (u2(-1) + u2(1)))


def _psinv(R, U, c):
    def r1(dx):
        return (_sh(R, 0, -1, dx) + _sh(R, 0, 1, dx) + _sh(R, -1, 0, dx) +
                _sh(R, 1, 0, dx))

    def r2(dx):
        return (_sh(R, -1, -1, dx) + _sh(R, -1, 1, dx) + _sh(R, 1, -1, dx) +
                _sh(R, 1, 1, dx))
    u = 0.0 if U is None else _sh(U, 0, 0, 0)
    return _interior(u + c[0] * _sh(R, 0, 0, 0) +
                     c[1] * (_sh(R, 0, 0, -1) + _sh(R, 0, 0, 1) + r1(0)) +
                     c[2] * (r2(0) + r1(-1) + r1(1)))


def _restrict(R):
    m = (R.shape[0] - 2) // 2
    i = np.arange(1, m + 1)
    zz = (2 * i)[:, None, None]
    yy = (2 * i)[None, :, None]
    xx = (2 * i)[None, None, :]

    def p(dz, dy, dx):
        return R[zz + dz, yy + dy, xx + dx]

    def x1(dx):
        return p(0, -1, dx) + p(0, 1, dx) + p(-1, 0, dx) + p(1, 0, dx)

    def y1(dx):
        return p(-1, -1, dx) + p(-1, 1, dx) + p(1, -1, dx) + p(1, 1, dx)
    return _interior(0.5 * p(0, 0, 0) +
                     0.25 * (p(0, 0, -1) + p(0, 0, 1) + x1(0)) +
                     0.125 * (x1(-1) + x1(1) + y1(0)) +
                     0.0625 * (y1(-1) + y1(1)))


def _interp(G, U, m):
    """Over the whole [0, m+1]^3 (no boundary case)."""
    i = np.arange(0, m + 2)
    z = i[:, None, None]
    y = i[None, :, None]
    x = i[None, None, :]
    zz, yy, xx = z // 2, y // 2, x // 2

    def g(dz, dy, dx):
        return G[zz + dz, yy + dy, xx + dx]

    def z1(dx):
        return g(0, 1, dx) + g(0, 0, dx)

    def z2(dx):
        return g(1, 0, dx) + g(0, 0, dx)

    def z3(dx):
        return g(1, 1, dx) + g(1, 0, dx) + g(0, 1, dx) + g(0, 0, dx)
    e = {(0, 0, 0): g(0, 0, 0),
         (0, 0, 1): 0.5 * (g(0, 0, 0) + g(0, 0, 1)),
         (0, 1, 0): 0.5 * z1(0),
         (0, 1, 1): 0.25 * (z1(0) + z1(1)),
         (1, 0, 0): 0.5 * z2(0),
         (1, 0, 1): 0.25 * (z2(0) + z2(1)),
         (1, 1, 0): 0.25 * z3(0),
         (1, 1, 1): 0.125 * (z3(0) + z3(1))}
    out = np.zeros((m + 2,) * 3)
    for (bz, by, bx), v in e.items():
        msk = (z % 2 == bz) & (y % 2 == by) & (x % 2 == bx)
        out = np.where(msk, v, out)
    return out if U is None else U + out


def mg3p(U, V, R, prob_class='S'):
    """U, V, R: float64 [n+2]^3 -> (MG_U, MG_R)."""
    a = A_COEF
    c = c_coef(prob_class)
    n = U.shape[0] - 2
    lt = n.bit_length() - 1
    restr = {lt: np.asarray(R, np.float64)}
    for l in range(lt, 1, -1):
        restr[l - 1] = _restrict(restr[l])
    smooth = {1: _psinv(restr[1], None, c)}
    for l in range(2, lt):
        m = n >> (lt - l)
        it = _interp(smooth[l - 1], None, m)
        rs = _residual(it, restr[l], a)
        smooth[l] = _psinv(rs, it, c)
    it = _interp(smooth[lt - 1], np.asarray(U, np.float64), n)
    r_top = _residual(it, np.asarray(V, np.float64), a)
    return _psinv(r_top, it, c), r_top


def make_input(n, seed=0):
    rng = np.random.default_rng(seed)
    return tuple(rng.random((n + 2,) * 3) for _ in range(3))
