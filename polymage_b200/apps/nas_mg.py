"""The NAS Parallel Benchmarks MG kernel's V-cycle (mg3P), as specified by
the reference's app (sandbox/apps/python/multigrid/NAS-PB-MG-3.2:
polymage_mg3p.py, polymage_restrict.py, polymage_interp.py,
polymage_residual.py, polymage_solver.py, polymage_common.py; classes and
coefficients in init.py:24-92).

Inputs ``U`` (the iterate), ``V`` (the right-hand side) and ``R`` (the
residual) are float64 [n+2]^3, n = 2^lt the problem size (class S 32, W
128, A and B 256, C 512).  Level l has n/2^(lt-l) interior points per side
plus a zero boundary ring.  The cycle restricts R from the top level down
to level 1, smooths there (``psinv``), then on each level up interpolates
the coarser correction, takes the residual and smooths; the top level adds
the interpolated correction to ``U``.  Two outputs: ``MG_U`` (the new
iterate) and ``MG_R`` (its residual).

Stencils (27-point, coefficients by distance class): residual with
a = (-8/3, 0, 1/6, 1/12), smoother with c = (-3/8, 1/32, -1/64, 0) for
classes S, W, A and (-3/17, 1/33, -1/61, 0) otherwise, full-weighting
restriction (1/2, 1/4, 1/8, 1/16), trilinear interpolation.
"""

from ..constructs import (Parameter, Variable, Interval, Image, Function,
                          Case, Condition, Select, Int, Double)
from ..expr_ast import Value
from ..compiler import buildPipeline

A_COEF = (-8.0 / 3.0, 0.0, 1.0 / 6.0, 1.0 / 12.0)
C_COEF = {'S': (-3.0 / 8.0, 1.0 / 32.0, -1.0 / 64.0, 0.0),
          'B': (-3.0 / 17.0, 1.0 / 33.0, -1.0 / 61.0, 0.0)}
SIZES = {'S': 32, 'W': 128, 'A': 256, 'B': 256, 'C': 512}


def coefficients(prob_class):
    c = C_COEF['S'] if prob_class in ('S', 'W', 'A') else C_COEF['B']
    return A_COEF, c


def mg3p(pipe_data=None, lt=5, prob_class='S'):
    a, c = coefficients(prob_class)
    a = [Value(v, Double) for v in a]
    c = [Value(v, Double) for v in c]
    n = Parameter(Int, "n")
    z = Variable(Int, "z")
    y = Variable(Int, "y")
    x = Variable(Int, "x")
    if pipe_data is not None:
        pipe_data['n'] = n
    lb = 1
    N = {lt: n + 2}
    for l in range(lt - 1, 0, -1):
        N[l] = n / (1 << (lt - l)) + 2

    def dom(l):
        return ([z, y, x], [Interval(Int, 0, N[l] - 1)] * 3)

    def within(v, l):
        return Condition(v, ">=", 1) & Condition(v, "<=", N[l] - 2)

    def inner(l):
        return within(z, l) & within(y, l) & within(x, l)

    def zero_ghosts(l):
        return [Case(Condition(z, "==", 0), 0.0),
                Case(Condition(z, "==", N[l] - 1), 0.0),
                Case(Condition(y, "==", 0) & within(z, l), 0.0),
                Case(Condition(y, "==", N[l] - 1) & within(z, l), 0.0),
                Case(Condition(x, "==", 0) & within(y, l) & within(z, l),
                     0.0),
                Case(Condition(x, "==", N[l] - 1) & within(y, l) &
                     within(z, l), 0.0)]

    def restrict(Rf, l, name):
        zz, yy, xx = 2 * z, 2 * y, 2 * x

        def x1(q):
            return (Rf(zz, yy - 1, q) + Rf(zz, yy + 1, q) +
                    Rf(zz - 1, yy, q) + Rf(zz + 1, yy, q))

        def y1(q):
            return (Rf(zz - 1, yy - 1, q) + Rf(zz - 1, yy + 1, q) +
                    Rf(zz + 1, yy - 1, q) + Rf(zz + 1, yy + 1, q))
        S = Function(dom(l - 1), Double, name)
        S.defn = [Case(inner(l - 1),
                       0.5 * Rf(zz, yy, xx) +
                       0.25 * (Rf(zz, yy, xx - 1) + Rf(zz, yy, xx + 1) +
                               x1(xx)) +
                       0.125 * (x1(xx - 1) + x1(xx + 1) + y1(xx)) +
                       0.0625 * (y1(xx - 1) + y1(xx + 1)))] + \
            zero_ghosts(l - 1)
        return S

    def interpolate(G, Uc, l, name):
        zz, yy, xx = z / 2, y / 2, x / 2

        def z1(q):
            return G(zz, yy + 1, q) + G(zz, yy, q)

        def z2(q):
            return G(zz + 1, yy, q) + G(zz, yy, q)

        def z3(q):
            return (G(zz + 1, yy + 1, q) + G(zz + 1, yy, q) +
                    G(zz, yy + 1, q) + G(zz, yy, q))
        e000 = G(zz, yy, xx)
        e001 = 0.5 * (G(zz, yy, xx) + G(zz, yy, xx + 1))
        e010 = 0.5 * z1(xx)
        e011 = 0.25 * (z1(xx) + z1(xx + 1))
        e100 = 0.5 * z2(xx)
        e101 = 0.25 * (z2(xx) + z2(xx + 1))
        e110 = 0.25 * z3(xx)
        e111 = 0.125 * (z3(xx) + z3(xx + 1))
        ex = Condition(x % 2, "==", 0)
        ey = Condition(y % 2, "==", 0)
        ez = Condition(z % 2, "==", 0)
        corr = 0.0 if Uc is None else Uc(z, y, x)
        W = Function(dom(l), Double, name)
        W.defn = [corr + Select(ez,
                                Select(ey, Select(ex, e000, e001),
                                       Select(ex, e010, e011)),
                                Select(ey, Select(ex, e100, e101),
                                       Select(ex, e110, e111)))]
        return W

    def residual(Uf, Vf, l, name):
        def u1(q):
            return (Uf(z, y - 1, q) + Uf(z, y + 1, q) +
                    Uf(z - 1, y, q) + Uf(z + 1, y, q))

        def u2(q):
            return (Uf(z - 1, y - 1, q) + Uf(z - 1, y + 1, q) +
                    Uf(z + 1, y - 1, q) + Uf(z + 1, y + 1, q))
        Rr = Function(dom(l), Double, name)
        Rr.defn = [Case(inner(l), Vf(z, y, x) - a[0] * Uf(z, y, x) -
                        a[2] * (u2(x) + u1(x - 1) + u1(x + 1)) -
                        a[3] * (u2(x - 1) + u2(x + 1)))] + zero_ghosts(l)
        return Rr

    def psinv(Rf, Uf, l, name):
        def r1(q):
            return (Rf(z, y - 1, q) + Rf(z, y + 1, q) +
                    Rf(z - 1, y, q) + Rf(z + 1, y, q))

        def r2(q):
            return (Rf(z - 1, y - 1, q) + Rf(z - 1, y + 1, q) +
                    Rf(z + 1, y - 1, q) + Rf(z + 1, y + 1, q))
        u = 0.0 if Uf is None else Uf(z, y, x)
        W = Function(dom(l), Double, name)
        W.defn = [Case(inner(l), u + c[0] * Rf(z, y, x) +
                       c[1] * (Rf(z, y, x - 1) + Rf(z, y, x + 1) + r1(x)) +
                       c[2] * (r2(x) + r1(x - 1) + r1(x + 1)))] + \
            zero_ghosts(l)
        return W

    U = Image(Double, "U", [n + 2] * 3)
    V = Image(Double, "V", [n + 2] * 3)
    R = Image(Double, "R", [n + 2] * 3)
    restr = {lt: R}
    for l in range(lt, lb, -1):
        restr[l - 1] = restrict(restr[l], l, "restrict_%d" % (l - 1))
    smooth = {lb: psinv(restr[lb], None, lb, "psinv_%d" % lb)}
    for l in range(lb + 1, lt):
        it = interpolate(smooth[l - 1], None, l, "interp_%d" % l)
        rs = residual(it, restr[l], l, "resid_%d" % l)
        smooth[l] = psinv(rs, it, l, "psinv_%d" % l)
    it = interpolate(smooth[lt - 1], U, lt, "interp_%d" % lt)
    r_top = residual(it, V, lt, "MG_R")
    u_top = psinv(r_top, it, lt, "MG_U")
    return u_top, r_top


def build_mg3p(prob_class='A', tile_sizes=(4, 8, 32), group_size=6,
               options=(), name="mg3p"):
    n = SIZES[prob_class]
    lt = n.bit_length() - 1
    data = {}
    u, r = mg3p(data, lt=lt, prob_class=prob_class)
    p = data['n']
    return buildPipeline([u, r], param_estimates=[(p, n)],
                         param_constraints=[Condition(p, "==", n)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size, options=list(options),
                         pipe_name=name)
