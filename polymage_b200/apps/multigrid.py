"""Multigrid V- and W-cycles for the 2-D Poisson problem, as specified by
the reference's multigrid app (sandbox/apps/python/multigrid/jacobi2D:
polymage_vcycle.py:8-140, polymage_wcycle.py, polymage_smoother.py,
polymage_defect.py,
polymage_restrict.py, polymage_interpolate.py, polymage_common.py:16-75;
defaults in arg_parser.py: n = 255, L = 2, nu1 = nuc = nu2 = 1).

Level l has N_l interior points per side: N_0 = n (the parameter, the
coarsest grid), N_l = 2 N_{l-1} + 1, so the finest grid is
N_L = 2^L (n + 1) - 1.  Inputs ``V_`` (the iterate) and ``F_`` (the
right-hand side) are float64 [N_L+2][N_L+2]; the output ``Vcycle`` is the
iterate after one cycle.  Stages, each a Function over [0, N_l+1]^2 (the
restriction over its fine level's extent, computed on the coarse box):

* weighted Jacobi smoothing (omega = 4/5, c_l = omega h_l^2 / 4; a zero
  initial guess gives c_l F); its boundary ring is the input's at the
  finest level and 0 below;
* defect F - A U (5-point Laplacian over h_l^2), boundary 0;
* full-weighting restriction (1/16, 1/8, 1/4 weights at 2y+-1, 2x+-1);
* bilinear interpolation by the parities of y and x, plus the
  correction, whose values also fill the boundary ring.

The recursion follows rec_v_cycle (polymage_vcycle.py:27-140): nuc
smoothings on the coarsest level from a zero guess, nu1 pre-smoothings,
defect, restriction, the coarser cycle, interpolation with correction and
nu2 post-smoothings on the others.
"""

from ..constructs import (Parameter, Variable, Interval, Image, Function,
                          Case, Condition, Select, Int, Double)
from ..expr_ast import Value
from ..compiler import buildPipeline


def v_cycle(pipe_data=None, L=2, nu1=1, nu2=1, nuc=1, name="Vcycle",
            gamma=1):
    """``gamma`` coarse-grid visits per level: 1 is the V-cycle, 2 the
    W-cycle (polymage_wcycle.py, pipeline name ``Wcycle``)."""
    assert nu1 + nu2 + nuc > 0
    n = Parameter(Int, "n")
    y = Variable(Int, "y")
    x = Variable(Int, "x")
    if pipe_data is not None:
        pipe_data['n'] = n
    N = {0: n}
    for l in range(1, L + 1):
        N[l] = 2 * N[l - 1] + 1
    one = Value(1.0, Double)

    def consts(l):
        h = one / (N[l] + 1)
        return one / (h * h), Value(4.0 / 5.0, Double) * ((h * h) /
                                                         Value(4.0, Double))

    def extent(l):
        return Interval(Int, 0, N[l] + 1)

    def in_y(l):
        return Condition(y, ">=", 1) & Condition(y, "<=", N[l])

    def inner(l):
        return in_y(l) & Condition(x, ">=", 1) & Condition(x, "<=", N[l])

    def ghosts(l, value):
        return [Case(Condition(y, "==", 0), value),
                Case(Condition(y, "==", N[l] + 1), value),
                Case(Condition(x, "==", 0) & in_y(l), value),
                Case(Condition(x, "==", N[l] + 1) & in_y(l), value)]

    def lap(U):
        return (U(y, x) * 4.0 - U(y - 1, x) - U(y + 1, x) - U(y, x - 1) -
                U(y, x + 1))

    def smooth(U, F, l, fname):
        invhh, c = consts(l)
        W = Function(([y, x], [extent(l), extent(l)]), Double, fname)
        if U is None:
            body = [Case(inner(l), c * F(y, x))]
        else:
            body = [Case(inner(l), U(y, x) - c * (lap(U) * invhh - F(y, x)))]
        W.defn = body + ghosts(l, U(y, x) if l == L else 0.0)
        return W

    def defect(U, F, l, fname):
        if U is None:
            return F
        invhh, _ = consts(l)
        W = Function(([y, x], [extent(l), extent(l)]), Double, fname)
        W.defn = [Case(inner(l), F(y, x) - lap(U) * invhh)] + \
            ghosts(l, 0.0)
        return W

    def restrict(U, l, fname):
        W = Function(([y, x], [extent(l), extent(l)]), Double, fname)
        W.defn = [Case(inner(l - 1),
                       (U(2 * y - 1, 2 * x - 1) + U(2 * y - 1, 2 * x + 1) +
                        U(2 * y + 1, 2 * x - 1) + U(2 * y + 1, 2 * x + 1)) *
                       0.0625 +
                       (U(2 * y - 1, 2 * x) + U(2 * y + 1, 2 * x) +
                        U(2 * y, 2 * x - 1) + U(2 * y, 2 * x + 1)) * 0.125 +
                       U(2 * y, 2 * x) * 0.25)] + ghosts(l - 1, 0.0)
        return W

    def interpolate(U, corr, l, fname):
        if U is None:
            return corr
        cv = corr(y, x) if corr is not None else 0.0
        hy, hx = y / 2, x / 2
        e00 = U(hy, hx)
        e01 = (U(hy, hx) + U(hy, hx + 1)) * 0.5
        e10 = (U(hy, hx) + U(hy + 1, hx)) * 0.5
        e11 = (U(hy, hx) + U(hy + 1, hx) + U(hy, hx + 1) +
               U(hy + 1, hx + 1)) * 0.25
        even_y = Condition(y % 2, "==", 0)
        even_x = Condition(x % 2, "==", 0)
        W = Function(([y, x], [extent(l), extent(l)]), Double, fname)
        W.defn = [Case(inner(l), cv + Select(
            even_y, Select(even_x, e00, e01), Select(even_x, e10, e11)))] + \
            ghosts(l, cv)
        return W

    visits = dict((l, 0) for l in range(L + 1))

    def cycle(v, f, l):
        visits[l] += 1
        tag = "__%d" % visits[l] if gamma > 1 else ""
        if l == 0:
            if nuc == 0:
                return v
            u = v
            for t in range(nuc):
                fname = name if (l == L and t == nuc - 1) else \
                    "T%d_coarse%s" % (t, tag)
                u = smooth(u, f, l, fname)
            return u
        u = v
        for t in range(nu1):
            u = smooth(u, f, l, "T%d_pre_L%d%s" % (t, l, tag))
        r = defect(u, f, l, "defect_L%d%s" % (l, tag))
        r2 = restrict(r, l, "restrict_L%d%s" % (l - 1, tag))
        # gamma coarse-grid visits: the V-cycle one, the W-cycle two, the
        # second starting from the first one's result
        # (polymage_wcycle.py:80-84)
        e = None
        for _ in range(gamma):
            e = cycle(e, r2, l - 1)
        fname = name if (l == L and nu2 <= 0) else \
            "interp_correct_L%d%s" % (l, tag)
        ec = interpolate(e, u, l, fname)
        if nu2 <= 0:
            return ec
        for t in range(nu2):
            fname = name if (l == L and t == nu2 - 1) else \
                "T%d_post_L%d%s" % (t, l, tag)
            ec = smooth(ec, f, l, fname)
        return ec

    V = Image(Double, "V_", [N[L] + 2, N[L] + 2])
    F = Image(Double, "F_", [N[L] + 2, N[L] + 2])
    return cycle(V, F, L)


def build_v_cycle(n=255, L=2, nu1=1, nu2=1, nuc=1, tile_sizes=(16, 64),
                  group_size=6, options=(), name="Vcycle", gamma=1):
    data = {}
    out = v_cycle(data, L=L, nu1=nu1, nu2=nu2, nuc=nuc, name=name,
                  gamma=gamma)
    p = data['n']
    return buildPipeline([out], param_estimates=[(p, n)],
                         param_constraints=[Condition(p, "==", n)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size, options=list(options),
                         pipe_name=name)
