"""Multigrid V- and W-cycles for the 2-D and 3-D Poisson problems, as
specified by the reference's multigrid apps (sandbox/apps/python/multigrid/jacobi2D:
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


# coarse points averaged per parity pattern (1: odd along that dimension),
# in the order the reference's interpolation sums them
_INTERP_ORDER = {
    2: {(0, 0): [(0, 0)],
        (0, 1): [(0, 0), (0, 1)],
        (1, 0): [(0, 0), (1, 0)],
        (1, 1): [(0, 0), (1, 0), (0, 1), (1, 1)]},
    3: {(0, 0, 0): [(0, 0, 0)],
        (0, 0, 1): [(0, 0, 0), (0, 0, 1)],
        (0, 1, 0): [(0, 0, 0), (0, 1, 0)],
        (1, 0, 0): [(0, 0, 0), (1, 0, 0)],
        (0, 1, 1): [(0, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1)],
        (1, 0, 1): [(0, 0, 0), (1, 0, 0), (0, 0, 1), (1, 0, 1)],
        (1, 1, 0): [(0, 0, 0), (0, 1, 0), (1, 0, 0), (1, 1, 0)],
        (1, 1, 1): [(0, 0, 0), (0, 1, 0), (0, 0, 1), (0, 1, 1),
                    (1, 0, 0), (1, 1, 0), (1, 0, 1), (1, 1, 1)]},
}


def _restrict_groups(dims):
    """(offsets, weight) groups of the full-weighting restriction."""
    import itertools
    offs = list(itertools.product((-1, 0, 1), repeat=dims))
    out = []
    for nz in range(dims, 0, -1):
        if nz == 1:
            grp = [tuple(o if j == k else 0 for j in range(dims))
                   for k in range(dims) for o in (-1, 1)]
        else:
            grp = [o for o in offs if sum(1 for t in o if t) == nz]
        out.append((grp, 1.0 / float(1 << (dims + nz))))
    out.append(([(0,) * dims], 1.0 / float(1 << dims)))
    return out


def v_cycle(pipe_data=None, L=2, nu1=1, nu2=1, nuc=1, name="Vcycle",
            gamma=1, dims=2):
    """``gamma`` coarse-grid visits per level: 1 is the V-cycle, 2 the
    W-cycle (polymage_wcycle.py, pipeline name ``Wcycle``).  ``dims`` 3 is
    the 3-D app (multigrid/jacobi3D: 7-point operator, omega 8/9,
    27-point restriction, trilinear interpolation)."""
    assert nu1 + nu2 + nuc > 0 and dims in (2, 3)
    n = Parameter(Int, "n")
    vs = [Variable(Int, v) for v in ("z", "y", "x")[3 - dims:]]
    if pipe_data is not None:
        pipe_data['n'] = n
    N = {0: n}
    for l in range(1, L + 1):
        N[l] = 2 * N[l - 1] + 1
    one = Value(1.0, Double)
    omega = Value(4.0 / 5.0 if dims == 2 else 8.0 / 9.0, Double)
    diag = Value(2.0 * dims, Double)

    def consts(l):
        h = one / (N[l] + 1)
        return one / (h * h), omega * ((h * h) / diag)

    def dom(l):
        return (list(vs), [Interval(Int, 0, N[l] + 1)] * dims)

    def within(v, l):
        return Condition(v, ">=", 1) & Condition(v, "<=", N[l])

    def inner(l):
        c = within(vs[0], l)
        for v in vs[1:]:
            c = c & within(v, l)
        return c

    def ghosts(l, value):
        """The boundary faces in the reference's order (polymage_common
        set_cases): the outermost dimension's two faces whole, each inner
        dimension's faces within the interior of the outer ones."""
        out = []
        for k, v in enumerate(vs):
            for side in (0, N[l] + 1):
                c = Condition(v, "==", side)
                for u in vs[:k]:
                    c = c & within(u, l)
                out.append(Case(c, value))
        return out

    def at(U, offs):
        return U(*[v + o for v, o in zip(vs, offs)])

    def lap(U):
        e = U(*vs) * (4.0 if dims == 2 else 6.0)
        for k in range(dims):
            for o in (-1, 1):
                e = e - at(U, [o if j == k else 0 for j in range(dims)])
        return e

    def smooth(U, F, l, fname):
        invhh, c = consts(l)
        W = Function(dom(l), Double, fname)
        if U is None:
            body = [Case(inner(l), c * F(*vs))]
        else:
            body = [Case(inner(l), U(*vs) - c * (lap(U) * invhh - F(*vs)))]
        W.defn = body + ghosts(l, U(*vs) if l == L else 0.0)
        return W

    def defect(U, F, l, fname):
        if U is None:
            return F
        invhh, _ = consts(l)
        W = Function(dom(l), Double, fname)
        W.defn = [Case(inner(l), F(*vs) - lap(U) * invhh)] + \
            ghosts(l, 0.0)
        return W

    def restrict(U, l, fname):
        """Full weighting, weight 2^-(dims + nonzero offsets), summed in
        the reference's groups and order (polymage_restrict.py): corners,
        then edges (3-D), then faces dimension by dimension, then the
        centre."""
        def pt(offs):
            return U(*[2 * v + o for v, o in zip(vs, offs)])
        body = None
        for grp, w in _restrict_groups(dims):
            t = pt(grp[0])
            for o in grp[1:]:
                t = t + pt(o)
            term = t * w
            body = term if body is None else body + term
        W = Function(dom(l), Double, fname)
        W.defn = [Case(inner(l - 1), body)] + ghosts(l - 1, 0.0)
        return W

    def interpolate(U, corr, l, fname):
        if U is None:
            return corr
        cv = corr(*vs) if corr is not None else 0.0
        hs = [v / 2 for v in vs]

        def avg(bits):
            """Mean of the coarse points around an odd/even pattern, in the
            reference's order (polymage_interpolate.py)."""
            pts = _INTERP_ORDER[dims][tuple(bits)]
            e = None
            for d in pts:
                t = U(*[h + k for h, k in zip(hs, d)])
                e = t if e is None else e + t
            return e if len(pts) == 1 else e * (1.0 / len(pts))

        def sel(k, bits):
            if k == dims:
                return avg(bits)
            return Select(Condition(vs[k] % 2, "==", 0),
                          sel(k + 1, bits + [0]), sel(k + 1, bits + [1]))
        W = Function(dom(l), Double, fname)
        W.defn = [Case(inner(l), cv + sel(0, []))] + ghosts(l, cv)
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

    V = Image(Double, "V_", [N[L] + 2] * dims)
    F = Image(Double, "F_", [N[L] + 2] * dims)
    return cycle(V, F, L)


def build_v_cycle(n=255, L=2, nu1=1, nu2=1, nuc=1, tile_sizes=(16, 64),
                  group_size=6, options=(), name="Vcycle", gamma=1, dims=2):
    data = {}
    out = v_cycle(data, L=L, nu1=nu1, nu2=nu2, nuc=nuc, name=name,
                  gamma=gamma, dims=dims)
    p = data['n']
    return buildPipeline([out], param_estimates=[(p, n)],
                         param_constraints=[Condition(p, "==", n)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size, options=list(options),
                         pipe_name=name)
