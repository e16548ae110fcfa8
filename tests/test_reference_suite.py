"""The reference's own compiler tests (sandbox/tests/), restated for this
compiler: each builds the reference test's pipeline with the same grouping
and options, generates its CUDA source (and compiles the ones with new
code paths), and writes the stage graph the reference tests write.  Where
the reference only builds, the statements are also evaluated point by
point (tests/dsl_eval.py) against NumPy on small inputs."""

import sys

import numpy as np
import pytest

from polymage_b200.constructs import *   # noqa: F401,F403
from polymage_b200.compiler import buildPipeline
from tests.dsl_eval import Evaluator

sys.setrecursionlimit(max(sys.getrecursionlimit(), 20000))


def _graph_ok(p, tmp_path, name):
    path = tmp_path / (name + ".dot")
    p.pipeline_graph.write(str(path))
    text = path.read_text()
    assert text.count("shape=box") == len(p.comps)
    assert text.count("->") == sum(len(c.parents) for c in p.comps)
    return text


def test_tree_graph(tmp_path):
    """sandbox/tests/test_grouping.py:8-55: a binary tree of 7 stages,
    group size 100 -> one group."""
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    row = Interval(Int, 0, R - 1)
    col = Interval(Int, 0, C - 1)
    img = Image(Float, "img", [R, C])
    alpha = 0.6
    F = {}
    L = 3
    for l in range(0, 2 ** L - 1):
        F[l] = Function(([x, y], [row, col]), Float, "F" + str(l))
    for l in range(0, 2 ** (L - 1) - 1):
        F[l].defn = [alpha * F[2 * l + 1](x, y) + (1 - alpha) *
                     F[2 * l + 2](x, y)]
    for l in range(2 ** (L - 1) - 1, 2 ** L - 1):
        F[l].defn = [l * img(x, y)]
    p = buildPipeline([F[0]], param_estimates=[(R, 1024), (C, 1024)],
                      group_size=100, pipe_name="tree")
    assert len(p.groups) == 1
    _graph_ok(p, tmp_path, "tree")
    assert "pipeline_tree(" in p.generate_code().source
    # the tree evaluates to sum_l w_l * l * img
    img_v = np.random.default_rng(0).random((5, 6))
    got = Evaluator({'R': 5, 'C': 6}, {'img': img_v}).array(F[0])
    w = {3: 0.36, 4: 0.24, 5: 0.24, 6: 0.16}
    ref = sum(wl * l * img_v for l, wl in w.items())
    assert np.abs(got - ref).max() < 1e-12


def test_blur(tmp_path):
    """sandbox/tests/test_blur.py:8-68: blurx, blury grouped together."""
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    c = Variable(Int, "c")
    cr = Interval(Int, 0, 2)
    xcond = (Condition(x, '>=', 1) & Condition(x, '<=', R) &
             Condition(y, '>=', 1) & Condition(y, '<=', C))
    ycond = (Condition(x, '>=', 2) & Condition(x, '<=', R - 1) &
             Condition(y, '>=', 2) & Condition(y, '<=', C - 1))
    img = Image(Float, "input", [3, R + 2, C + 2])
    blurx = Function(([c, x, y], [cr, Interval(Int, 1, R),
                                  Interval(Int, 1, C)]), Float, "blurx")
    blurx.defn = [Case(xcond, (img(c, x - 1, y) + img(c, x, y) +
                               img(c, x + 1, y) / 3.0))]
    blury = Function(([c, x, y], [cr, Interval(Int, 2, R - 1),
                                  Interval(Int, 2, C - 1)]), Float, "blury")
    blury.defn = [Case(ycond, (blurx(c, x, y - 1) + blurx(c, x, y) +
                               blurx(c, x, y + 1) / 3.0))]
    p = buildPipeline([blury], grouping=[[blurx, blury]],
                      param_estimates=[(R, 1024), (C, 1024)],
                      pipe_name="blur")
    assert len(p.groups) == 1
    _graph_ok(p, tmp_path, "blur")
    assert "pipeline_blur(" in p.generate_code().source


def test_sampling_spec_reads_outside_its_domain():
    """sandbox/tests/test_sampling.py:8-124 as written reads level 9 at
    x/2 - 1 = -1 from x = 1: the build-time bounds check refuses it."""
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    L = 10
    row, col, cond = {}, {}, {}
    for l in range(L):
        RL, CL = R / (1 << l), C / (1 << l)
        row[l] = Interval(Int, 0, RL + 1)
        col[l] = Interval(Int, 0, CL + 1)
        cond[l] = (Condition(x, '>=', 1) & Condition(x, '<=', RL) &
                   Condition(y, '>=', 1) & Condition(y, '<=', CL))

    def taps(f, ix, iy):
        return ((f(ix - 1, iy - 1) + f(ix + 1, iy - 1) + f(ix - 1, iy + 1) +
                 f(ix + 1, iy + 1)) * 0.0625 +
                (f(ix - 1, iy) + f(ix + 1, iy) + f(ix, iy - 1) +
                 f(ix, iy + 1)) * 0.125 + f(ix, iy) * 0.25)

    def down(f, l):
        o = Function(([x, y], [row[l], col[l]]), Float, "down_%d" % l)
        o.defn = [Case(cond[l], taps(f, 2 * x, 2 * y))]
        return o

    def up(f, l):
        o = Function(([x, y], [row[l - 1], col[l - 1]]), Float,
                     "up_%d" % (l - 1))
        o.defn = [Case(cond[l - 1], taps(f, x / 2, y / 2))]
        return o
    img = Image(Float, "img", [R + 2, C + 2])
    d = {1: down(img, 1)}
    for l in range(2, L):
        d[l] = down(d[l - 1], l)
    u = {L - 2: up(d[L - 1], L - 1)}
    for l in range(L - 2, 0, -1):
        u[l - 1] = up(u[l], l)
    with pytest.raises(TypeError, match="out of domain"):
        buildPipeline([u[0]], param_estimates=[(R, 1024), (C, 1024)],
                      pipe_name="up")


def test_histogram_mixed_operators():
    """sandbox/tests/test_hist.py:8-65: one Reduction whose parts reduce
    channel 0 with Min, 1 with Max and 2 with Sum; the parts update
    disjoint cells, so each accumulates with its own atomic."""
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    c = Variable(Int, "c")
    row = Interval(Int, 0, R + 1)
    col = Interval(Int, 0, C + 1)
    img = Image(Float, "img", [R + 2, C + 2])
    hist = Reduction(([c, x], [Interval(Int, 0, 2), row]),
                     ([c, x, y], [Interval(Int, 0, 2), row, col]),
                     Float, "hist")
    hist.defn = [Case(Condition(c, '==', 0),
                      Reduce(hist(c, x), img(x, y), Op.Min)),
                 Case(Condition(c, '==', 1),
                      Reduce(hist(c, x), img(x, y), Op.Max)),
                 Case(Condition(c, '==', 2),
                      Reduce(hist(c, x), img(x, y), Op.Sum))]
    p = buildPipeline([hist], param_estimates=[(R, 1024), (C, 1024)],
                      pipe_name="hist")
    src = p.generate_code().source
    for a in ("pm_atomic_min", "pm_atomic_max", "pm_atomic_add"):
        assert a in src
    assert p.build().so_path.endswith(".so")
    v = np.random.default_rng(1).random((6, 7)) - 0.5
    got = Evaluator({'R': 4, 'C': 5}, {'img': v}).array(hist)
    # the default 0 takes part in every reduction
    ref = np.stack([np.minimum(0.0, v.min(axis=1)),
                    np.maximum(0.0, v.max(axis=1)), v.sum(axis=1)])
    assert np.abs(got - ref).max() < 1e-12


def test_math_builtins(tmp_path):
    """sandbox/tests/test_math.py:8-100: sin, cos, max, min, powf, exp,
    sqrtf, int cast, sqrt, abs, pow and a data-dependent select, fused
    (group size 100, the reference's storage options)."""
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    row = Interval(Int, 0, R - 1)
    col = Interval(Int, 0, C - 1)
    img1 = Image(Float, "img1", [R, C])
    img2 = Image(Float, "img2", [R, C])
    cond = (Condition(x, '>=', 0) & Condition(x, '<=', R - 1) &
            Condition(y, '<=', C - 1) & Condition(y, '>=', 0))

    def fn(name, typ, e):
        f = Function(([x, y], [row, col]), typ, name)
        f.defn = [Case(cond, e)]
        return f
    sin = fn("_sin", Float, Sin(img1(x, y)))
    cos = fn("_cos", Float, Cos(img2(x, y)))
    imax = fn("_max", Float, Max(sin(x, y), cos(x, y)))
    imin = fn("_min", Float, Min(sin(x, y), cos(x, y)))
    powf = fn("_powf", Float, Powf(imax(x, y), imin(x, y)))
    exp = fn("_exp", Float, Exp(powf(x, y)))
    sqrtf = fn("_sqrtf1", Float, Sqrtf(img1(x, y)))
    cast = fn("_cast", Int, Cast(Int, img2(x, y)))
    sqrt = fn("_sqrt2", Int, Sqrt(cast(x, y)))
    iabs = fn("_abs", Float, Abs(sqrtf(x, y) - sqrt(x, y)))
    ipow = fn("_pow", Float, Pow(iabs(x, y), 3))
    select = fn("_select", Float, Select(Condition(img1(x, y), '>',
                                                   img2(x, y)),
                                         ipow(x, y), exp(x, y)))
    p = buildPipeline([select], group_size=100, pipe_name="aimless",
                      options=['optimize_storage', 'early_free',
                               'pool_alloc', 'multipar'])
    _graph_ok(p, tmp_path, "math")
    assert p.build().so_path.endswith(".so")
    rng = np.random.default_rng(2)
    a = rng.random((5, 6)) * 10.0
    b = rng.random((5, 6)) * 10.0
    got = Evaluator({'R': 5, 'C': 6}, {'img1': a, 'img2': b}).array(select)
    s, co = np.sin(a), np.cos(b)
    with np.errstate(invalid='ignore'):     # C powf: NaN on a domain error
        e = np.exp(np.maximum(s, co) ** np.minimum(s, co))
    sq = np.sqrt(np.trunc(b)).astype(int)
    ip = np.abs(np.sqrt(a) - sq) ** 3
    ref = np.where(a > b, ip, e)
    ok = np.isfinite(ref)
    assert np.abs(got[ok] - ref[ok]).max() < 1e-9


@pytest.mark.parametrize("case", ["gray", "flip", "robin", "high_dim"])
def test_alignment_permuted_dimensions(case):
    """sandbox/tests/test_alignment.py:8-133: stages whose dimensions are
    permuted against their consumers' (2-D to 1-D, transposes, 3-D and
    4-D permutations) fuse into one group with the reference's grouping.
    (test_gray's 1-D stage keeps only the x conjuncts of the 2-D
    condition, whose y is not a variable of that stage.)"""
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    P = Parameter(Int, "P")
    B = Parameter(Int, "B")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    z = Variable(Int, "z")
    w = Variable(Int, "w")
    c = Variable(Int, "c")
    row = Interval(Int, 0, R + 1)
    col = Interval(Int, 0, C + 1)
    plane = Interval(Int, 0, P + 1)
    box = Interval(Int, 0, B + 1)
    cr = Interval(Int, 0, 2)
    inx = Condition(x, '>=', 1) & Condition(x, '<=', R)
    cond = inx & Condition(y, '>=', 1) & Condition(y, '<=', C)
    cond3 = cond & Condition(z, '>=', 1) & Condition(z, '<=', P)
    cond4 = cond3 & Condition(w, '>=', 1) & Condition(w, '<=', B)
    est = [(R, 512), (C, 512)]
    if case == "gray":
        img = Image(Float, "img", [R + 2, C + 2, 3])
        g = Function(([x, y], [row, col]), Float, "gray")
        g.defn = [Case(cond, img(x, y, 0) * 0.299 + img(x, y, 1) * 0.587 +
                       img(x, y, 2) * 0.114)]
        v = Function(([x], [row]), Float, "vector")
        v.defn = [Case(inx, g(x, 0))]
        groups, out = [[g, v]], v
    elif case == "flip":
        img = Image(Int, "img", [R + 2, C + 2])
        f1 = Function(([y, x], [col, row]), Int, "flip1")
        f1.defn = [Case(cond, img(x + 1, y) + img(x, y + 1))]
        f2 = Function(([x, y], [row, col]), Int, "flip2")
        f2.defn = [Case(cond, f1(y - 1, x) + f1(y, x - 1))]
        groups, out = [[f1, f2]], f2
    elif case == "robin":
        img = Image(Short, "img", [R + 2, C + 2, 3])
        r1 = Function(([c, x, y], [cr, row, col]), Short, "robin1")
        r1.defn = [Case(cond, img(x, y, c) + 1)]
        r2 = Function(([y, c, x], [col, cr, row]), Short, "robin2")
        r2.defn = [Case(cond, r1(c, x, y) - 1)]
        r3 = Function(([x, y, c], [row, col, cr]), Short, "robin3")
        r3.defn = [Case(cond, r2(y, c, x) + 1)]
        groups, out = [[r1, r2, r3]], r3
    else:
        est = est + [(P, 8), (B, 4)]
        img = Image(Short, "img", [B + 2, P + 2, R + 2, C + 2])
        specs = [([w, z, y, x], [box, plane, row, col]),
                 ([w, y, z, x], [box, row, plane, col]),
                 ([z, x, y, w], [plane, col, row, box]),
                 ([x, w, y, z], [col, box, row, plane]),
                 ([y, z, w, x], [row, plane, box, col]),
                 ([z, w, x, y], [plane, box, col, row])]
        rs = []
        prev = None
        for i, dom in enumerate(specs):
            f = Function(dom, Double, "random%d" % i)
            src = img(w, z, y, x) if prev is None else prev(*prev.variables)
            f.defn = [Case(cond4, src + (1 if i % 2 else -1))]
            rs.append(f)
            prev = f
        r6 = Function(([z, y, x], [plane, row, col]), Double, "random6")
        r6.defn = [Case(cond3, (rs[5](z, 0, x, y) + rs[5](z, 1, x, y) +
                                rs[5](z, 2, x, y) - 3) / 3.0)]
        r7 = Function(([y, x, w, z], [row, col, box, plane]), Double,
                      "random7")
        r7.defn = [Case(cond4, r6(z, y, x) * 2)]
        groups, out = [rs + [r6, r7]], r7
    p = buildPipeline([out], grouping=groups, param_estimates=est)
    assert len(p.groups) == 1
    assert len(p.generate_code().source) > 0


def test_stencil_pipeline(tmp_path):
    """sandbox/tests/test_stencil.py:10-60: two stages defined by Stencil
    macros (a 3x3 and a 2x3 kernel), grouping given as a flat list."""
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    xrow = Interval(Int, 1, R)
    xcol = Interval(Int, 1, C)
    bounds = (Condition(x, '>=', 2) & Condition(x, '<=', R - 2) &
              Condition(y, '>=', 2) & Condition(y, '<=', C - 2))
    img = Image(Float, "input", [R + 2, C + 2])
    k1 = [[1, 0, 0], [0, 2, 0], [0, 0, 1]]
    f1 = Function(([x, y], [xrow, xcol]), Float, "f1")
    f1.defn = [Case(bounds, Stencil(img, [x, y], k1))]
    k2 = [[-1, 2, -3.8], [0, -1, 0]]
    f2 = Function(([x, y], [xrow, xcol]), Float, "f2")
    f2.defn = [Case(bounds, Stencil(f1, [x, y], k2))]
    p = buildPipeline([f2], grouping=[f1, f2],
                      param_estimates=[(R, 1024), (C, 1024)],
                      pipe_name="stencil")
    _graph_ok(p, tmp_path, "stencil")
    assert "pipeline_stencil(" in p.generate_code().source
    # f2 = -f1(x, y-1) + 2 f1(x, y) - 3.8 f1(x, y+1) - f1(x+1, y) with
    # f1 = img(x-1, y-1) + 2 img(x, y) + img(x+1, y+1) on its Case box
    # [2, R-2] x [2, C-2] and 0 elsewhere (never computed there)
    v = np.random.default_rng(3).random((10, 11))
    got = Evaluator({'R': 8, 'C': 9}, {'input': v}).array(f2)

    def f1v(i, j):
        if not (2 <= i <= 6 and 2 <= j <= 7):
            return 0.0
        return v[i - 1, j - 1] + 2 * v[i, j] + v[i + 1, j + 1]
    for i in range(2, 7):
        for j in range(2, 8):
            ref = (-f1v(i, j - 1) + 2 * f1v(i, j) - 3.8 * f1v(i, j + 1) -
                   f1v(i + 1, j))
            assert abs(got[i - 1, j - 1] - ref) < 1e-12


def test_harris_with_inline_directives(tmp_path):
    """sandbox/tests/test_harris.py:8-110: Harris with the products, det
    and trace inlined by directive, and an explicit zero Case at (0, 0);
    the statement reproduces the pinned Harris oracle."""
    import oracle.harris as OH
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    row = Interval(Int, 0, R + 1)
    col = Interval(Int, 0, C + 1)
    cond = (Condition(x, '>=', 1) & Condition(x, '<=', R) &
            Condition(y, '<=', C) & Condition(y, '>=', 1))
    cred = (Condition(x, '>=', 2) & Condition(x, '<=', R - 1) &
            Condition(y, '<=', C - 1) & Condition(y, '>=', 2))
    img = Image(Float, "img", [R + 2, C + 2])

    def fn(name, c, e):
        f = Function(([x, y], [row, col]), Float, name)
        f.defn = [Case(c, e)]
        return f
    Iy = fn("Iy", cond, img(x - 1, y - 1) * (-1.0 / 12) +
            img(x - 1, y + 1) * (1.0 / 12) + img(x, y - 1) * (-2.0 / 12) +
            img(x, y + 1) * (2.0 / 12) + img(x + 1, y - 1) * (-1.0 / 12) +
            img(x + 1, y + 1) * (1.0 / 12))
    Ix = fn("Ix", cond, img(x - 1, y - 1) * (-1.0 / 12) +
            img(x + 1, y - 1) * (1.0 / 12) + img(x - 1, y) * (-2.0 / 12) +
            img(x + 1, y) * (2.0 / 12) + img(x - 1, y + 1) * (-1.0 / 12) +
            img(x + 1, y + 1) * (1.0 / 12))
    Ixx = fn("Ixx", cond, Ix(x, y) * Ix(x, y))
    Iyy = fn("Iyy", cond, Iy(x, y) * Iy(x, y))
    Ixy = fn("Ixy", cond, Ix(x, y) * Iy(x, y))

    def box3(f):
        return sum(f(x + i, y + j) for i in (-1, 0, 1) for j in (-1, 0, 1))
    Sxx = fn("Sxx", cred, box3(Ixx))
    Syy = fn("Syy", cred, box3(Iyy))
    Sxy = fn("Sxy", cred, box3(Ixy))
    det = fn("det", cred, Sxx(x, y) * Syy(x, y) - Sxy(x, y) * Sxy(x, y))
    trace = fn("trace", cred, Sxx(x, y) + Syy(x, y))
    harris = fn("harris", cred, det(x, y) - 0.04 * trace(x, y) * trace(x, y))
    harris.defn.append(Case(Condition(x, '==', 0) & Condition(y, '==', 0),
                            0.0))
    p = buildPipeline([harris], inline_directives=[Ixx, Iyy, Ixy, det, trace],
                      param_estimates=[(R, 1024), (C, 1024)],
                      pipe_name="harris_ref")
    names = set(c.func.name for c in p.comps)
    assert not names & {"Ixx", "Iyy", "Ixy", "det", "trace"}
    _graph_ok(p, tmp_path, "harris")
    assert p.build().so_path.endswith(".so")
    im = OH.make_input(16, 20, seed=4)
    ref = OH.harris(im)
    # the statement, and the pipeline's copy after inlining (the inlined
    # single-Case functions became Selects in their consumers)
    for f in (harris, p._clone_map[harris]):
        got = Evaluator({'R': 14, 'C': 18},
                        {'img': im.astype(np.float64)}).array(f)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
