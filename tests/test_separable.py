"""Option 'separable' (polymage_b200/separable.py) on CPU: which sums are
rewritten into row sums, and that the rewritten statements compute the
same values (FP64 point-by-point evaluation; only the association of the
sums changes)."""

import sys

import numpy as np

from tests.dsl_eval import Evaluator

sys.setrecursionlimit(max(sys.getrecursionlimit(), 20000))


def _stage(p, name):
    return [c.func for c in p.comps if c.func.name == name][0]


def test_harris_box_sums_and_sobel_become_row_sums():
    import oracle.harris as OH
    from polymage_b200.apps import catalog
    p = catalog.variant("harris", ("separable",))
    assert sorted(p._separable) == ['Ix', 'Iy', 'Sxx', 'Sxy', 'Syy']
    sxx = str(_stage(p, 'Sxx').defn[0].expression)
    # three row sums of three taps each, added
    assert sxx.count('Ixx') == 9 and sxx.startswith('((((Ixx((x - 1)')
    ix = str(_stage(p, 'Ix').defn[0].expression)
    assert ') - (' in ix and ix.count('img') == 6
    # the rewritten statement computes the oracle's values
    out = [c.func for c in p.comps if c.is_output][0]
    img = OH.make_input(20, 24, seed=3)
    got = Evaluator({'R': 18, 'C': 22},
                    {'img': img.astype(np.float64)}).array(out)
    ref = OH.harris(img)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_only_rank_one_float_rectangles_are_rewritten():
    from polymage_b200.constructs import (Parameter, Variable, Interval,
                                          Image, Function, Int, Float)
    from polymage_b200.compiler import buildPipeline
    from polymage_b200.separable import separable_pass
    R = Parameter(Int, "R")
    x, y = Variable(Int, "x"), Variable(Int, "y")
    big = ([x, y], [Interval(Int, 1, R - 2), Interval(Int, 1, R - 2)])
    dom = ([x, y], [Interval(Int, 2, R - 3), Interval(Int, 2, R - 3)])
    img = Image(Float, "img", [R, R])
    rank2 = Function(big, Float, "rank2")
    rank2.defn = [img(x, y) * 1.0 + img(x, y + 1) * 2.0 +
                  img(x, y - 1) * 4.0 + img(x + 1, y) * 3.0 +
                  img(x + 1, y + 1) * 5.0 + img(x + 1, y - 1) * 7.0]
    line = Function(dom, Float, "line")
    line.defn = [rank2(x, y - 1) + rank2(x, y) + rank2(x, y + 1)]
    iimg = Image(Int, "iimg", [R, R])
    ibox = Function(dom, Int, "ibox")
    ibox.defn = [iimg(x, y) + iimg(x, y + 1) + iimg(x, y - 1) +
                 iimg(x + 1, y) + iimg(x + 1, y + 1) + iimg(x + 1, y - 1)]
    out = Function(dom, Float, "out")
    out.defn = [line(x, y) + ibox(x, y)]
    p = buildPipeline([out], param_estimates=[(R, 64)],
                      pipe_name="sep_none")
    # rank two (rank2), one dimension (line), integer (ibox): none
    assert separable_pass(p) == []


def test_separable_off_by_default():
    from polymage_b200.apps import catalog
    # the catalog's Harris build asks for it; without the option the
    # spec's left-to-right sums are kept
    assert "separable" in catalog.HARRIS['options']
    p = catalog.variant("harris", (), ("separable",))
    assert not getattr(p, '_separable', None)
    sxx = str(_stage(p, 'Sxx').defn[0].expression)
    assert sxx.startswith('((((((((Ixx')
    # NAS MG's 2x2 groups inside its 27-point sums are too small to share
    assert catalog.variant("mg3p", ("separable",))._separable == []
