"""Non-local means denoising, as specified by the reference app
(sandbox/apps/python/img_proc/non_local_means/polymage_nlmeans.py:13-165)
with its settings (non_local_means/Makefile:11-12: patch size 7, search
area 7; builder.py:53-80).

Input ``img`` is float32 [3][R][C]; output ``non_local_means`` is float32
[3][R][C]; parameters ``C, R, patch_size, search_area`` (sorted by name in
the C ABI).  With s = search_area and p = patch_size:

  dc(c, x, y, dx, dy)   squared difference of the edge-clamped image at
                        (x, y) and (x+dx, y+dy), for c in 0..3 and offsets
                        dx, dy in [-s/2, s+1]
  d(x, y, dx, dy)       Reduction: the sum of dc over c in 0..3
  blur_d_y, blur_d      Reductions: sums of d over a window [-p/2, p+1]
                        along y, then along x (each on its interior)
  w(x, y, dx, dy)       exp(blur_d * (-1 / (0.12^2 p^2)))
  clamped_with_alpha    the edge-clamped image for c in 0..2, 1.0 for c = 3
  non_local_means_sum   Reduction over the offsets (and the interior of x,
                        y) of w * clamped_with_alpha(c, x+dx, y+dy)
  non_local_means       clamp(sum(c) / sum(3), 0, 1)

The spec reads channel 3 of the 3-channel image (``dc`` ranges c over
0..3): the reference's driver hands it a 4-channel buffer whose channel 3
is zero (non_local_means/init.py:28-29).  Built with option 'oob_zero',
such a read outside the image's domain reads 0 here, which is that
driver's value.  The windows and offsets are the spec's, asymmetric as it
writes them.
"""

from ..constructs import (Parameter, Variable, Interval, Image, Function,
                          Reduction, Reduce, Op, Condition, Select, Cast,
                          Max, Min, Exp, Powf, Int, Float)
from ..compiler import buildPipeline

SIGMA = 0.12


def nlmeans(pipe_data=None):
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    patch_size = Parameter(Int, "patch_size")
    search_area = Parameter(Int, "search_area")
    if pipe_data is not None:
        pipe_data['R'] = R
        pipe_data['C'] = C
        pipe_data['patch_size'] = patch_size
        pipe_data['search_area'] = search_area
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    c = Variable(Int, "c")
    dx = Variable(Int, "dx")
    dy = Variable(Int, "dy")
    pv = Variable(Int, "patch_var")
    img = Image(Float, "img", [3, R, C])
    rows = Interval(Int, 0, R - 1)
    cols = Interval(Int, 0, C - 1)
    colours = Interval(Int, 0, 3)
    offs = Interval(Int, -search_area / 2, search_area + 1)

    def clamped(k, i, j):
        return img(k, Max(Min(i, R - 1), 0), Max(Min(j, C - 1), 0))

    inv_sigma_sq = -1.0 / (SIGMA * SIGMA * patch_size * patch_size)
    dom4 = ([x, y, dx, dy], [rows, cols, offs, offs])

    dc = Function(([c, x, y, dx, dy], [colours, rows, cols, offs, offs]),
                  Float, "dc")
    dc.defn = [Powf(clamped(c, x, y) - clamped(c, x + dx, y + dy), 2)]

    d = Reduction(dom4, ([x, y, dx, dy, c],
                         [rows, cols, offs, offs, colours]), Float, "d")
    d.defn = [Reduce(d(x, y, dx, dy), dc(c, x, y, dx, dy), Op.Sum)]
    d.default = 0.0

    window = Interval(Int, -patch_size / 2, patch_size + 1)
    blur_d_y = Reduction(dom4, ([x, y, dx, dy, pv],
                                [rows, Interval(Int, patch_size / 2,
                                                C - patch_size - 2),
                                 offs, offs, window]), Float, "blur_d_y")
    blur_d_y.defn = [Reduce(blur_d_y(x, y, dx, dy), d(x, y + pv, dx, dy),
                            Op.Sum)]
    blur_d_y.default = 0.0
    blur_d = Reduction(dom4, ([x, y, dx, dy, pv],
                              [Interval(Int, patch_size / 2,
                                        R - patch_size - 2),
                               cols, offs, offs, window]), Float, "blur_d")
    blur_d.defn = [Reduce(blur_d(x, y, dx, dy), blur_d_y(x + pv, y, dx, dy),
                          Op.Sum)]
    blur_d.default = 0.0

    w = Function(dom4, Float, "w")
    w.defn = [Exp(blur_d(x, y, dx, dy) * inv_sigma_sq)]

    rgb = Condition(c, ">=", 0) & Condition(c, "<=", 2)
    cwa = Function(([c, x, y], [colours, rows, cols]), Float,
                   "clamped_with_alpha")
    cwa.defn = [Select(rgb, clamped(c, x, y), 1.0)]

    nls = Reduction(([c, x, y], [colours, rows, cols]),
                    ([c, x, y, dx, dy],
                     [colours, Interval(Int, search_area / 2,
                                        R - search_area - 2),
                      Interval(Int, search_area / 2, C - search_area - 2),
                      offs, offs]), Float, "non_local_means_sum")
    nls.defn = [Reduce(nls(c, x, y),
                       w(x, y, dx, dy) * cwa(c, x + dx, y + dy), Op.Sum)]
    nls.default = 0.0

    out = Function(([c, x, y], [Interval(Int, 0, 2), rows, cols]), Float,
                   "non_local_means")
    out.defn = [Max(Min(nls(c, x, y) / nls(3, x, y), 1.0), 0.0)]
    if pipe_data is not None:
        pipe_data['pointwise'] = [dc, w, cwa]
    return out


def build_nlmeans(rows=256, cols=256, patch_size=7, search_area=7,
                  tile_sizes=(16, 64), group_size=5,
                  options=('oob_zero',
                           ('red_tile', (1, 16, 12, 12, 16)),
                           ('red_tile:non_local_means_sum',
                            (4, 2, 32, 12, 12))),
                  inline=True, name="nlmeans"):
    """The reductions are output-stationary: a thread owns cells of the
    target and sums over the remaining reduction variable(s).  d, blur_d_y
    and blur_d take tiles of 1 x 16 pixels x all 12 x 12 offsets (the
    offsets innermost, as in memory); the weighted sum takes 4 channels x
    2 x 32 pixels per tile and loops over the 144 offsets.  With
    ``inline`` the pointwise stages dc, w and clamped_with_alpha are
    substituted into their consumers (inline directives, as the
    reference's compiler takes them) instead of being stored."""
    data = {}
    out = nlmeans(data)
    R, C = data['R'], data['C']
    ps, sa = data['patch_size'], data['search_area']
    return buildPipeline([out],
                         inline_directives=data['pointwise'] if inline
                         else [],
                         param_estimates=[(R, rows), (C, cols),
                                          (ps, patch_size),
                                          (sa, search_area)],
                         param_constraints=[Condition(R, "==", rows),
                                            Condition(C, "==", cols)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size,
                         options=list(options),
                         pipe_name=name)
