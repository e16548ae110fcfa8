"""Circular max filter (radius 26), as specified by the reference app
(sandbox/apps/python/img_proc/max_filter/polymage_maxfilter.py:14-103).

Input ``img`` is float32 [3][R][C] holding 0..255 (the reference loads an
8-bit image as floats: max_filter/init.py); output ``final`` is int32
[R][C][3].  With r = 26 and slices = ceil(log2 r) + 1 = 6:

  vert_log(x, y, c, t)  Reduction (max): for y in [r, C-R-3r-1] and t in
                        [1, slices-1], the larger of the edge-clamped image
                        at (x, y) and at (x, y + min(max(2^(t-1), 0), 2r))
  slice_for_radius(t)   (int)(log(2t+1) / 0.693147)
  vert(x, y, c, t)      max of vert_log at (y - t) and at
                        (y + t + 1 - clamp(2^e, 0, 2r)), e = its slice
  filter_height(x)      Reduction (sum): the dy in [0, r+1] with
                        x^2 + dy^2 < (r + 1/4)^2, for x in [0, r]
  final(x, y, c)        Reduction (max) over dx in [-r, 2r+1], for x in
                        [r, R-2r-2], of vert(x+dx, y, c, clamp(h(dx)))

The spec is kept as the reference writes it, with two readings of what it
leaves ill-formed:
* its first Reduce targets vert_log(x, y, c, t) where y and t are not
  reduction variables; the target here is the reduction variables' point,
  vert_log(x, rx, c, ry), the only well-formed reading;
* vert reads vert_log at y - t < 0, outside its domain; built with option
  'oob_zero' such reads give 0;
* final passes vert a slice index filter_height(dx) of up to r + 1, past
  vert's slices 0..6; that index is data dependent and, as every
  data-dependent index here, is clamped into the producer's domain.
Reduce operators are those the spec names (Op.Max / Op.Sum).  Defaults
are the Reduction default, 0.
"""

import math

from ..constructs import (Parameter, Variable, Interval, Image, Function,
                          Reduction, Reduce, Op, Case, Condition, Cast,
                          Max, Min, Pow, Log, Int, Float)
from ..compiler import buildPipeline

RADIUS = 26


def maxfilter(pipe_data=None):
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    if pipe_data is not None:
        pipe_data['R'] = R
        pipe_data['C'] = C
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    c = Variable(Int, "c")
    t = Variable(Int, "t")
    img = Image(Float, "img", [3, R, C])
    radius = RADIUS
    slices = int(math.ceil(math.log(radius, 2))) + 1
    rows = Interval(Int, 0, R - 1)
    cols = Interval(Int, 0, C - 1)
    c_int = Interval(Int, 0, 2)
    t_int = Interval(Int, 0, slices)

    def clamped(i, j, k):
        return img(k, Max(0, Min(i, R - 1)), Max(0, Min(j, C - 1)))

    def clamp(e, mn, mx):
        return Max(Min(e, mx), mn)

    rx = Variable(Int, "rx")
    ry = Variable(Int, "ry")
    vert_log = Reduction(([x, y, c, t], [rows, cols, c_int, t_int]),
                         ([x, rx, c, ry],
                          [rows, Interval(Int, radius, C - R - radius * 3 - 1),
                           c_int, Interval(Int, 1, slices - 1)]),
                         Int, "vert_log")
    vert_log.defn = [Reduce(
        vert_log(x, rx, c, ry),
        Max(clamped(x, rx, c),
            clamped(x, rx + clamp(Cast(Int, Pow(2, ry - 1)), 0, radius * 2),
                    c)),
        Op.Max)]

    slice_for_radius = Function(([t], [t_int]), Int, "slice_for_radius")
    slice_for_radius.defn = [Cast(Int, Log(2 * t + 1) / 0.693147)]

    vert = Function(([x, y, c, t], [rows, cols, c_int, t_int]), Int, "vert")
    eslice = clamp(slice_for_radius(t), 0, slices)
    first = vert_log(x, y - t, c, eslice)
    second = vert_log(x, y + t + 1 - clamp(Cast(Int, Pow(2, eslice)), 0,
                                           2 * radius), c, eslice)
    vert.defn = [Max(first, second)]

    dx = Variable(Int, "dx")
    dy = Variable(Int, "dy")
    dx_int = Interval(Int, -radius, 2 * radius + 1)
    inside = x * x + dy * dy
    rr = (radius + 0.25) * (radius + 0.25)
    filter_height = Reduction(([x], [dx_int]),
                              ([x, dy], [Interval(Int, 0, radius),
                                         Interval(Int, 0, radius + 1)]),
                              Int, "filter_height")
    filter_height.defn = [
        Case(Condition(inside, "<", rr),
             Reduce(filter_height(x), 1, Op.Sum)),
        Case(Condition(inside, ">=", rr),
             Reduce(filter_height(x), 0, Op.Sum))]

    final = Reduction(([x, y, c], [rows, cols, c_int]),
                      ([x, y, c, dx],
                       [Interval(Int, radius, R - 2 * radius - 2), cols,
                        c_int, dx_int]), Int, "final")
    final.defn = [Reduce(final(x, y, c),
                         vert(x + dx, y, c,
                              clamp(filter_height(dx), 0, radius + 1)),
                         Op.Max)]
    return final


def build_maxfilter(rows=1536, cols=2560, tile_sizes=(8, 32, 3, 7),
                    group_size=5,
                    options=('oob_zero', ('red_tile', (8, 32, 1, 16))),
                    name="maxfilter"):
    """Tiles (8, 32, 3, 7) of vert (x, y, c, t): every channel and slice
    of an 8 x 32 block; the Reductions take (8, 32, 1, 16) of their
    reduction variables."""
    data = {}
    out = maxfilter(data)
    R, C = data['R'], data['C']
    return buildPipeline([out],
                         param_estimates=[(R, rows), (C, cols)],
                         param_constraints=[Condition(R, "==", rows),
                                            Condition(C, "==", cols)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size,
                         options=list(options),
                         pipe_name=name)
