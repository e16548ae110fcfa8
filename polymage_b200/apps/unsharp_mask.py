"""Unsharp mask, as specified by the reference app
(sandbox/apps/python/img_proc/unsharp_mask/polymage_unsharp_mask.py:16-77),
built with its group size (unsharp_mask/builder.py:58-82).

Input ``img`` is float32 [3][R+4][C+4] (planar, 2-pixel ghost zone, as
unsharp_mask/init.py:26-35 prepares it); output ``mask`` is float32
[3][R][C] (domain x, y in [2, R+1] x [2, C+1]; row/col R+1, C+1 are never
written):

  blurx = 5-tap [1,4,6,4,1]/16 along x (rows)     on x in [2,R], y in [1,C]
  blury = 5-tap [1,4,6,4,1]/16 along y (columns)  on x in [2,R], y in [2,C]
  sharpen = img*(1+weight) - blury*weight
  mask = |img - blury| < threshold ? img : sharpen
"""

from ..constructs import (Parameter, Variable, Interval, Image, Function,
                          Case, Condition, Select, Abs, Int, Float)
from ..compiler import buildPipeline


def unsharp_mask(pipe_data=None):
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    threshold = Parameter(Float, "threshold")
    weight = Parameter(Float, "weight")
    if pipe_data is not None:
        pipe_data.update(R=R, C=C, threshold=threshold, weight=weight)
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    c = Variable(Int, "c")
    img = Image(Float, "img", [3, R + 4, C + 4])
    cr = Interval(Int, 0, 2)
    xrow = Interval(Int, 2, R + 1)
    xcol = Interval(Int, 0, C + 3)
    yrow = Interval(Int, 2, R + 1)
    ycol = Interval(Int, 2, C + 1)
    inside = (Condition(x, '>=', 1) & Condition(x, '<=', R) &
              Condition(y, '<=', C) & Condition(y, '>=', 1))

    blurx = Function(([c, x, y], [cr, xrow, xcol]), Float, "blurx")
    blurx.defn = [Case(inside, (img(c, x - 2, y) +
                                img(c, x - 1, y) * 4.0 +
                                img(c, x, y) * 6.0 +
                                img(c, x + 1, y) * 4.0 +
                                img(c, x + 2, y)) * 0.0625)]
    blury = Function(([c, x, y], [cr, yrow, ycol]), Float, "blury")
    blury.defn = [Case(inside, (blurx(c, x, y - 2) +
                                blurx(c, x, y - 1) * 4.0 +
                                blurx(c, x, y) * 6.0 +
                                blurx(c, x, y + 1) * 4.0 +
                                blurx(c, x, y + 2)) * 0.0625)]
    sharpen = Function(([c, x, y], [cr, yrow, ycol]), Float, "sharpen")
    sharpen.defn = [Case(inside, img(c, x, y) * (1 + weight) -
                         blury(c, x, y) * weight)]
    masked = Function(([c, x, y], [cr, yrow, ycol]), Float, "mask")
    masked.defn = [Case(inside,
                        Select(Condition(Abs(img(c, x, y) - blury(c, x, y)),
                                         '<', threshold),
                               img(c, x, y), sharpen(c, x, y)))]
    return masked


def build_unsharp(rows=4096, cols=4096, tile_sizes=(32, 256), group_size=11,
                  options=(), name="unsharp"):
    """``rows``/``cols`` are the output sides (R, C)."""
    data = {}
    out = unsharp_mask(data)
    R, C = data['R'], data['C']
    return buildPipeline([out],
                         param_estimates=[(R, rows), (C, cols)],
                         param_constraints=[Condition(R, "==", rows),
                                            Condition(C, "==", cols)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size,
                         options=list(options),
                         pipe_name=name)
