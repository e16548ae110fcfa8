"""Harris corner detection, as specified by the reference app
(sandbox/apps/python/img_proc/harris/polymage_harris.py:13-78) and built with
its settings (harris/builder.py:49-84: estimates R=rows-2, C=cols-2,
group_size 11).

Input ``img`` is float32 [R+2][C+2]; output ``harris`` is float32
[R+2][C+2] with only [2..R-1] x [2..C-1] written:

  Ix, Iy   3x3 Sobel with weights 1/12, 2/12 on x in [1,R], y in [1,C]
  Ixx, Iyy, Ixy   products
  Sxx, Syy, Sxy   3x3 box sums on [2,R-1] x [2,C-1]
  harris = Sxx*Syy - Sxy^2 - 0.04 (Sxx+Syy)^2
"""

from ..constructs import (Parameter, Variable, Interval, Image, Function,
                          Case, Condition, Int, Float)
from ..compiler import buildPipeline


def harris_pipe(pipe_data=None):
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    if pipe_data is not None:
        pipe_data['R'] = R
        pipe_data['C'] = C
    row = Interval(Int, 0, R + 1)
    col = Interval(Int, 0, C + 1)
    inner = (Condition(x, '>=', 1) & Condition(x, '<=', R) &
             Condition(y, '<=', C) & Condition(y, '>=', 1))
    inner2 = (Condition(x, '>=', 2) & Condition(x, '<=', R - 1) &
              Condition(y, '<=', C - 1) & Condition(y, '>=', 2))
    img = Image(Float, "img", [R + 2, C + 2])

    def fn(name):
        return Function(([x, y], [row, col]), Float, name)

    Iy = fn("Iy")
    Iy.defn = [Case(inner,
                    img(x - 1, y - 1) * (-1.0 / 12) +
                    img(x - 1, y + 1) * (1.0 / 12) +
                    img(x, y - 1) * (-2.0 / 12) +
                    img(x, y + 1) * (2.0 / 12) +
                    img(x + 1, y - 1) * (-1.0 / 12) +
                    img(x + 1, y + 1) * (1.0 / 12))]
    Ix = fn("Ix")
    Ix.defn = [Case(inner,
                    img(x - 1, y - 1) * (-1.0 / 12) +
                    img(x + 1, y - 1) * (1.0 / 12) +
                    img(x - 1, y) * (-2.0 / 12) +
                    img(x + 1, y) * (2.0 / 12) +
                    img(x - 1, y + 1) * (-1.0 / 12) +
                    img(x + 1, y + 1) * (1.0 / 12))]
    Ixx = fn("Ixx")
    Ixx.defn = [Case(inner, Ix(x, y) * Ix(x, y))]
    Iyy = fn("Iyy")
    Iyy.defn = [Case(inner, Iy(x, y) * Iy(x, y))]
    Ixy = fn("Ixy")
    Ixy.defn = [Case(inner, Ix(x, y) * Iy(x, y))]

    def box3(f):
        return (f(x - 1, y - 1) + f(x - 1, y) + f(x - 1, y + 1) +
                f(x, y - 1) + f(x, y) + f(x, y + 1) +
                f(x + 1, y - 1) + f(x + 1, y) + f(x + 1, y + 1))

    Sxx = fn("Sxx")
    Sxx.defn = [Case(inner2, box3(Ixx))]
    Syy = fn("Syy")
    Syy.defn = [Case(inner2, box3(Iyy))]
    Sxy = fn("Sxy")
    Sxy.defn = [Case(inner2, box3(Ixy))]
    det = fn("det")
    det.defn = [Case(inner2, Sxx(x, y) * Syy(x, y) - Sxy(x, y) * Sxy(x, y))]
    trace = fn("trace")
    trace.defn = [Case(inner2, Sxx(x, y) + Syy(x, y))]
    harris = fn("harris")
    harris.defn = [Case(inner2, det(x, y) - 0.04 * trace(x, y) *
                        trace(x, y))]
    return harris


def build_harris(rows=2048, cols=2048, tile_sizes=(32, 256), group_size=11,
                 options=(), name="harris"):
    """``rows``/``cols`` are the full image sides (R = rows-2, C = cols-2)."""
    data = {}
    out = harris_pipe(data)
    R, C = data['R'], data['C']
    return buildPipeline([out],
                         param_estimates=[(R, rows - 2), (C, cols - 2)],
                         param_constraints=[Condition(R, "==", rows - 2),
                                            Condition(C, "==", cols - 2)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size,
                         options=list(options),
                         pipe_name=name)
