"""Bilateral grid, as specified by the reference app
(sandbox/apps/python/img_proc/bilateral_grid/polymage_bilateral_grid.py:
16-130) and built with its settings (bilateral_grid/builder.py:53-80: tiles
[16, 16, 16], group size 5).

Input ``input`` is float32 [rows][cols]; output ``filtered`` is float32
[1][rows][cols]; parameter order in the C ABI is ``cols, rows``
(bilateral_grid/exec_pipe.py:26-30).  sigma_s = 8, sigma_r = 0.1:

  grid(c, x, y, z)   Reduction over every pixel: value (c=0) and weight
                     (c=1) splatted into cell (2+x/8, 2+y/8, 2+(int)(img*10))
  blurz, blurx, blury   unnormalised 5-tap [1,4,6,4,1] along z, x, y on the
                     grid interior
  interpolated(c,x,y)  trilinear slice of blury at the pixel
  filtered = interp(1) > 0 ? interp(0)/interp(1) : img
"""

from ..constructs import (Parameter, Variable, Interval, Image, Function,
                          Reduction, Reduce, Op, Case, Condition, Select,
                          Cast, Int, Float)
from ..compiler import buildPipeline


def bilateral_grid(pipe_data=None):
    rows = Parameter(Int, "rows")
    cols = Parameter(Int, "cols")
    if pipe_data is not None:
        pipe_data['R'] = rows
        pipe_data['C'] = cols
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    z = Variable(Int, "z")
    c = Variable(Int, "c")
    rowr = Interval(Int, 0, rows - 1)
    colr = Interval(Int, 0, cols - 1)
    img = Image(Float, "input", [rows, cols])
    inv_sigma_r = 10
    sigma_s = 8
    gridrowr = Interval(Int, 0, rows / sigma_s + 3)
    gridcolr = Interval(Int, 0, cols / sigma_s + 3)
    gridintr = Interval(Int, 0, inv_sigma_r + 3)
    cr = Interval(Int, 0, 1)
    cd = Interval(Int, 0, 0)

    grid = Reduction(([c, x, y, z], [cr, gridrowr, gridcolr, gridintr]),
                     ([x, y], [rowr, colr]), Float, "grid")
    zbin = Cast(Int, img(x, y) * inv_sigma_r)
    cell = [2 + x / sigma_s, 2 + y / sigma_s, 2 + zbin]
    grid.defn = [Case(Condition(c, '==', 0),
                      Reduce(grid(0, *cell), img(x, y), Op.Sum)),
                 Case(Condition(c, '==', 1),
                      Reduce(grid(1, *cell), 1, Op.Sum))]
    grid.default = 0

    interior = (Condition(x, '>=', 2) & Condition(x, '<=', rows / sigma_s + 1)
                & Condition(y, '>=', 2) &
                Condition(y, '<=', cols / sigma_s + 1) &
                Condition(z, '>=', 2) & Condition(z, '<=', inv_sigma_r + 1))
    dom4 = ([c, x, y, z], [cr, gridrowr, gridcolr, gridintr])

    def blur(src, name, axis):
        def at(k):
            idx = [c, x, y, z]
            idx[axis] = idx[axis] + k
            return src(*idx)
        f = Function(dom4, Float, name)
        f.defn = [Case(interior, at(-2) + at(-1) * 4 + at(0) * 6 +
                       at(1) * 4 + at(2))]
        return f

    blurz = blur(grid, "blurz", 3)
    blurx = blur(blurz, "blurx", 1)
    blury = blur(blurx, "blury", 2)

    zv = img(x, y) * inv_sigma_r
    zi = Cast(Int, zv)
    zf = zv - zi
    xf = Cast(Float, x % sigma_s) / sigma_s
    yf = Cast(Float, y % sigma_s) / sigma_s
    xi = x / sigma_s
    yi = y / sigma_s

    def lerp(a, b, w):
        return a + w * (b - a)

    def g(dx, dy, dz):
        return blury(c, 2 + xi + dx, 2 + yi + dy, 2 + zi + dz)

    z0 = lerp(lerp(g(0, 0, 0), g(1, 0, 0), xf),
              lerp(g(0, 1, 0), g(1, 1, 0), xf), yf)
    z1 = lerp(lerp(g(0, 0, 1), g(1, 0, 1), xf),
              lerp(g(0, 1, 1), g(1, 1, 1), xf), yf)
    interpolated = Function(([c, x, y], [cr, rowr, colr]), Float,
                            "interpolated")
    interpolated.defn = [lerp(z0, z1, zf)]

    filtered = Function(([c, x, y], [cd, rowr, colr]), Float, "filtered")
    filtered.defn = [Select(Condition(interpolated(1, x, y), '>', 0),
                            interpolated(0, x, y) / interpolated(1, x, y),
                            img(x, y))]
    return filtered


def build_bilateral(rows=1536, cols=2560, tile_sizes=(16, 16, 16),
                    group_size=5, options=(), name="bilateral"):
    data = {}
    out = bilateral_grid(data)
    R, C = data['R'], data['C']
    return buildPipeline([out],
                         param_estimates=[(R, rows), (C, cols)],
                         param_constraints=[Condition(R, "==", rows),
                                            Condition(C, "==", cols)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size,
                         options=list(options),
                         pipe_name=name)
