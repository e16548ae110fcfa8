"""Pyramid interpolation of an image with an alpha channel (fills pixels of
low alpha from coarser levels), as specified by the reference app
(sandbox/apps/python/img_proc/interpolate/polymage_interpolate.py:14-189)
with its build settings (interpolate/builder.py:59-82: tiles 16x16, group
size 11).

Input ``img`` is float32 [4][R+2][C+2] (R, G, B, alpha in [0, 1] with a
one-pixel ghost border, interpolate/init.py:29-40); output ``interpolate``
is float32 [3][R][C].  Ten levels:

* ``downsampled_L0 = img * alpha`` (premultiplied);
* down: a [1 2 1]/4 filter and decimation along x, then y, on
  [1, n/2^l] with zero borders (:39-85);
* up: ``Ux`` averages rows (x+1)/2 and (x+2)/2 of the coarser level,
  then along y; ``interpolated_Ll = D_l + (1 - alpha_l) * up`` with zero
  borders (:87-149);
* ``interpolate = interpolated_L0[c] / interpolated_L0[alpha]`` on the
  interior (:163-169).
"""

from ..constructs import (Parameter, Variable, Interval, Image, Function,
                          Case, Condition, Int, Float)
from ..compiler import buildPipeline

LEVELS = 10


def interpolate(pipe_data=None, L=LEVELS):
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    if pipe_data is not None:
        pipe_data['R'] = R
        pipe_data['C'] = C
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    c = Variable(Int, "c")
    img = Image(Float, "img", [4, R + 2, C + 2])
    rgba = Interval(Int, 0, 3)
    rgb = Interval(Int, 0, 2)

    def box(xhi, yhi):
        return (Condition(x, '>=', 1) & Condition(x, '<=', xhi) &
                Condition(y, '>=', 1) & Condition(y, '<=', yhi))

    def borders(xhi, yhi):
        """The zero cases outside the interior box (left, right, top,
        bottom), as the reference lists them."""
        return [Case(Condition(y, '<=', 0), 0),
                Case(Condition(y, '>=', yhi + 1), 0),
                Case(Condition(x, '>=', xhi + 1), 0),
                Case(Condition(x, '<=', 0), 0)]

    def down(f, l, name):
        rd, cd, co = R / (1 << l), C / (1 << l), C / (1 << (l - 1))
        dx = Function(([c, x, y], [rgba, Interval(Int, 0, rd + 1),
                                   Interval(Int, 0, co + 1)]), Float,
                      "Dx_%d_%s" % (l, name))
        dx.defn = [Case(box(rd, co), (f(c, 2 * x - 2, y) +
                                      f(c, 2 * x - 1, y) * 2.0 +
                                      f(c, 2 * x, y)) * 0.25)] + \
            borders(rd, co)
        d = Function(([c, x, y], [rgba, Interval(Int, 0, rd + 1),
                                  Interval(Int, 0, cd + 1)]), Float,
                     "D_%d_%s" % (l, name))
        d.defn = [Case(box(rd, cd), (dx(c, x, 2 * y - 2) +
                                     dx(c, x, 2 * y - 1) * 2.0 +
                                     dx(c, x, 2 * y)) * 0.25)] + \
            borders(rd, cd)
        return d

    def up(f, dl, l, name):
        ro, co, cd = R / (1 << l), C / (1 << l), C / (1 << (l + 1))
        ux = Function(([c, x, y], [rgba, Interval(Int, 0, ro + 1),
                                   Interval(Int, 0, cd + 1)]), Float,
                      "Ux_" + name)
        ux.defn = [Case(box(ro, cd), (f(c, (x + 1) / 2, y) +
                                      f(c, (x + 2) / 2, y)) / 2.0)] + \
            borders(ro, cd)
        upy = (ux(c, x, (y + 1) / 2) + ux(c, x, (y + 2) / 2)) / 2.0
        out = Function(([c, x, y], [rgba, Interval(Int, 0, ro + 1),
                                    Interval(Int, 0, co + 1)]), Float, name)
        out.defn = [Case(box(ro, co), dl(c, x, y) +
                         (1.0 - dl(3, x, y)) * upy)] + borders(ro, co)
        return out

    ds = {}
    ds[0] = Function(([c, x, y], [rgba, Interval(Int, 0, R + 1),
                                  Interval(Int, 0, C + 1)]), Float,
                     "downsampled_L0")
    ds[0].defn = [img(c, x, y) * img(3, x, y)]
    for l in range(1, L):
        ds[l] = down(ds[l - 1], l, "downsampled")
    it = ds[L - 1]
    for l in range(L - 2, -1, -1):
        it = up(it, ds[l], l, "interpolated_L%d" % l)
    out = Function(([c, x, y], [rgb, Interval(Int, 0, R - 1),
                                Interval(Int, 0, C - 1)]), Float,
                   "interpolate")
    out.defn = [it(c, x + 1, y + 1) / it(3, x + 1, y + 1)]
    return out


def build_interpolate(rows=2048, cols=2048, tile_sizes=(16, 16),
                      group_size=11, options=(), name="interpolate"):
    data = {}
    out = interpolate(data)
    R, C = data['R'], data['C']
    return buildPipeline([out],
                         param_estimates=[(R, rows), (C, cols)],
                         param_constraints=[Condition(R, "==", rows),
                                            Condition(C, "==", cols)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size,
                         options=list(options),
                         pipe_name=name)
