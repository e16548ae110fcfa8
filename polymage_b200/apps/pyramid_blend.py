"""Laplacian pyramid blending, as specified by the reference app
(sandbox/apps/python/img_proc/pyramid_blend/polymage_blending.py:13-196)
and built with its settings (pyramid_blend/builder.py:63-67: tiles
[16, 256], group size 10).  The number of levels ``L`` is a parameter of
the spec builder (the reference fixes L = 4, :24).

Inputs ``img1``, ``img2`` float32 [3][R][C] and ``mask`` float32 [R][C]
(the reference driver pads the images by 60 pixels, 31 on the left:
pyramid_blend/init.py); output ``blend`` float32 [3][R-2m][C-2m] with
m = 2^(L+1) - 1 - (L-1)... i.e. domain [2^(L+1)-1, R/1 - 2^(L+1) + 2]
per side (for L = 4: [31, R-30]).

  Gaussian levels: 5-tap [1,4,6,4,1]/16 down-sampling by 2 along x then y
  Laplacian levels: level - upsampled(next level) (even/odd selects)
  blend: lap1 * m + lap2 * (1 - m) per level, then collapse
"""

from ..constructs import (Parameter, Variable, Interval, Image, Function,
                          Condition, Select, Int, Float)
from ..compiler import buildPipeline


def pyramid_blending(pipe_data=None, L=4):
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    c = Variable(Int, "c")
    if pipe_data is not None:
        pipe_data['R'] = R
        pipe_data['C'] = C
    img1 = Image(Float, "img1", [3, R, C])
    img2 = Image(Float, "img2", [3, R, C])
    mask = Image(Float, "mask", [R, C])
    cr = Interval(Int, 0, 2)

    # Gaussian pyramid (:42-89)
    def pyr_down(f, l, color, name):
        dec = 1 << l
        org = 1 << (l - 1)
        dec_rowr = Interval(Int, l, (R / dec) - 2)
        dec_colr = Interval(Int, l, (C / dec) - 2)
        colr = Interval(Int, l - 1, (C / org) - 2)

        def fx(k):
            return f(c, 2 * x + k, y) if color else f(2 * x + k, y)

        if color:
            downx = Function(([c, x, y], [cr, dec_rowr, colr]), Float,
                             "Dx_%d_%s" % (l, name))
        else:
            downx = Function(([x, y], [dec_rowr, colr]), Float,
                             "Dx_%d_%s" % (l, name))
        downx.defn = [(1 * fx(-2) + 4 * fx(-1) + 6 * fx(0) + 4 * fx(1) +
                       1 * fx(2)) * 0.0625]

        def dy(k):
            return downx(c, x, 2 * y + k) if color else downx(x, 2 * y + k)

        if color:
            downy = Function(([c, x, y], [cr, dec_rowr, dec_colr]), Float,
                             "Dy_%d_%s" % (l, name))
        else:
            downy = Function(([x, y], [dec_rowr, dec_colr]), Float,
                             "Dy_%d_%s" % (l, name))
        downy.defn = [(1 * dy(-2) + 4 * dy(-1) + 6 * dy(0) + 4 * dy(1) +
                       1 * dy(2)) * 0.0625]
        return downy

    g1 = {0: img1}
    g2 = {0: img2}
    gm = {0: mask}
    for l in range(1, L):
        g1[l] = pyr_down(g1[l - 1], l, True, "img1")
        g2[l] = pyr_down(g2[l - 1], l, True, "img2")
        gm[l] = pyr_down(gm[l - 1], l, False, "mask")

    def upsample(fd, f, l, name, sign, up_name):
        """f + sign * up(fd): even/odd selects of 3-tap [1,6,1]/8 and 2-tap
        [4,4]/8 interpolation along x then y (:91-136, :152-194)."""
        dec_colr = Interval(Int, (1 << (L - l)) - 1,
                            C / (1 << (l + 1)) - (1 << (L - l)) + 2)
        colr = Interval(Int, (1 << (L - l + 1)) - 1,
                        C / (1 << l) - (1 << (L - l + 1)) + 2)
        rowr = Interval(Int, (1 << (L - l + 1)) - 1,
                        R / (1 << l) - (1 << (L - l + 1)) + 2)
        upx = Function(([c, x, y], [cr, rowr, dec_colr]), Float, up_name)
        even_x = (1 * fd(c, (x / 2) - 1, y) + 6 * fd(c, (x / 2), y) +
                  1 * fd(c, (x / 2) + 1, y)) * 0.125
        odd_x = (4 * fd(c, (x - 1) / 2, y) + 4 * fd(c, (x + 1) / 2, y)) * \
            0.125
        upx.defn = [Select(Condition(x % 2, "==", 0), even_x, odd_x)]
        even_y = (1 * upx(c, x, (y / 2) - 1) + 6 * upx(c, x, (y / 2)) +
                  1 * upx(c, x, (y / 2) + 1)) * 0.125
        odd_y = (4 * upx(c, x, (y - 1) / 2) + 4 * upx(c, x, (y + 1) / 2)) * \
            0.125
        if sign < 0:
            e, o = f(c, x, y) - even_y, f(c, x, y) - odd_y
        else:
            e, o = f(c, x, y) + even_y, f(c, x, y) + odd_y
        upy = Function(([c, x, y], [cr, rowr, colr]), Float, name)
        upy.defn = [Select(Condition(y % 2, "==", 0), e, o)]
        return upy

    # Laplacian pyramids (:138-149)
    lap1 = {}
    lap2 = {}
    for l in range(0, L - 1):
        lap1[l] = upsample(g1[l + 1], g1[l], l, "Uy_%d_img1" % l, -1,
                           "Ux_%d_img1" % l)
        lap2[l] = upsample(g2[l + 1], g2[l], l, "Uy_%d_img2" % l, -1,
                           "Ux_%d_img2" % l)
    lap1[L - 1] = g1[L - 1]
    lap2[L - 1] = g2[L - 1]

    # blend each level (:138-150)
    res = {}
    for l in range(0, L):
        colr = Interval(Int, (1 << (L - l + 1)) - 1,
                        C / (1 << l) - (1 << (L - l + 1)) + 2)
        rowr = Interval(Int, (1 << (L - l + 1)) - 1,
                        R / (1 << l) - (1 << (L - l + 1)) + 2)
        f = Function(([c, x, y], [cr, rowr, colr]), Float, "Res_%d" % l)
        f.defn = [lap1[l](c, x, y) * gm[l](x, y) +
                  lap2[l](c, x, y) * (1 - gm[l](x, y))]
        res[l] = f

    # collapse (:152-194)
    out = {L - 1: res[L - 1]}
    for l in range(L - 2, 0, -1):
        out[l] = upsample(out[l + 1], res[l], l, "Col_%d" % l, +1,
                          "Col_%d_x" % l)
    out[0] = upsample(out[1], res[0], 0, "blend", +1, "blend_x")
    return out[0]


def build_pyramid(rows=2048 + 60, cols=2048 + 60, L=4, tile_sizes=(16, 256),
                  group_size=10, options=(), name="pyramid"):
    """``rows``/``cols`` are the padded image sides (R, C)."""
    data = {}
    out = pyramid_blending(data, L=L)
    R, C = data['R'], data['C']
    return buildPipeline([out],
                         param_estimates=[(R, rows), (C, cols)],
                         param_constraints=[Condition(R, "==", rows),
                                            Condition(C, "==", cols)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size,
                         options=list(options),
                         pipe_name=name)
