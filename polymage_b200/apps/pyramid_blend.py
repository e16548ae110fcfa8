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
                          Condition, Select, Max, Min, Int, Float)
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


def pyramid_blending_clamped(pipe_data=None, L=8):
    """Laplacian pyramid blending with ``L`` levels on images of any size:
    the reference's filters (5-tap [1,4,6,4,1]/16 decimation, [1,6,1]/8 and
    [4,4]/8 even/odd interpolation, per-level blend and collapse:
    polymage_blending.py:42-194) with indices clamped to each level's
    domain instead of the reference's shrinking interior margins, which at
    L = 8 leave no valid output below ~1100 pixels.  Level l has
    ceil(R / 2^l) x ceil(C / 2^l) points; the output ``blend`` is
    [3][R][C].  No counterpart in the reference: its oracle is the FP64
    restatement of this generalized spec (oracle/pyramid.py)."""
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
    rows = [R]
    cols = [C]
    for l in range(1, L):
        rows.append((R + (1 << l) - 1) / (1 << l))
        cols.append((C + (1 << l) - 1) / (1 << l))

    def clamp(v, n):
        return Min(Max(v, 0), n - 1)

    def ref(f, color, a, b):
        return f(c, a, b) if color else f(a, b)

    def dom(color, nr, nc):
        if color:
            return ([c, x, y], [cr, Interval(Int, 0, nr - 1),
                                Interval(Int, 0, nc - 1)])
        return ([x, y], [Interval(Int, 0, nr - 1), Interval(Int, 0, nc - 1)])

    def down(f, l, color, name):
        w = (1, 4, 6, 4, 1)
        dx = Function(dom(color, rows[l], cols[l - 1]), Float,
                      "Dx_%d_%s" % (l, name))
        dx.defn = [sum(w[k] * ref(f, color, clamp(2 * x + k - 2,
                                                   rows[l - 1]), y)
                       for k in range(5)) * 0.0625]
        dy = Function(dom(color, rows[l], cols[l]), Float,
                      "Dy_%d_%s" % (l, name))
        dy.defn = [sum(w[k] * ref(dx, color, x, clamp(2 * y + k - 2,
                                                       cols[l - 1]))
                       for k in range(5)) * 0.0625]
        return dy

    g1 = {0: img1}
    g2 = {0: img2}
    gm = {0: mask}
    for l in range(1, L):
        g1[l] = down(g1[l - 1], l, True, "img1")
        g2[l] = down(g2[l - 1], l, True, "img2")
        gm[l] = down(gm[l - 1], l, False, "mask")

    def up(fd, f, l, sign, name):
        """f + sign * (level l+1 ``fd`` interpolated to level l)."""
        upx = Function(dom(True, rows[l], cols[l + 1]), Float,
                       "%s_x" % name)
        h = x / 2
        even_x = (fd(c, clamp(h - 1, rows[l + 1]), y) + 6 * fd(c, h, y) +
                  fd(c, clamp(h + 1, rows[l + 1]), y)) * 0.125
        odd_x = (4 * fd(c, h, y) + 4 * fd(c, clamp(h + 1, rows[l + 1]),
                                           y)) * 0.125
        upx.defn = [Select(Condition(x % 2, "==", 0), even_x, odd_x)]
        k = y / 2
        even_y = (upx(c, x, clamp(k - 1, cols[l + 1])) + 6 * upx(c, x, k) +
                  upx(c, x, clamp(k + 1, cols[l + 1]))) * 0.125
        odd_y = (4 * upx(c, x, k) + 4 * upx(c, x, clamp(k + 1,
                                                          cols[l + 1]))) * \
            0.125
        if sign < 0:
            e, o = f(c, x, y) - even_y, f(c, x, y) - odd_y
        else:
            e, o = f(c, x, y) + even_y, f(c, x, y) + odd_y
        out = Function(dom(True, rows[l], cols[l]), Float, name)
        out.defn = [Select(Condition(y % 2, "==", 0), e, o)]
        return out

    lap1 = dict((l, up(g1[l + 1], g1[l], l, -1, "Lap_%d_img1" % l))
                for l in range(L - 1))
    lap2 = dict((l, up(g2[l + 1], g2[l], l, -1, "Lap_%d_img2" % l))
                for l in range(L - 1))
    lap1[L - 1] = g1[L - 1]
    lap2[L - 1] = g2[L - 1]
    res = {}
    for l in range(L):
        f = Function(dom(True, rows[l], cols[l]), Float, "Res_%d" % l)
        f.defn = [lap1[l](c, x, y) * gm[l](x, y) +
                  lap2[l](c, x, y) * (1 - gm[l](x, y))]
        res[l] = f
    out = res[L - 1]
    for l in range(L - 2, 0, -1):
        out = up(out, res[l], l, +1, "Col_%d" % l)
    return up(out, res[0], 0, +1, "blend")


def build_pyramid_clamped(rows=2048, cols=2048, L=8, tile_sizes=(32, 64),
                          group_size=10, options=('rblock=8',),
                          name="pyramid8"):
    """The generalized ``L``-level blend (any image size)."""
    data = {}
    out = pyramid_blending_clamped(data, L=L)
    R, C = data['R'], data['C']
    return buildPipeline([out],
                         param_estimates=[(R, rows), (C, cols)],
                         param_constraints=[Condition(R, "==", rows),
                                            Condition(C, "==", cols)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size,
                         options=list(options),
                         pipe_name=name)
