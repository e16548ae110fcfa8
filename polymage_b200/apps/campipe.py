"""Camera raw pipeline, as specified by the reference app
(sandbox/apps/python/img_proc/campipe/polymage_campipe.py:13-304) and built
with its settings (campipe/builder.py:53-82: tiles [64, 256], group size 5).

Input ``img`` is int16 [R][C] (a GRBG Bayer raw, values 0..1023 in the
benchmark); ``matrix_3200``/``matrix_7000`` are float32 [3][4]
(campipe/init.py:26-40); output ``process`` is uint8 [3][R-48][C-64]
(domain x in [12, R-37], y in [16, C-49]); parameter order in the C ABI is
``C, R, colour_temp, contrast, gamma`` (campipe/exec_pipe.py:33-42).

Stages: hot-pixel suppression (clamp to the min/max of the +-2 same-colour
neighbours), deinterleave into 4 planes, Halide-style demosaic in integer
arithmetic with truncating /2, re-interleave, a 3x4 colour matrix (a const
Int function, Q8.8 from colour_temp), and a const uint8 curve LUT over the
int16 range.  Channel order: c=2 red, c=1 green, c=0 blue (:254-262).
"""

from ..constructs import (Parameter, Variable, Interval, Image, Function,
                          Case, Condition, Select, Cast, Max, Min, Powf, Int,
                          Float, Short, UChar)
from ..compiler import buildPipeline

# The app's colour-correction matrices at 3200 K and 7000 K (campipe/
# init.py:26-40), rows r, g, b of [3x3 | offset]: benchmark inputs.
MATRIX_3200 = ((1.6697, -0.2693, -0.4004, -42.4346),
               (-0.3576, 1.0615, 1.5949, -37.1158),
               (-0.2175, -1.8751, 6.9640, -26.6970))
MATRIX_7000 = ((2.2997, -0.4478, 0.1706, -39.0923),
               (-0.3826, 1.5906, -0.2080, -25.4311),
               (-0.0888, -0.7344, 2.2832, -20.0826))


def camera_pipe(pipe_data=None):
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    c = Variable(Int, "c")
    v = Variable(Int, "v")
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    kelvin = Parameter(Float, "colour_temp")
    gamma = Parameter(Float, "gamma")
    contrast = Parameter(Float, "contrast")
    if pipe_data is not None:
        pipe_data['R'] = R
        pipe_data['C'] = C

    gx, gy = 12, 16      # ghost zone per dimension
    # intervals (:41-62)
    ghost_zone_2x = Interval(Int, gx - 4, (R - 24 - gx + 6) - 1)
    ghost_zone_2y = Interval(Int, gy - 4, (C - 32 - gy + 6) - 1)
    ghost_zone_0x = Interval(Int, gx, (R - 24 - gx) - 1)
    ghost_zone_0y = Interval(Int, gy, (C - 32 - gy) - 1)
    half_2x = Interval(Int, gx // 2 - 2, (R - 24 - gx) // 2 + 2)
    half_2y = Interval(Int, gy // 2 - 2, (C - 32 - gy) // 2 + 2)
    half_1x = Interval(Int, gx // 2 - 1, (R - 24 - gx) // 2 + 1)
    half_1y = Interval(Int, gy // 2 - 1, (C - 32 - gy) // 2 + 1)
    half_0x = Interval(Int, gx // 2, (R - 24 - gx) // 2)
    half_0y = Interval(Int, gy // 2, (C - 32 - gy) // 2)
    rgb = Interval(Int, 0, 2)
    grbg = Interval(Int, 0, 3)
    lut_range = Interval(Int, -32768, 32767)

    matrix_3200 = Image(Float, "matrix_3200", [3, 4])
    matrix_7000 = Image(Float, "matrix_7000", [3, 4])
    img = Image(Short, "img", [R, C])

    # 1. hot-pixel suppression (:72-83)
    x_max = Max(img(x - 2, y), img(x + 2, y))
    y_max = Max(img(x, y - 2), img(x, y + 2))
    x_min = Min(img(x - 2, y), img(x + 2, y))
    y_min = Min(img(x, y - 2), img(x, y + 2))
    # clamp img into [min of neighbours, max of neighbours]
    clamp = Max(Min(x_min, y_min), Min(Max(x_max, y_max), img(x, y)))
    denoised = Function(([x, y], [ghost_zone_2x, ghost_zone_2y]), Short,
                        "denoised")
    denoised.defn = [clamp]

    # 2. deinterleave (:86-92)
    deinterleaved = Function(([c, x, y], [grbg, half_2x, half_2y]), Short,
                             "deinterleaved")
    deinterleaved.defn = [
        Case(Condition(c, '==', 0), denoised(2 * x, 2 * y)),
        Case(Condition(c, '==', 1), denoised(2 * x, 2 * y + 1)),
        Case(Condition(c, '==', 2), denoised(2 * x + 1, 2 * y)),
        Case(Condition(c, '==', 3), denoised(2 * x + 1, 2 * y + 1))]

    # 3. demosaic (:103-212)
    def plane(name, k):
        f = Function(([x, y], [half_2x, half_2y]), Short, name)
        f.defn = [deinterleaved(k, x, y)]
        return f
    g_gr = plane("g_gr", 0)
    r_r = plane("r_r", 1)
    b_b = plane("b_b", 2)
    g_gb = plane("g_gb", 3)

    def absd(a, b):
        return Select(Condition(a, '>', b), a - b, b - a)

    g_r = Function(([x, y], [half_1x, half_1y]), Short, "g_r")
    gv_r = (g_gb(x - 1, y) + g_gb(x, y)) / 2
    gvd_r = absd(g_gb(x - 1, y), g_gb(x, y))
    gh_r = (g_gr(x, y + 1) + g_gr(x, y)) / 2
    ghd_r = absd(g_gr(x, y + 1), g_gr(x, y))
    g_r.defn = [Select(Condition(ghd_r, '<', gvd_r), gh_r, gv_r)]

    g_b = Function(([x, y], [half_1x, half_1y]), Short, "g_b")
    gv_b = (g_gr(x + 1, y) + g_gr(x, y)) / 2
    gvd_b = absd(g_gr(x + 1, y), g_gr(x, y))
    gh_b = (g_gb(x, y - 1) + g_gb(x, y)) / 2
    ghd_b = absd(g_gb(x, y - 1), g_gb(x, y))
    g_b.defn = [Select(Condition(ghd_b, '<', gvd_b), gh_b, gv_b)]

    def at_green(name, gg, gsum, csum):
        f = Function(([x, y], [half_0x, half_0y]), Short, name)
        f.defn = [gg - gsum / 2 + csum / 2]
        return f
    r_gr = at_green("r_gr", g_gr(x, y), g_r(x, y) + g_r(x, y - 1),
                    r_r(x, y - 1) + r_r(x, y))
    b_gr = at_green("b_gr", g_gr(x, y), g_b(x, y) + g_b(x - 1, y),
                    b_b(x, y) + b_b(x - 1, y))
    r_gb = at_green("r_gb", g_gb(x, y), g_r(x, y) + g_r(x + 1, y),
                    r_r(x, y) + r_r(x + 1, y))
    b_gb = at_green("b_gb", g_gb(x, y), g_b(x, y) + g_b(x, y + 1),
                    b_b(x, y) + b_b(x, y + 1))

    corr = g_b(x, y) - (g_r(x, y) + g_r(x + 1, y - 1)) / 2
    rp_b = corr + (r_r(x, y) + r_r(x + 1, y - 1)) / 2
    rpd_b = absd(r_r(x, y), r_r(x + 1, y - 1))
    corr = g_b(x, y) - (g_r(x, y - 1) + g_r(x + 1, y)) / 2
    rn_b = corr + (r_r(x, y - 1) + r_r(x + 1, y)) / 2
    rnd_b = absd(r_r(x, y - 1), r_r(x + 1, y))
    r_b = Function(([x, y], [half_0x, half_0y]), Short, "r_b")
    r_b.defn = [Select(Condition(rpd_b, '<', rnd_b), rp_b, rn_b)]

    corr = g_r(x, y) - (g_b(x, y) + g_b(x - 1, y + 1)) / 2
    bp_r = corr + (b_b(x, y) + b_b(x - 1, y + 1)) / 2
    bpd_r = absd(b_b(x, y), b_b(x - 1, y + 1))
    corr = g_r(x, y) - (g_b(x, y + 1) + g_b(x - 1, y)) / 2
    bn_r = corr + (b_b(x, y + 1) + b_b(x - 1, y)) / 2
    bnd_r = absd(b_b(x, y + 1), b_b(x - 1, y))
    b_r = Function(([x, y], [half_0x, half_0y]), Short, "b_r")
    b_r.defn = [Select(Condition(bpd_r, '<', bnd_r), bp_r, bn_r)]

    # 4. re-interleave (:215-235)
    def interleave_x(a, b, name):
        out = Function(([x, y], [ghost_zone_0x, ghost_zone_0y]), Short, name)
        out.defn = [Select(Condition(x % 2, '==', 0), a(x / 2, y),
                           b(x / 2, y))]
        return out

    def interleave_y(a, b, name):
        out = Function(([x, y], [half_0x, ghost_zone_0y]), Short, name)
        out.defn = [Select(Condition(y % 2, '==', 0), a(x, y / 2),
                           b(x, y / 2))]
        return out

    red = interleave_x(interleave_y(r_gr, r_r, "red_x1"),
                       interleave_y(r_b, r_gb, "red_x2"), "red")(x, y)
    green = interleave_x(interleave_y(g_gr, g_r, "green_x1"),
                         interleave_y(g_b, g_gb, "green_x2"), "green")(x, y)
    blue = interleave_x(interleave_y(b_gr, b_r, "blue_x1"),
                        interleave_y(b_b, b_gb, "blue_x2"), "blue")(x, y)

    # 5. colour correction (:243-262)
    alpha = (1.0 / kelvin - 1.0 / 3200) / (1.0 / 7000 - 1.0 / 3200)
    mat = Function(([x, y], [rgb, grbg]), Int, "matrix", "const")
    val = matrix_3200(x, y) * alpha + matrix_7000(x, y) * (1 - alpha)
    mat.defn = [Cast(Int, val * 256.0)]
    r = mat(0, 3) + mat(0, 0) * red + mat(0, 1) * green + mat(0, 2) * blue
    g = mat(1, 3) + mat(1, 0) * red + mat(1, 1) * green + mat(1, 2) * blue
    b = mat(2, 3) + mat(2, 0) * red + mat(2, 1) * green + mat(2, 2) * blue
    corrected = Function(([c, x, y], [rgb, ghost_zone_0x, ghost_zone_0y]),
                         Short, "corrected")
    corrected.defn = [Case(Condition(c, '==', 2), r / 256),
                      Case(Condition(c, '==', 1), g / 256),
                      Case(Condition(c, '==', 0), b / 256)]

    # 6. tone curve LUT (:269-300)
    def lut_value(anything):
        xf = Cast(Float, anything / 1024.0)
        xf = Min(1.0, xf)
        xf = Max(0.0, xf)
        gg = Powf(xf, 1.0 / gamma)
        bb = 2.0 - Powf(2.0, contrast / 100.0)
        aa = 2.0 - 2.0 * bb
        z = Select(Condition(gg, '>', 0.5),
                   1.0 - (aa * (1.0 - gg) * (1.0 - gg) + bb * (1.0 - gg)),
                   aa * gg * gg + bb * gg)
        return Cast(UChar, Min(Max(z * 256.0, 0.0), 255.0))

    curve = Function(([v], [lut_range]), UChar, "curveLUT", "const")
    curve.defn = [lut_value(v)]
    curved = Function(([c, x, y], [rgb, ghost_zone_0x, ghost_zone_0y]),
                      UChar, "process")
    curved.defn = [curve(corrected(c, x, y))]
    return curved


def build_campipe(rows=1968, cols=2592, tile_sizes=(64, 256), group_size=5,
                  options=(), name="campipe"):
    """``rows``/``cols`` are the raw image sides (R, C)."""
    data = {}
    out = camera_pipe(data)
    R, C = data['R'], data['C']
    return buildPipeline([out],
                         param_estimates=[(R, rows), (C, cols)],
                         param_constraints=[Condition(R, "==", rows),
                                            Condition(C, "==", cols)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size,
                         options=list(options),
                         pipe_name=name)
