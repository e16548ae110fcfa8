"""Local Laplacian filter (Paris, Hasinoff and Kautz's edge-aware detail
manipulation, in the Halide formulation), with the semantics of the
reference's generated pipeline ``pipeline_laplacian``
(sandbox/video_demo/laplacian_polymage.cpp:10; the same stages, untiled, in
laplacian_naive.cpp).  The reference keeps only that generated C++ in its
tree; this module states the pipeline in the DSL.

ABI (laplacian_polymage.cpp:10, video_demo.py:128-147):
``pipeline_laplacian(int C, int R, float alpha, float beta, void*
img_colour, void* laplacian)``; ``R``/``C`` are the frame's sides plus 92
(the pipeline's total ghost zone), ``img_colour`` is the uint8 frame
[R-92][C-92][3] (B, G, R interleaved) and ``laplacian`` the uint8 result
of the same shape.  The video demo calls it with 4 intensity levels:
``alpha = 1/3``, ``beta = 1`` (video_demo.py:54-57).

Stages (``K = 4`` intensity levels, ``J = 5`` pyramid levels):

* ``img``: grey level 0.299 R + 0.587 G + 0.114 B over 255 (a double
  division, as the reference writes it), on the frame padded by 31 pixels
  on the top/left and 61 on the bottom/right with its edge values
  (laplacian_polymage.cpp:64-135: here indices clamped into the frame).
* ``remapLUT(i)``, i in [-768, 767]: alpha * (i/256) * exp(-(i/256)^2 / 2).
* ``gPyramid_L0(k, x, y)``: beta * (img - k/3) + k/3 + remapLUT(v - 256 k),
  v = clamp((int)(img * 768), 0, 768).
* Gaussian pyramids of every ``gPyramid`` level and of ``img``: a [1 3 3 1]
  / 8 decimation by 2 along x then y, levels 1..4 over [1, n/2^l - 2].
* Laplacian levels ``U_lPyramid_Ll = G_l - up(G_{l+1})`` with
  up(f)(x) = 0.25 f(x/2 - 1 + 2 (x%2)) + 0.75 f(x/2) along x, then y.
* ``outLPyramid_Ll``: the two Laplacian levels around the input's own
  intensity, li = clamp((int)(3 inG_l), 0, 2), blended linearly.
* Collapse ``outGPyramid_Ll = outLPyramid_Ll + up(outGPyramid_{l+1})``
  down to ``result_ref_gray`` at level 0.
* ``laplacian(x, y, c)`` = (uint8)(255 clamp(r (colour/256 + 0.01) /
  (img + 0.01), 0, 1)) with r the result at (x + 31, y + 31).

Domains shrink with the level as the reference's do: the collapse at
level l covers [2^(5-l) - 1, n/2^l - 2^(6-l) + 2] (level 4: [1, n/16 -
2]).  One deliberate difference: the LUT index of a pure-white pixel
(v = 768 with k = 0) is 768, one past the LUT, which the reference reads
out of bounds; here it reads entry 767 (data-dependent reads are clamped
into their domain).
"""

from ..constructs import (Parameter, Variable, Interval, Image, Function,
                          Condition, Select, Cast, Max, Min, Exp, Int, Float,
                          Double, UChar)
from ..expr_ast import Value
from ..compiler import buildPipeline

LEVELS = 4          # intensity levels (K)
J = 5               # pyramid levels
GHOST = 92          # total padding per dimension
OFF = 31            # padding before the frame


def local_laplacian(pipe_data=None):
    R = Parameter(Int, "R")
    C = Parameter(Int, "C")
    alpha = Parameter(Float, "alpha")
    beta = Parameter(Float, "beta")
    x = Variable(Int, "x")
    y = Variable(Int, "y")
    k = Variable(Int, "k")
    c = Variable(Int, "c")
    i = Variable(Int, "i")
    if pipe_data is not None:
        pipe_data['R'] = R
        pipe_data['C'] = C
    img_colour = Image(UChar, "img_colour", [R - GHOST, C - GHOST, 3])
    kr = Interval(Int, 0, LEVELS - 1)
    cr = Interval(Int, 0, 2)

    def n_r(l):
        return R if l == 0 else R / (1 << l)

    def n_c(l):
        return C if l == 0 else C / (1 << l)

    def gauss(n, l):
        return Interval(Int, 1, n(l) - 2)

    def inner(n, l):
        if l == J - 1:
            return Interval(Int, 1, n(l) - 2)
        return Interval(Int, (1 << (5 - l)) - 1, n(l) - (1 << (6 - l)) + 2)

    def up(f, v, args_at):
        """0.25 f(v/2 - 1 + 2 (v%2)) + 0.75 f(v/2) along one dimension;
        ``args_at(t)`` builds f's arguments with t at that dimension."""
        h = v / 2
        even = 0.25 * f(*args_at(h - 1)) + 0.75 * f(*args_at(h))
        odd = 0.25 * f(*args_at(h + 1)) + 0.75 * f(*args_at(h))
        return Select(Condition(v % 2, "==", 0), even, odd)

    # grey level of the edge-padded frame (laplacian_polymage.cpp:64-135)
    img = Function(([x, y], [Interval(Int, 0, R - 1), Interval(Int, 0, C - 1)]),
                   Float, "img")
    xc = Min(Max(x - OFF, 0), R - GHOST - 1)
    yc = Min(Max(y - OFF, 0), C - GHOST - 1)
    img.defn = [(0.299 * img_colour(xc, yc, 2) + 0.587 * img_colour(xc, yc, 1)
                 + 0.114 * img_colour(xc, yc, 0)) / Value(255.0, Double)]

    lut = Function(([i], [Interval(Int, -768, 767)]), Float, "remapLUT")
    fi = Cast(Float, i) / 256.0
    lut.defn = [(alpha * fi) * Exp(((-fi) * fi) / 2.0)]

    g0 = Function(([k, x, y], [kr, Interval(Int, 0, R - 1),
                               Interval(Int, 0, C - 1)]), Float,
                  "gPyramid_L0")
    v = Min(Max(Cast(Int, img(x, y) * 768.0), 0), 768)
    g0.defn = [(beta * (img(x, y) - k * 0.333333333333) +
                k * 0.333333333333) + lut(v - 256 * k)]

    def down(prev, l, name, levels):
        """[1 3 3 1]/8 decimation of level l-1 along x, then y."""
        lead = [k] if levels else []
        lr = [kr] if levels else []
        dx = Function((lead + [x, y], lr + [gauss(n_r, l),
                                            Interval(Int, 1, n_c(l - 1) - 2)]),
                      Float, "Dx_%s_L%d" % (name, l))

        def p(a, b):
            return prev(*(lead + [a, b]))
        dx.defn = [(p(2 * x - 1, y) + 3.0 * p(2 * x, y) +
                    3.0 * p(2 * x + 1, y) + p(2 * x + 2, y)) * 0.125]
        d = Function((lead + [x, y], lr + [gauss(n_r, l), gauss(n_c, l)]),
                     Float, "D_%s_L%d" % (name, l))

        def q(a, b):
            return dx(*(lead + [a, b]))
        d.defn = [(q(x, 2 * y - 1) + 3.0 * q(x, 2 * y) +
                   3.0 * q(x, 2 * y + 1) + q(x, 2 * y + 2)) * 0.125]
        return d

    gP = {0: g0}
    inG = {0: img}
    for l in range(1, J):
        gP[l] = down(gP[l - 1], l, "gPyramid", True)
        inG[l] = down(inG[l - 1], l, "inGPyramid", False)

    # Laplacian pyramid of every intensity level
    lP = {J - 1: gP[J - 1]}
    for l in range(J - 2, -1, -1):
        ux = Function(([k, x, y], [kr, inner(n_r, l), inner(n_c, l + 1)]),
                      Float, "Ux_lPyramid_L%d" % l)
        ux.defn = [up(gP[l + 1], x, lambda t: (k, t, y))]
        u = Function(([k, x, y], [kr, inner(n_r, l), inner(n_c, l)]), Float,
                     "U_lPyramid_L%d" % l)
        u.defn = [gP[l](k, x, y) - up(ux, y, lambda t: (k, x, t))]
        lP[l] = u

    # blend the two intensity levels around the input's own grey level
    outL = {}
    for l in range(J):
        f = Function(([x, y], [inner(n_r, l), inner(n_c, l)]), Float,
                     "outLPyramid_L%d" % l)
        g3 = inG[l](x, y) * 3.0
        li = Min(Max(Cast(Int, g3), 0), LEVELS - 2)
        f.defn = [(1.0 - (g3 - li)) * lP[l](li, x, y) +
                  (g3 - li) * lP[l](li + 1, x, y)]
        outL[l] = f

    # collapse
    outG = outL[J - 1]
    for l in range(J - 2, -1, -1):
        top = "result_ref_gray" if l == 0 else "outGPyramid_L%d" % l
        ux = Function(([x, y], [inner(n_r, l), inner(n_c, l + 1)]), Float,
                      "Ux_" + top)
        ux.defn = [up(outG, x, lambda t: (t, y))]
        g = Function(([x, y], [inner(n_r, l), inner(n_c, l)]), Float, top)
        g.defn = [outL[l](x, y) + up(ux, y, lambda t: (x, t))]
        outG = g

    out = Function(([x, y, c], [Interval(Int, 0, R - GHOST - 1),
                                Interval(Int, 0, C - GHOST - 1), cr]),
                   UChar, "laplacian")
    val = (outG(x + OFF, y + OFF) * (img_colour(x, y, c) / 256.0 + 0.01)) / \
        (img(x + OFF, y + OFF) + 0.01)
    out.defn = [Cast(UChar, Min(Max(val, 0.0), 1.0) * 255.0)]
    return out


def build_laplacian(rows=1080, cols=1920, tile_sizes=(32, 64),
                    group_size=10, options=('rblock=8',), name="laplacian"):
    """``rows``/``cols``: the frame's sides (the parameters are the padded
    sides, rows + 92 and cols + 92)."""
    data = {}
    out = local_laplacian(data)
    R, C = data['R'], data['C']
    return buildPipeline([out],
                         param_estimates=[(R, rows + GHOST),
                                          (C, cols + GHOST)],
                         param_constraints=[Condition(R, "==", rows + GHOST),
                                            Condition(C, "==", cols + GHOST)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size,
                         options=list(options),
                         pipe_name=name)
