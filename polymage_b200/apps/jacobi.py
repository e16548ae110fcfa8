"""Weighted Jacobi smoothing of the 2-D Poisson problem, T steps, as
specified by the reference's stencil app
(sandbox/apps/python/stencil/jacobi2D/polymage_jacobi.py:8-60 with
polymage_common.py:16-75) and built with its settings
(jacobi2D/builder.py:53-76: tiles 16x64; group size 1 there, any here).

Inputs ``V_`` (the initial iterate) and ``F_`` (the right-hand side) are
float64 [N+2][N+2]; each step updates the interior [1, N]^2:

    W = U - c ((4 U - U(y-1) - U(y+1) - U(x-1) - U(x+1)) / h^2 - F)

with h = 1/(N+1), c = omega h^2 / 4, omega = 4/5 (double precision, as
the reference's unsuffixed literals are).  The boundary ring of each step
is not written by the spec; the steps after the first read it as 0 (the
oracle's convention for uncomputed points).  The output is the last step,
``jacobi``.  The steps are separate functions, so fusing groups of them
with overlapped tiles tiles the time loop.
"""

from ..constructs import (Parameter, Variable, Interval, Image, Function,
                          Case, Condition, Int, Double)
from ..expr_ast import Value
from ..compiler import buildPipeline


def jacobi2d(pipe_data=None, T=4):
    N = Parameter(Int, "N")
    y = Variable(Int, "y")
    x = Variable(Int, "x")
    if pipe_data is not None:
        pipe_data['N'] = N
    one = Value(1.0, Double)
    h = one / (N + 1)
    invhh = one / (h * h)
    c = Value(4.0 / 5.0, Double) * ((h * h) / Value(4.0, Double))
    extent = Interval(Int, 0, N + 1)
    inner = (Condition(y, ">=", 1) & Condition(y, "<=", N) &
             Condition(x, ">=", 1) & Condition(x, "<=", N))
    V = Image(Double, "V_", [N + 2, N + 2])
    F = Image(Double, "F_", [N + 2, N + 2])
    four = Value(4.0, Double)
    u = V
    for t in range(1, T + 1):
        w = Function(([y, x], [extent, extent]), Double,
                     "jacobi" if t == T else "jacobi_%d" % t)
        w.defn = [Case(inner, u(y, x) - c * ((u(y, x) * four -
                                             u(y - 1, x) - u(y + 1, x) -
                                             u(y, x - 1) - u(y, x + 1)) *
                                            invhh - F(y, x)))]
        u = w
    return u


def build_jacobi2d(N=4094, T=4, tile_sizes=(16, 64), group_size=4,
                   options=(), name="jacobi2d"):
    data = {}
    out = jacobi2d(data, T=T)
    Np = data['N']
    return buildPipeline([out], param_estimates=[(Np, N)],
                         param_constraints=[Condition(Np, "==", N)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size, options=list(options),
                         pipe_name=name)


def jacobi3d(pipe_data=None, T=2):
    """The 3-D variant (stencil/jacobi3D/polymage_jacobi.py:8-60,
    polymage_common.py:30-43): 7-point Laplacian, omega = 8/9,
    c = omega h^2 / 6, on [N+2]^3 float64 arrays."""
    N = Parameter(Int, "N")
    z = Variable(Int, "z")
    y = Variable(Int, "y")
    x = Variable(Int, "x")
    if pipe_data is not None:
        pipe_data['N'] = N
    one = Value(1.0, Double)
    h = one / (N + 1)
    invhh = one / (h * h)
    c = Value(8.0 / 9.0, Double) * ((h * h) / Value(6.0, Double))
    extent = Interval(Int, 0, N + 1)
    inner = (Condition(z, ">=", 1) & Condition(z, "<=", N) &
             Condition(y, ">=", 1) & Condition(y, "<=", N) &
             Condition(x, ">=", 1) & Condition(x, "<=", N))
    V = Image(Double, "V_", [N + 2, N + 2, N + 2])
    F = Image(Double, "F_", [N + 2, N + 2, N + 2])
    six = Value(6.0, Double)
    u = V
    for t in range(1, T + 1):
        w = Function(([z, y, x], [extent, extent, extent]), Double,
                     "jacobi" if t == T else "jacobi_%d" % t)
        w.defn = [Case(inner, u(z, y, x) - c * (
            (u(z, y, x) * six - u(z - 1, y, x) - u(z + 1, y, x) -
             u(z, y - 1, x) - u(z, y + 1, x) - u(z, y, x - 1) -
             u(z, y, x + 1)) * invhh - F(z, y, x)))]
        u = w
    return u


def build_jacobi3d(N=254, T=2, tile_sizes=(16, 16, 64), group_size=2,
                   options=(), name="jacobi3d"):
    data = {}
    out = jacobi3d(data, T=T)
    Np = data['N']
    return buildPipeline([out], param_estimates=[(Np, N)],
                         param_constraints=[Condition(Np, "==", N)],
                         tile_sizes=list(tile_sizes),
                         group_size=group_size, options=list(options),
                         pipe_name=name)
