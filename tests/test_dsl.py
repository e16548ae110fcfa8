"""The PolyMage language front end, with the behaviour the reference's own
unit tests pin (sandbox/tests/test_constructs.py, test_expression.py,
test_expression_simplify.py, test_stencil.py)."""

from fractions import Fraction

import pytest

from polymage_b200.constructs import *   # noqa: F401,F403
from polymage_b200.expression import (isAffine, get_affine_var_and_param_coeff,
                                      get_constant_from_expr, simplify_expr)

D = Parameter(Int, "D")
R = Parameter(Int, "R")
C = Parameter(Int, "C")
z = Variable(Int, "z")
y = Variable(Int, "y")
x = Variable(Int, "x")


def test_constructs_basics():
    p = Parameter(Int, "n")
    v = Variable(Float, "v")
    assert p.name == "n" and p.typ is Int
    assert v.name == "v" and v.typ is Float
    iv = Interval(Int, 0, p - 1)
    assert str(iv.lowerBound) == "0"
    assert str(iv.upperBound) == "(n - 1)"
    assert iv.typ is Int
    val = Value(5, Int)
    assert val.value == 5 and val.typ is Int


def test_expression_affine():
    assert isAffine(x + 2 * y - 3)
    assert isAffine(x / 2)
    assert not isAffine(x * y)
    assert not isAffine(x % 2)
    assert isAffine(x % 2, include_modulo=True)
    c = get_affine_var_and_param_coeff(3 * x - y + R)
    assert c[x] == 3 and c[y] == -1 and c[R] == 1
    c = get_affine_var_and_param_coeff((x + 1) / 2)
    assert c[x] == Fraction(1, 2)
    assert get_constant_from_expr(x + 7 - 2) == 5


def test_expression_simplify():
    e = simplify_expr((x + 1) + (x - 3) + 2 * y)
    c = get_affine_var_and_param_coeff(e)
    assert c[x] == 2 and c[y] == 2
    assert get_constant_from_expr(e) == -2


def test_operator_shortcuts():
    assert (x + 0) is x and (x * 1) is x and (x - 0) is x
    assert isinstance(x * 0, Value) and (x * 0).value == 0
    assert str(0 - x) == "-(x)"
    assert str(x / 2) == "(x / 2)" and str(x // 2) == "(x / 2)"


def test_stencil_macro_expansion_strings():
    xrow = Interval(Int, 1, R)
    xcol = Interval(Int, 1, C)
    bounds = (Condition(x, '>=', 2) & Condition(x, '<=', R - 2) &
              Condition(y, '>=', 2) & Condition(y, '<=', C - 2))
    img = Image(Float, "input", [R + 2, C + 2])
    k1 = [[1, 0, 0], [0, 2, 0], [0, 0, 1]]
    s1 = Stencil(img, [x, y], k1)
    f1 = Function(([x, y], [xrow, xcol]), Float, "f1")
    f1.defn = [Case(bounds, s1)]
    assert s1.sizes == [3, 3] and s1.origin == [1, 1]
    assert str(Stencil.macro_expand(s1)) == \
        '((input((x + -1), (y + -1)) + (input(x, y) * 2)) + ' \
        'input((x + 1), (y + 1)))'
    k2 = [[-1, 2, -3.8], [0, -1, 0]]
    s2 = Stencil(f1, [x, y], k2)
    assert s2.sizes == [2, 3] and s2.origin == [0, 1]
    assert str(Stencil.macro_expand(s2)) == \
        '((((f1(x, (y + -1)) * -1) + (f1(x, y) * 2)) + ' \
        '(f1(x, (y + 1)) * -3.8)) + (f1((x + 1), y) * -1))'


def test_stencil_3d_origin_and_expansion():
    grid = Image(Float, "grid", [D, R, C])
    k = [[[1, 2], [2, 1]], [[2, 1], [1, 2]]]
    s = Stencil(grid, [x, y, z], k, _origin=[1, 1, 1])
    assert s.sizes == [2, 2, 2] and s.origin == [1, 1, 1]
    assert str(Stencil.macro_expand(s)) == \
        '((((((' \
        '(grid((x + -1), (y + -1), (z + -1)) + ' \
        '(grid((x + -1), (y + -1), z) * 2)) + ' \
        '(grid((x + -1), y, (z + -1)) * 2)) + ' \
        'grid((x + -1), y, z)) + ' \
        '(grid(x, (y + -1), (z + -1)) * 2)) + ' \
        'grid(x, (y + -1), z)) + ' \
        'grid(x, y, (z + -1))) + ' \
        '(grid(x, y, z) * 2))'


def test_invalid_stencil_kernel():
    img = Image(Float, "input", [R, C])
    with pytest.raises(AssertionError):
        Stencil(img, [x, y], [[1, 2], [3]])
    with pytest.raises(TypeError):
        Stencil(x, [x, y], [[1]])


def test_condition_split_to_conjuncts():
    c = (Condition(x, '>', 1) & Condition(y, '!=', 3)) | \
        Condition(x, '==', 0)
    conj = c.split_to_conjuncts()
    assert len(conj) == 3
    assert [len(k) for k in conj] == [2, 2, 1]


def test_select_type_check_and_max_min():
    a = Max(x, y)
    assert isinstance(a, Select) and a.condition.conditional == '>'
    b = Min(x, 3)
    assert b.condition.conditional == '<'
    with pytest.raises(AssertionError):
        Select(Condition(x, '<', 1), Value(1.0, Float), Value(1, Int))


def test_function_definition_rules():
    f = Function(([x], [Interval(Int, 0, R)]), Float, "f")
    with pytest.raises(AssertionError):
        f.defn = [x + 1, Case(Condition(x, '<', 2), x)]
    g = Function(([x], [Interval(Int, 0, R)]), Float, "g")
    g.defn = [Case(Condition(x, '<', 2), 1.0), Case(Condition(x, '>=', 2),
                                                    2.0)]
    assert len(g.defn) == 2
    with pytest.raises(AssertionError):
        g(x, y)
