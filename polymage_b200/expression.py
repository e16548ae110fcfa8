"""Analysis and rewriting of expression trees.

Public functions keep the reference's names and meaning
(sandbox/expression.py): ``get_affine_var_and_param_coeff`` (:29),
``get_constant_from_expr`` (:114), ``is_constant_expr`` (:138),
``simplify_expr`` (:158), ``substitute_refs`` (:201), ``substitute_vars``
(:240), ``isAffine`` (:283) and ``getType`` (:355).  ``rebuild`` and
``affine_form`` are helpers of this backend.
"""

from fractions import Fraction

from .expr_types import Int, Rational, result_type
from .expr_ast import (AbstractExpression, Value, AbstractBinaryOpNode,
                       AbstractUnaryOpNode, InbuiltFunction, UnaryMinus,
                       UnaryPlus, make_binop)
from . import constructs as C


def _lift(e):
    return Value.numericToValue(e)


# ---------------------------------------------------------------------------
def getType(expr):
    """Scalar type of an expression under the language's promotion rules."""
    expr = _lift(expr)
    if isinstance(expr, Value):
        return expr.typ
    if isinstance(expr, C.Variable):
        return expr.typ
    if isinstance(expr, C.Reference):
        return expr.objectRef.typ
    if isinstance(expr, AbstractBinaryOpNode):
        return result_type(getType(expr.left), getType(expr.right))
    if isinstance(expr, AbstractUnaryOpNode):
        return getType(expr.child)
    if isinstance(expr, C.Cast):
        return expr.typ
    if isinstance(expr, C.Select):
        t = getType(expr.true_expression)
        f = getType(expr.false_expression)
        if t is f:
            return t
        return result_type(t, f)
    if isinstance(expr, InbuiltFunction):
        return expr.getType()
    raise TypeError(type(expr))


# ---------------------------------------------------------------------------
def _has_var_or_param(e):
    return e.has(C.Variable) or e.has(C.Parameter)


def isAffine(expr, include_div=True, include_modulo=False):
    """Conservative affinity test over variables and parameters
    (rules of sandbox/expression.py:283-353)."""
    expr = _lift(expr)
    if isinstance(expr, Value):
        return (expr.typ is Int) or (include_div and expr.typ is Rational)
    if isinstance(expr, C.Variable):
        return True
    if isinstance(expr, C.Reference):
        return False
    if isinstance(expr, AbstractBinaryOpNode):
        if not (isAffine(expr.left, include_div, include_modulo) and
                isAffine(expr.right, include_div, include_modulo)):
            return False
        if expr.op in ('+', '-'):
            return True
        if expr.op == '*':
            return not (_has_var_or_param(expr.left) and
                        _has_var_or_param(expr.right))
        if include_div and expr.op == '/':
            return not _has_var_or_param(expr.right)
        if include_modulo and expr.op == '%':
            if _has_var_or_param(expr.right):
                return False
            return isAffine(expr.left, include_div, False)
        return False
    if isinstance(expr, AbstractUnaryOpNode):
        return isAffine(expr.child, include_div, include_modulo)
    if isinstance(expr, C.Condition):
        if expr.conditional in ('&&', '||'):
            return isAffine(expr.lhs, include_div, include_modulo) and \
                isAffine(expr.rhs, include_div, include_modulo)
        return isAffine(expr.lhs, include_div, include_modulo) and \
            isAffine(expr.rhs, include_div, include_modulo)
    if isinstance(expr, (C.Select, C.Cast, InbuiltFunction)):
        return False
    raise TypeError(type(expr))


def _eval_binop(l, r, op, affine):
    if op == '/':
        return Fraction(l, r) if affine else l / r
    if op == '+':
        return l + r
    if op == '-':
        return l - r
    if op == '*':
        return l * r
    if op == '%':
        return l % r
    if op == '>>':
        return l >> r
    if op == '<<':
        return l << r
    if op == '|':
        return l | r
    if op == '^':
        return l ^ r
    if op == '&':
        return l & r
    raise TypeError(op)


def get_constant_from_expr(expr, affine=False):
    """Constant term of an expression (references, variables and
    non-arithmetic nodes contribute 0)."""
    expr = _lift(expr)
    if isinstance(expr, Value):
        if affine:
            assert expr.typ is Int or expr.typ is Rational
        return expr.value
    if isinstance(expr, (C.Variable, C.Reference)):
        return 0
    if isinstance(expr, AbstractBinaryOpNode):
        return _eval_binop(get_constant_from_expr(expr.left, affine),
                           get_constant_from_expr(expr.right, affine),
                           expr.op, affine)
    if isinstance(expr, AbstractUnaryOpNode):
        v = get_constant_from_expr(expr.child, affine)
        return -v if expr.op == '-' else v
    if isinstance(expr, (C.Select, C.Cast, InbuiltFunction)):
        return 0
    raise TypeError(type(expr))


def is_constant_expr(expr, affine=False):
    expr = _lift(expr)
    if isinstance(expr, Value):
        if affine:
            return expr.typ is Int or expr.typ is Rational
        return True
    if isinstance(expr, (C.Variable, C.Reference)):
        return False
    if isinstance(expr, AbstractBinaryOpNode):
        return is_constant_expr(expr.left, affine) and \
            is_constant_expr(expr.right, affine)
    if isinstance(expr, AbstractUnaryOpNode):
        return is_constant_expr(expr.child, affine)
    if isinstance(expr, (C.Select, C.Cast, InbuiltFunction)):
        return False
    raise TypeError(type(expr))


def get_affine_var_and_param_coeff(expr):
    """Coefficients of the variables and parameters of an affine expression
    (``{}`` for constants and non-affine expressions)."""
    expr = _lift(expr)
    if not isAffine(expr) or isinstance(expr, Value) or \
            is_constant_expr(expr):
        return {}
    if isinstance(expr, C.Variable):
        return {expr: 1}
    if isinstance(expr, AbstractBinaryOpNode):
        lc = get_affine_var_and_param_coeff(expr.left)
        rc = get_affine_var_and_param_coeff(expr.right)
        keys = list(lc) + [k for k in rc if k not in lc]
        if expr.op == '+':
            return dict((k, lc.get(k, 0) + rc.get(k, 0)) for k in keys)
        if expr.op == '-':
            return dict((k, lc.get(k, 0) - rc.get(k, 0)) for k in keys)
        if expr.op == '*':
            lconst = is_constant_expr(expr.left, affine=True)
            rconst = is_constant_expr(expr.right, affine=True)
            assert not (lconst and rconst)
            if lconst:
                k0 = get_constant_from_expr(expr.left, affine=True)
                return dict((k, k0 * v) for k, v in rc.items())
            if rconst:
                k0 = get_constant_from_expr(expr.right, affine=True)
                return dict((k, k0 * v) for k, v in lc.items())
            return {}
        if expr.op == '/':
            assert is_constant_expr(expr.right, affine=True)
            d = get_constant_from_expr(expr.right, affine=True)
            return dict((k, Fraction(1, d) * v) for k, v in lc.items())
        return {}
    if isinstance(expr, AbstractUnaryOpNode):
        c = get_affine_var_and_param_coeff(expr.child)
        if expr.op == '-':
            return dict((k, -v) for k, v in c.items())
        return c
    raise TypeError(type(expr))


def simplify_expr(expr):
    """Collect like terms of an affine, division-free expression into
    ``const + sum(coeff * var)``; other expressions are cloned unchanged
    (sandbox/expression.py:158-199)."""
    expr = _lift(expr)
    if isinstance(expr, (Value, C.Variable)):
        return expr.clone()
    if isinstance(expr, C.Reference):
        return expr.objectRef(*[simplify_expr(a) for a in expr.arguments])
    if isinstance(expr, (AbstractBinaryOpNode, AbstractUnaryOpNode)):
        if isAffine(expr, include_div=False):
            coeff = get_affine_var_and_param_coeff(expr)
            out = get_constant_from_expr(expr)
            vs = [v for v in coeff if not isinstance(v, C.Parameter)]
            ps = [v for v in coeff if isinstance(v, C.Parameter)]
            for v in vs + ps:
                c = coeff[v]
                if c == 0:
                    continue
                if c == 1:
                    out = out + v
                elif c == -1:
                    out = out - v
                else:
                    out = out + c * v
            return _lift(out)
        return expr.clone()
    if isinstance(expr, (C.Select, C.Cast, InbuiltFunction)):
        return expr.clone()
    raise TypeError(type(expr))


# ---------------------------------------------------------------------------
def rebuild(expr, leaf):
    """Rebuild an expression bottom-up.  ``leaf(node)`` is called on every
    node first; if it returns something other than ``None`` that replaces the
    node, otherwise the node is rebuilt from its rebuilt children (without
    the building shortcuts, so the shape is preserved)."""
    expr = _lift(expr)
    r = leaf(expr)
    if r is not None:
        return r
    if isinstance(expr, (Value, C.Variable)):
        return expr
    if isinstance(expr, C.Reference):
        return C.Reference(expr.objectRef,
                           [rebuild(a, leaf) for a in expr.arguments])
    if isinstance(expr, AbstractBinaryOpNode):
        return make_binop(expr.op, rebuild(expr.left, leaf),
                          rebuild(expr.right, leaf))
    if isinstance(expr, AbstractUnaryOpNode):
        cls = UnaryMinus if expr.op == '-' else UnaryPlus
        return cls(rebuild(expr.child, leaf))
    if isinstance(expr, C.Cast):
        return C.Cast(expr.typ, rebuild(expr.expression, leaf))
    if isinstance(expr, C.Select):
        return C.Select(rebuild_cond(expr.condition, leaf),
                        rebuild(expr.true_expression, leaf),
                        rebuild(expr.false_expression, leaf),
                        typeCheck=False)
    if isinstance(expr, InbuiltFunction):
        return expr.rebuild([rebuild(a, leaf) for a in expr.arguments])
    raise TypeError(type(expr))


def rebuild_cond(cond, leaf):
    if cond.conditional in ('&&', '||'):
        return C.Condition(rebuild_cond(cond.lhs, leaf), cond.conditional,
                           rebuild_cond(cond.rhs, leaf))
    return C.Condition(rebuild(cond.lhs, leaf), cond.conditional,
                       rebuild(cond.rhs, leaf))


def substitute_vars(expr, var_to_expr_map):
    """Replace variables by expressions (then simplify affine parts)."""
    if isinstance(expr, C.Condition):
        return rebuild_cond(expr, lambda n: _sub_var_leaf(n, var_to_expr_map))
    out = rebuild(expr, lambda n: _sub_var_leaf(n, var_to_expr_map))
    return simplify_expr(out) if isAffine(out, include_div=False) else out


def _sub_var_leaf(node, m):
    if isinstance(node, C.Variable) and node in m:
        return _lift(m[node])
    return None


def substitute_refs(expr, ref_to_expr_map):
    """Replace the given Reference objects by expressions.  When the map
    holds a function's body keyed by a reference, the body's variables are
    bound to that reference's arguments (sandbox/expression.py:201-238)."""
    def leaf(n):
        if isinstance(n, C.Reference) and n in ref_to_expr_map:
            fvars = n.objectRef.variables
            binding = dict(zip(fvars, n.arguments))
            return substitute_vars(ref_to_expr_map[n], binding)
        return None
    return rebuild(expr, leaf)


# ---------------------------------------------------------------------------
def affine_form(expr):
    """``(coeffs, const)`` of an affine integer expression without division,
    where ``coeffs`` maps Variable/Parameter objects to ints; ``None`` when
    the expression is not of that form."""
    expr = _lift(expr)
    if isinstance(expr, Value):
        if expr.typ is Int:
            return ({}, expr.value)
        return None
    if isinstance(expr, C.Variable):
        return ({expr: 1}, 0)
    if isinstance(expr, AbstractUnaryOpNode):
        f = affine_form(expr.child)
        if f is None:
            return None
        if expr.op == '-':
            return (dict((k, -v) for k, v in f[0].items()), -f[1])
        return f
    if isinstance(expr, AbstractBinaryOpNode):
        if expr.op not in ('+', '-', '*'):
            return None
        lf = affine_form(expr.left)
        rf = affine_form(expr.right)
        if lf is None or rf is None:
            return None
        if expr.op in ('+', '-'):
            s = 1 if expr.op == '+' else -1
            c = dict(lf[0])
            for k, v in rf[0].items():
                c[k] = c.get(k, 0) + s * v
            return (dict((k, v) for k, v in c.items() if v != 0),
                    lf[1] + s * rf[1])
        if not lf[0]:
            k0 = lf[1]
            return (dict((k, k0 * v) for k, v in rf[0].items() if k0 * v),
                    k0 * rf[1])
        if not rf[0]:
            k0 = rf[1]
            return (dict((k, k0 * v) for k, v in lf[0].items() if k0 * v),
                    k0 * lf[1])
        return None
    return None
