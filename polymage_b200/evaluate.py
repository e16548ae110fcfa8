"""Compile-time evaluation of index and bound expressions.

Domain bounds, index expressions and parameter estimates are evaluated with
C integer semantics (truncating ``/`` and ``%``), because that is what the
generated code computes (the reference emits C ``/`` for ``Div``:
sandbox/expr_ast.py:92-111, targetc printing).  Evaluation also works on
numpy integer arrays so region inference can be simulated for many tile
origins at once.
"""

from fractions import Fraction

import numpy as np

from .expr_ast import Value, AbstractBinaryOpNode, AbstractUnaryOpNode
from . import constructs as C


class EvalError(Exception):
    pass


def c_div(a, b):
    """C99 integer division (truncate toward zero), scalar or numpy."""
    if isinstance(a, np.ndarray) or isinstance(b, np.ndarray):
        a = np.asarray(a, dtype=np.int64)
        b = np.asarray(b, dtype=np.int64)
        q = np.abs(a) // np.abs(b)
        return np.where((a < 0) != (b < 0), -q, q)
    if b == 0:
        raise EvalError("division by zero")
    q = abs(a) // abs(b)
    return -q if (a < 0) != (b < 0) else q


def c_mod(a, b):
    """C99 remainder (sign of the dividend)."""
    return a - b * c_div(a, b)


def eval_int(expr, env):
    """Evaluate an integer expression of variables/parameters in ``env``
    (a dict keyed by Variable/Parameter objects).  Raises EvalError for
    anything that is not plain integer arithmetic."""
    expr = Value.numericToValue(expr)
    if isinstance(expr, Value):
        v = expr.value
        if isinstance(v, Fraction):
            if v.denominator != 1:
                raise EvalError("non-integer constant %s" % v)
            return int(v)
        if isinstance(v, float):
            if v != int(v):
                raise EvalError("non-integer constant %s" % v)
            return int(v)
        return v
    if isinstance(expr, C.Variable):
        if expr in env:
            return env[expr]
        raise EvalError("unbound %s" % expr.name)
    if isinstance(expr, AbstractBinaryOpNode):
        a = eval_int(expr.left, env)
        b = eval_int(expr.right, env)
        op = expr.op
        if op == '+':
            return a + b
        if op == '-':
            return a - b
        if op == '*':
            return a * b
        if op == '/':
            return c_div(a, b)
        if op == '%':
            return c_mod(a, b)
        if op == '<<':
            return a << b
        if op == '>>':
            return a >> b
        if op == '&':
            return a & b
        if op == '|':
            return a | b
        if op == '^':
            return a ^ b
        raise EvalError(op)
    if isinstance(expr, AbstractUnaryOpNode):
        v = eval_int(expr.child, env)
        return -v if expr.op == '-' else v
    if isinstance(expr, C.Select):
        c = eval_cond(expr.condition, env)
        t = eval_int(expr.true_expression, env)
        f = eval_int(expr.false_expression, env)
        if isinstance(c, np.ndarray):
            return np.where(c, t, f)
        return t if c else f
    raise EvalError("cannot evaluate %s at compile time" % (expr,))


def eval_cond(cond, env):
    op = cond.conditional
    if op in ('&&', '||'):
        a = eval_cond(cond.lhs, env)
        b = eval_cond(cond.rhs, env)
        if isinstance(a, np.ndarray) or isinstance(b, np.ndarray):
            return (a & b) if op == '&&' else (a | b)
        return (a and b) if op == '&&' else (a or b)
    a = eval_int(cond.lhs, env)
    b = eval_int(cond.rhs, env)
    return {'<': a < b, '<=': a <= b, '>': a > b, '>=': a >= b,
            '==': a == b, '!=': a != b}[op]


def try_eval_int(expr, env):
    try:
        return eval_int(expr, env)
    except EvalError:
        return None


def _has_loop_var(e):
    return any(not isinstance(v, C.Parameter)
               for v in e.collect(C.Variable)) if hasattr(e, 'collect') \
        else False


def divisors_in(expr):
    """Positive integer divisors used by ``/`` nodes whose numerator
    varies with a (non-parameter) variable: the divisions that make an
    index periodic in that variable.  Divisions of parameters and literals
    only (a level size ``(R + 63) / 64`` in a clamp bound) are constants
    and contribute nothing."""
    out = []
    stack = [expr]
    while stack:
        n = stack.pop()
        if isinstance(n, AbstractBinaryOpNode) and n.op == '/':
            r = n.right
            if isinstance(r, Value) and isinstance(r.value, int) and \
                    r.value > 0 and _has_loop_var(n.left):
                out.append(r.value)
        if hasattr(n, 'children'):
            stack.extend(n.children())
    return out


def is_min_max(e):
    """Whether a Select is a max or min of its two arms (``a > b ? a : b``
    and the like, also after cloning, which loses the Max/Min classes)."""
    if not isinstance(e, C.Select):
        return False
    c = e.condition
    if c.conditional not in ('<', '<=', '>', '>='):
        return False
    t, f = str(e.true_expression), str(e.false_expression)
    return (str(c.lhs), str(c.rhs)) in ((t, f), (f, t))


def monotone_dir(expr, var):
    """Direction in which an integer expression varies with ``var`` when
    everything else is fixed: +1 non-decreasing, -1 non-increasing,
    0 independent of ``var``, None when not provably monotone (products of
    parameters, remainders, references, selects...)."""
    expr = Value.numericToValue(expr)
    if isinstance(expr, Value):
        return 0
    if isinstance(expr, C.Parameter):
        return 0
    if isinstance(expr, C.Variable):
        return 1 if expr is var else 0      # another variable is held fixed
    if isinstance(expr, AbstractUnaryOpNode):
        d = monotone_dir(expr.child, var)
        if d is None:
            return None
        return -d if expr.op == '-' else d
    if isinstance(expr, AbstractBinaryOpNode):
        op = expr.op
        if op in ('+', '-'):
            a = monotone_dir(expr.left, var)
            b = monotone_dir(expr.right, var)
            if a is None or b is None:
                return None
            if op == '-':
                b = -b
            if a == 0:
                return b
            if b == 0 or a == b:
                return a
            return None
        if op == '*':
            a = monotone_dir(expr.left, var)
            b = monotone_dir(expr.right, var)
            if a is None or b is None:
                return None
            if a == 0 and b == 0:
                return 0
            const, d = (expr.left, b) if a == 0 else (expr.right, a)
            if b != 0 and a != 0:
                return None
            const = Value.numericToValue(const)
            if isinstance(const, Value) and isinstance(const.value, int):
                if const.value == 0:
                    return 0
                return d if const.value > 0 else -d
            return None
        if op == '/':
            a = monotone_dir(expr.left, var)
            r = Value.numericToValue(expr.right)
            if a is None or not isinstance(r, Value) or \
                    not isinstance(r.value, int) or r.value == 0:
                return None
            return a if r.value > 0 else -a
        return None
    if is_min_max(expr):
        # the max/min of two functions monotone in the same direction (or
        # constant in var) is monotone in that direction: clamped indices
        a = monotone_dir(expr.true_expression, var)
        b = monotone_dir(expr.false_expression, var)
        if a is None or b is None:
            return None
        if a == 0:
            return b
        if b == 0 or a == b:
            return a
        return None
    return None
