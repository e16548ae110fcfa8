"""Direct evaluation of DSL definitions, point by point, in FP64 with C
integer semantics -- a test aid.  It reads the spec the way the reference
defines it (later Cases override earlier ones; points no Case covers read
as 0, the convention of the oracles) and so checks a restatement against
the definitions it restates, independently of the compiler.  Slow:
tiny images only."""

import math

import numpy as np

from polymage_b200 import constructs as C
from polymage_b200.expr_ast import (Value, AbstractBinaryOpNode,
                                    AbstractUnaryOpNode)
from polymage_b200.evaluate import c_div, c_mod
from polymage_b200.pipe import body_parts

_BUILTINS = {C.Exp: math.exp, C.Log: math.log, C.Sqrt: math.sqrt,
             C.Sqrtf: math.sqrt, C.Abs: abs, C.Sin: math.sin,
             C.Cos: math.cos, C.Pow: math.pow, C.Powf: math.pow}
_INTS = (C.Int, C.UInt, C.Short, C.UShort, C.Char, C.UChar, C.Long,
         C.ULong)


class Evaluator(object):
    def __init__(self, params, images, oob_zero=False):
        """``params``: {name: value}; ``images``: {name: numpy array}
        indexed from 0 (the image's domain lower bounds are 0).
        ``oob_zero``: an image read outside the array reads 0 (the
        convention of compiler option 'oob_zero')."""
        self.params = params
        self.images = images
        self.oob_zero = oob_zero
        self.memo = {}

    def value(self, f, args):
        args = tuple(int(a) for a in args)
        if isinstance(f, C.Image):
            a = self.images[f.name]
            if self.oob_zero and any(i < 0 or i >= n
                                     for i, n in zip(args, a.shape)):
                return 0.0
            return a[args].item()
        key = (id(f), args)
        if key in self.memo:
            return self.memo[key]
        if isinstance(f, C.Reduction):
            self.reduce(f)
            return self.memo.get(key, self.expr(f.default, {}))
        env = dict(zip([id(v) for v in f.variables], args))
        v = 0
        for cond, expr, red in body_parts(f):
            if cond is None or self.cond(cond, env):
                v = self.expr(expr, env)
        if f.typ in _INTS:
            v = int(v)
        self.memo[key] = v
        return v

    def reduce(self, f):
        """Every cell of a Reduction: the default, then each part's
        ``Reduce`` applied in order over the reduction domain (sequential
        accumulation, as the reference's generated loops do)."""
        done = (id(f), 'reduced')
        if done in self.memo:
            return
        self.memo[done] = True
        ranges = []
        for d in f.reductionDomain:
            ranges.append(range(self.expr(d.lowerBound, {}),
                                self.expr(d.upperBound, {}) + 1))
        ids = [id(v) for v in f.reductionVariables]
        dflt = self.expr(f.default, {})
        ops = {C.Op.Sum: lambda a, b: a + b, C.Op.Mul: lambda a, b: a * b,
               C.Op.Min: min, C.Op.Max: max}
        for cond, expr, red in body_parts(f):
            op = ops[red.op_type]
            for pt in np.ndindex(*[len(r) for r in ranges]):
                env = dict((i, r[k]) for i, r, k in zip(ids, ranges, pt))
                cell = tuple(int(self.expr(a, env)) for a in
                             red.accumulate_ref.arguments)
                # a function variable that is not reduced over stands for
                # the target cell's index (a condition on it selects cells)
                for fv, ci in zip(f.variables, cell):
                    if id(fv) not in env:
                        env[id(fv)] = ci
                if cond is not None and not self.cond(cond, env):
                    continue
                key = (id(f), cell)
                cur = self.memo.get(key, dflt)
                v = op(cur, self.expr(expr, env))
                self.memo[key] = int(v) if f.typ in _INTS else v

    def cond(self, c, env):
        op = c.conditional
        if op in ('&&', '||'):
            a = self.cond(c.lhs, env)
            if op == '&&':
                return a and self.cond(c.rhs, env)
            return a or self.cond(c.rhs, env)
        a = self.expr(c.lhs, env)
        b = self.expr(c.rhs, env)
        return {'<': a < b, '<=': a <= b, '>': a > b, '>=': a >= b,
                '==': a == b, '!=': a != b}[op]

    def expr(self, e, env):
        e = Value.numericToValue(e)
        if isinstance(e, Value):
            v = e.value
            return int(v) if e.typ in _INTS else float(v)
        if isinstance(e, C.Parameter):
            return self.params[e.name]
        if isinstance(e, C.Variable):
            return env[id(e)]
        if isinstance(e, C.Reference):
            f = e.objectRef
            args = [self.expr(a, env) for a in e.arguments]
            if not isinstance(f, C.Image):
                # a data-dependent index is clamped into the producer's
                # domain, as the compiled code clamps it
                for d, a in enumerate(e.arguments):
                    if a.has(C.Reference) if hasattr(a, 'has') else False:
                        lo = self.expr(f.domain[d].lowerBound, {})
                        hi = self.expr(f.domain[d].upperBound, {})
                        args[d] = min(max(args[d], lo), hi)
            return self.value(f, args)
        if isinstance(e, AbstractBinaryOpNode):
            a = self.expr(e.left, env)
            b = self.expr(e.right, env)
            ints = isinstance(a, int) and isinstance(b, int)
            op = e.op
            if op == '+':
                return a + b
            if op == '-':
                return a - b
            if op == '*':
                return a * b
            if op == '/':
                if ints:
                    return c_div(a, b)
                if b == 0:                  # IEEE: 0/0 is NaN, x/0 inf
                    return float('nan') if a == 0 or a != a else \
                        math.copysign(math.inf, a) * math.copysign(1.0, b)
                return a / b
            if op == '%':
                return c_mod(a, b)
            raise NotImplementedError(op)
        if isinstance(e, AbstractUnaryOpNode):
            v = self.expr(e.child, env)
            return -v if e.op == '-' else v
        if isinstance(e, C.Select):
            if self.cond(e.condition, env):
                return self.expr(e.true_expression, env)
            return self.expr(e.false_expression, env)
        if isinstance(e, C.Cast):
            v = self.expr(e.expression, env)
            return int(v) if e.typ in _INTS else float(v)
        for cls, fn in _BUILTINS.items():
            if isinstance(e, cls):
                args = [self.expr(a, env) for a in e.arguments]
                try:
                    return fn(*args)
                except ValueError:          # C: a domain error is NaN
                    return float('nan')
                except OverflowError:
                    return float('inf')
        raise NotImplementedError(type(e).__name__)

    def array(self, f, params_shape=None):
        """Every point of ``f``'s domain (lower bounds must be 0)."""
        dom = []
        for d in f.domain:
            lo = self.expr(d.lowerBound, {})
            hi = self.expr(d.upperBound, {})
            dom.append((lo, hi))
        shape = tuple(hi - lo + 1 for lo, hi in dom)
        out = np.zeros(shape)
        for idx in np.ndindex(*shape):
            out[idx] = self.value(f, [i + lo for i, (lo, _) in
                                      zip(idx, dom)])
        return out
