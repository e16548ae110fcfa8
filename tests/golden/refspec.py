"""Loads the reference's own, unmodified PolyMage DSL and app specs, and
evaluates a spec point by point with the C semantics of the reference's
generated code -- test infrastructure only: it runs where the reference
tree is present, to write the golden fixtures that pin the oracle's
restatements (tests/golden/make_spec_golden.py).  Nothing under
polymage_b200/ imports it, and no test needs it at run time.

Loading (the reference's DSL needs two things Python 3.12 lacks):
  * ``fractions.gcd`` (removed in Python 3.9; imported by
    sandbox/expr_ast.py:26 and sandbox/utils.py:26): stood in by math.gcd.
  * the ``cgen`` package (an empty submodule in the reference tree;
    sandbox/targetc.py:25 imports it and uses it only when printing code):
    stood in by a module whose every attribute is an inert class.
  * The app spec modules start with ``from __init__ import *`` (their
    directory's ROOT) and ``from compiler import *`` (the reference's
    compiler, which needs islpy): both stood in by modules that define
    only ROOT.  The spec functions use neither.

Evaluation follows the C the reference emits (sandbox/codegen.py:574-715,
sandbox/targetc.py:80-86):
  * every value carries its C type; integer operands smaller than int are
    promoted to int, mixed operands take the usual arithmetic conversions
    (double > float > integers), float arithmetic is IEEE single;
  * Python float literals print without a suffix, so they are double
    (Value(..., Float) -> double);
  * '/' and '%' on integers truncate toward zero;
  * ``Select`` (and Max/Min, which are Selects: sandbox/constructs.py:
    312-319) takes the common type of its two arms;
  * a store converts to the function's element type (float rounding,
    integer truncation and wrap-around);
  * later Cases of a definition override earlier ones (the reference
    emits one loop nest per Case, in order); a point no Case covers reads
    as 0 (the oracle's convention for points the reference leaves
    uninitialised);
  * a Reduction starts from its default and adds each Reduce's value
    sequentially over its reduction domain, outermost variable first
    (sandbox/codegen.py:268-295; the C target emits a sum whatever the
    Reduce's operator);
  * powf and pow call the C library's (ctypes on libm), as the compiled
    code does.
"""

import ctypes
import ctypes.util
import fractions
import importlib.util
import math
import os
import sys
import types

import numpy as np

REF_SANDBOX = os.environ.get("POLYMAGE_REFERENCE",
                             "/root/reference") + "/sandbox"
APPS = os.path.join(REF_SANDBOX, "apps", "python", "img_proc")

_libm = ctypes.CDLL(ctypes.util.find_library("m"))
_libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]
_libm.powf.restype = ctypes.c_float
_libm.pow.argtypes = [ctypes.c_double, ctypes.c_double]
_libm.pow.restype = ctypes.c_double

K = None        # the reference's constructs module, once loaded


def load_reference_dsl():
    """Import the reference's sandbox/constructs.py (and what it imports)
    from the reference tree, with the stand-ins described above."""
    global K
    if K is not None:
        return K
    if not os.path.isdir(REF_SANDBOX):
        raise FileNotFoundError("reference tree not found at %s"
                                % REF_SANDBOX)
    if not hasattr(fractions, "gcd"):
        fractions.gcd = math.gcd
    if "cgen" not in sys.modules:
        cg = types.ModuleType("cgen")

        class _Inert(object):
            def __init__(self, *a, **k):
                pass

        cg.__getattr__ = lambda name: _Inert
        sys.modules["cgen"] = cg
    if REF_SANDBOX not in sys.path:
        sys.path.insert(0, REF_SANDBOX)
    # the reference's own import order (sandbox/pipe.py:33-37): targetc
    # first, which pulls in cexpr and through it constructs
    import targetc      # noqa: E402,F401  (the reference's modules)
    import constructs   # noqa: E402
    K = constructs
    return K


def load_spec(app_dir, module_file):
    """Load a reference app spec module (e.g. ``campipe``,
    ``polymage_campipe.py``) and return it."""
    load_reference_dsl()
    for name in ("__init__", "compiler"):
        m = types.ModuleType(name)
        m.ROOT = REF_SANDBOX
        m.__all__ = ["ROOT"]
        sys.modules[name] = m
    path = os.path.join(APPS, app_dir, module_file)
    spec = importlib.util.spec_from_file_location(
        "refspec_" + app_dir, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# ---------------------------------------------------------------------------
# C types
_NP = {"Char": np.int8, "UChar": np.uint8, "Short": np.int16,
       "UShort": np.uint16, "Int": np.int32, "UInt": np.uint32,
       "Long": np.int64, "ULong": np.uint64, "Float": np.float32,
       "Double": np.float64}
_RANK = ["Int", "UInt", "Long", "ULong", "Float", "Double"]


def _tname(t):
    return t.__name__


def _promote(t):
    """C integer promotion: types narrower than int become int."""
    return "Int" if t in ("Char", "UChar", "Short", "UShort") else t


def _common(a, b):
    a, b = _promote(a), _promote(b)
    return a if _RANK.index(a) >= _RANK.index(b) else b


def convert(v, t):
    """The C conversion of Python number ``v`` to type name ``t``."""
    if t in ("Float", "Double"):
        return float(_NP[t](v))
    if isinstance(v, float):
        if math.isnan(v) or math.isinf(v):
            raise ValueError("float -> int conversion of %r" % v)
        v = int(v)                      # truncation toward zero
    info = np.iinfo(_NP[t])
    span = info.max - info.min + 1
    return (v - info.min) % span + info.min


def _cdiv(a, b):
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b >= 0) else -q


def _cmod(a, b):
    return a - _cdiv(a, b) * b


class CEvaluator(object):
    """Point-by-point evaluation of the reference's spec objects."""

    def __init__(self, params, images, fp64=False):
        """``params``: {name: value}; ``images``: {name: numpy array}
        indexed from 0.

        ``fp64``: float stages are kept in double (no float rounding of
        arithmetic or stores) -- the spec in FP64, the form the oracles
        restate -- except where a float expression is converted to an
        integer (a bin index), which is taken in float as the compiled
        code takes it, so that every discrete decision matches it."""
        self.K = load_reference_dsl()
        self.params = params
        self.images = images
        self.fp64 = fp64
        self.memo = {}

    def conv(self, v, t):
        if self.fp64 and t == "Float":
            return float(v)
        return convert(v, t)

    # -- values are (python number, C type name) ---------------------------
    def value(self, f, args):
        K = self.K
        args = tuple(int(a) for a in args)
        t = _tname(f.typ)
        if isinstance(f, K.Image):
            return convert(self.images[f.name][args].item(), t), t
        key = (id(f), args, self.fp64)
        if key in self.memo:
            return self.memo[key], t
        if isinstance(f, K.Reduction):
            self.reduce(f)
            if key in self.memo:
                return self.memo[key], t
            v, vt = self.expr(f.default, {})
            return self.conv(v, t), t
        env = dict((id(fv), (a, "Int")) for fv, a in zip(f.variables, args))
        v = 0
        for part in f.defn:
            if isinstance(part, K.Case):
                if self.cond(part.condition, env):
                    v = self.expr(part.expression, env)[0]
            else:
                v = self.expr(part, env)[0]
        v = self.conv(v, t)
        self.memo[key] = v
        return v, t

    def reduce(self, f):
        K = self.K
        done = (id(f), "reduced", self.fp64)
        if done in self.memo:
            return
        self.memo[done] = True
        t = _tname(f.typ)
        ranges = [range(self.expr(d.lowerBound, {})[0],
                        self.expr(d.upperBound, {})[0] + 1)
                  for d in f.reductionDomain]
        ids = [id(v) for v in f.reductionVariables]
        dflt = self.conv(self.expr(f.default, {})[0], t)
        for part in f.defn:
            cond, red = (part.condition, part.expression) \
                if isinstance(part, K.Case) else (None, part)
            for pt in np.ndindex(*[len(r) for r in ranges]):
                env = dict((i, (r[k], "Int"))
                           for i, r, k in zip(ids, ranges, pt))
                cell = tuple(self.expr(a, env)[0]
                             for a in red.accumulate_ref.arguments)
                for fv, ci in zip(f.variables, cell):
                    if id(fv) not in env:
                        env[id(fv)] = (ci, "Int")
                if cond is not None and not self.cond(cond, env):
                    continue
                key = (id(f), cell, self.fp64)
                cur = self.memo.get(key, dflt)
                v, vt = self.expr(red.expression, env)
                # the reference's C target emits ``ref = ref + expr`` for
                # every Reduce (sandbox/codegen.py:281); its Reduce.op_type
                # property returns the expression, so read the operator
                # from the attribute and accept sums only
                if red._op_typ != K.Op.Sum:
                    raise NotImplementedError("Reduce op %r" % red._op_typ)
                r = self._arith('+', cur, t, v, vt)[0]
                self.memo[key] = self.conv(r, t)

    def cond(self, c, env):
        op = c.conditional
        if op in ('&&', '||'):
            a = self.cond(c.lhs, env)
            if op == '&&':
                return a and self.cond(c.rhs, env)
            return a or self.cond(c.rhs, env)
        a, at = self.expr(c.lhs, env)
        b, bt = self.expr(c.rhs, env)
        ct = _common(at, bt)
        a, b = self.conv(a, ct), self.conv(b, ct)
        return {'<': a < b, '<=': a <= b, '>': a > b, '>=': a >= b,
                '==': a == b, '!=': a != b}[op]

    def _arith(self, op, a, at, b, bt):
        ct = _common(at, bt)
        a, b = self.conv(a, ct), self.conv(b, ct)
        if ct == "Float" and not self.fp64:
            fa, fb = np.float32(a), np.float32(b)
            with np.errstate(all='ignore'):
                r = {'+': fa + fb, '-': fa - fb, '*': fa * fb,
                     '/': fa / fb}[op]
            return float(r), ct
        if ct in ("Float", "Double"):
            if op == '/' and b == 0.0:
                r = math.copysign(math.inf, a) if a != 0 else math.nan
            else:
                r = {'+': a + b, '-': a - b, '*': a * b,
                     '/': (a / b) if b != 0 else 0.0}[op]
            return r, ct
        if op == '+':
            r = a + b
        elif op == '-':
            r = a - b
        elif op == '*':
            r = a * b
        elif op == '/':
            r = _cdiv(a, b)
        elif op == '%':
            r = _cmod(a, b)
        else:
            raise NotImplementedError(op)
        return convert(r, ct), ct

    def expr(self, e, env):
        K = self.K
        e = K.Value.numericToValue(e)
        if isinstance(e, K.Value):
            t = _tname(e.typ)
            if t == "Float":            # printed unsuffixed: a double
                return float(e.value), "Double"
            if t == "Rational":
                return float(e.value), "Double"
            return convert(e.value, t), t
        if isinstance(e, K.Parameter):
            t = _tname(e.typ)
            return convert(self.params[e.name], t), t
        if isinstance(e, K.Variable):
            return env[id(e)]
        if isinstance(e, K.Reference):
            args = [self.expr(a, env)[0] for a in e.arguments]
            return self.value(e.objectRef, args)
        if isinstance(e, K.AbstractBinaryOpNode):
            a, at = self.expr(e.left, env)
            b, bt = self.expr(e.right, env)
            return self._arith(e.op, a, at, b, bt)
        if isinstance(e, K.AbstractUnaryOpNode):
            v, t = self.expr(e.child, env)
            t = _promote(t)
            if e.op == '-':
                return self.conv(-v, t), t
            return v, t
        if isinstance(e, K.Select):
            a, at = self.expr(e.true_expression, env)
            b, bt = self.expr(e.false_expression, env)
            ct = _common(at, bt)
            if self.cond(e.condition, env):
                return self.conv(a, ct), ct
            return self.conv(b, ct), ct
        if isinstance(e, K.Cast):
            t = _tname(e.typ)
            v, vt = self.expr(e.expression, env)
            if self.fp64 and vt == "Float" and t not in ("Float", "Double"):
                self.fp64 = False       # the bin index, as compiled
                try:
                    v, vt = self.expr(e.expression, env)
                finally:
                    self.fp64 = True
            return self.conv(v, t), t
        if isinstance(e, K.Powf):
            a = convert(self.expr(e.arguments[0], env)[0], "Float")
            b = convert(self.expr(e.arguments[1], env)[0], "Float")
            return float(_libm.powf(a, b)), "Float"
        if isinstance(e, K.Pow):
            a = convert(self.expr(e.arguments[0], env)[0], "Double")
            b = convert(self.expr(e.arguments[1], env)[0], "Double")
            return float(_libm.pow(a, b)), "Double"
        for cls, fn in ((K.Exp, math.exp), (K.Log, math.log),
                        (K.Sqrt, math.sqrt), (K.Sin, math.sin),
                        (K.Cos, math.cos)):
            if isinstance(e, cls):
                v = convert(self.expr(e.arguments[0], env)[0], "Double")
                return fn(v), "Double"
        if isinstance(e, K.Sqrtf):
            v = convert(self.expr(e.arguments[0], env)[0], "Float")
            return float(np.sqrt(np.float32(v))), "Float"
        if isinstance(e, K.Abs):
            v, t = self.expr(e.arguments[0], env)
            return abs(v), _promote(t)
        raise NotImplementedError(type(e).__name__)

    def array(self, f):
        """Every point of ``f``'s domain; returns (values, lower bounds)."""
        dom = [(self.expr(d.lowerBound, {})[0],
                self.expr(d.upperBound, {})[0]) for d in f.domain]
        shape = tuple(hi - lo + 1 for lo, hi in dom)
        t = _tname(f.typ)
        out = np.zeros(shape, dtype=np.float64 if self.fp64 and
                       t == "Float" else _NP[t])
        for idx in np.ndindex(*shape):
            out[idx] = self.value(f, [i + lo for i, (lo, _) in
                                      zip(idx, dom)])[0]
        return out, tuple(lo for lo, _ in dom)

    def function_named(self, out, name):
        """The stage called ``name`` among ``out``'s producers."""
        K = self.K
        seen, todo = set(), [out]
        while todo:
            f = todo.pop()
            if id(f) in seen:
                continue
            seen.add(id(f))
            if f.name == name:
                return f
            parts = list(f.defn)
            if isinstance(f, K.Reduction):
                parts.append(f.default)
            for p in parts:
                for r in _refs(K, p):
                    todo.append(r.objectRef)
        raise KeyError(name)


def _refs(K, e):
    """Every Reference inside an expression, Case, Reduce or Condition."""
    out = []
    stack = [e]
    while stack:
        x = stack.pop()
        x = K.Value.numericToValue(x)
        if isinstance(x, K.Reference):
            out.append(x)
            stack.extend(x.arguments)
        elif isinstance(x, K.Case):
            stack += [x.condition, x.expression]
        elif isinstance(x, K.Reduce):
            stack += [x.accumulate_ref, x.expression]
        elif isinstance(x, K.Condition):
            stack += [x.lhs, x.rhs]
        elif isinstance(x, K.AbstractBinaryOpNode):
            stack += [x.left, x.right]
        elif isinstance(x, K.AbstractUnaryOpNode):
            stack.append(x.child)
        elif isinstance(x, K.Select):
            stack += [x.condition, x.true_expression, x.false_expression]
        elif isinstance(x, K.Cast):
            stack.append(x.expression)
        elif isinstance(x, K.InbuiltFunction):
            stack.extend(x.arguments)
    return out
