"""CUDA code generation for sm_100a (replaces sandbox/codegen.py and
sandbox/targetc.py).

For every pipeline this module emits one CUDA translation unit:

* one kernel per fused stencil group (``GroupPlan``): a CTA per tile of the
  group's anchor runs region inference for its tile, stages stencil inputs
  into shared memory (TMA ``cp.async.bulk.tensor`` with an mbarrier when the
  buffer is 16-byte aligned, cooperative loads otherwise), computes every
  materialized stage over its region into shared memory in topological
  order (cheap stages are evaluated in registers at their use points, with
  common subexpressions shared), and writes live-outs to HBM for the points
  the tile owns;
* for a ``Reduction``: an init pass and a tiled accumulation kernel that
  privatizes the tile's target footprint in shared memory and flushes it
  with global atomics (the reference only supports ``+=``,
  sandbox/codegen.py:268-295; Min/Max/Mul are supported here too);
* for a ``const`` function: host C++ that tabulates it (compiled by the host
  compiler with the reference's flags so the table is bit-identical to what
  the reference's generated C++ computes) and an upload to HBM;
* host code: parameter validation (the bounds checks, per call), a
  workspace for intermediate arrays (storage_mapping.py), launches, and the
  ``extern "C"`` entry points.

Entry points of ``pipeline_<name>``, with the reference's argument order
(parameters sorted by name, then inputs, then outputs:
sandbox/codegen.py:957-1007, sandbox/targetc.py:344-366):

* ``void pipeline_<name>(params..., void* in..., void* out...)`` -- host
  buffers, synchronous: the reference's drop-in ABI.
* ``int pipeline_<name>_dev(params..., void* in..., void* out...,
  void* stream)`` -- device buffers, asynchronous on ``stream``.
* ``int pipeline_<name>_batch(int n, const int* iparams,
  const float* fparams, void* const* in, void* const* out, void* stream)``
  -- many images (each with its own parameters) in one launch per group;
  when a group has more tiles than fit on the GPU at once, a persistent
  grid drains a device-side tile queue over all images.
* ``int pipeline_<name>_batch_graph(...)`` -- the batch as one CUDA graph.
* ``int pipeline_<name>_graph(params..., ptrs..., void* stream)`` -- replays
  a CUDA graph of the whole pipeline captured on first use.
* ``int pipeline_<name>_status(void)`` and ``int pipeline_<name>_check(void)``
  -- last status, and the device error word (synchronizing).

Semantics kept from the reference's C target: C integer arithmetic and
promotion, truncating ``/`` and ``%``, stores convert to the stage's
element type (also for stages computed in registers), ``Select`` evaluates
both arms.  Float literals are emitted as ``float`` on the device (the
reference prints them as double, sandbox/targetc.py:80-86; the difference
is inside the stated tolerance) and exactly as the reference prints them in
host code for const tables.  Points of a stage not covered by any ``Case``
read as 0 (a defined value for what the reference leaves uninitialized);
points of a pipeline output not covered by any ``Case`` are left untouched,
as in the reference.
"""

import math
import re

import numpy as np

from . import constructs as C
from .expr_ast import (Value, AbstractBinaryOpNode, AbstractUnaryOpNode,
                       InbuiltFunction)
from .expression import substitute_vars, getType, affine_form
from .bounds import part_boxes
from .pipe import body_parts
from .tiling import is_data_dependent
from .evaluate import monotone_dir, is_min_max

_INT_T = (C.Int, C.UInt, C.Short, C.UShort, C.Char, C.UChar, C.Long,
          C.ULong)


# concurrent streams of the single-image entry points (option 'streams=N';
# 1 launches every group on the caller's stream)
DEFAULT_STREAMS = 4


class CodegenError(Exception):
    pass


class CudaModule(object):
    """Generated sources of one pipeline."""

    def __init__(self, name, source, host_source, header, meta):
        self.name = name
        self.source = source
        self.host_source = host_source
        self.header = header
        self.meta = meta

    def __str__(self):
        return self.source


class W(object):
    """Indented line writer."""

    def __init__(self):
        self.lines = []
        self.ind = 0

    def __call__(self, s=""):
        for line in s.split("\n"):
            self.lines.append(("  " * self.ind + line) if line else "")

    def open(self, s):
        self(s + " {")
        self.ind += 1

    def close(self, s="}"):
        self.ind -= 1
        self(s)

    def text(self):
        return "\n".join(self.lines) + "\n"


def ctype(t):
    if t not in _INT_T and t not in (C.Float, C.Double):
        raise CodegenError("no C type for %s" % t)
    return t.c_decl()


def _float_lit(v, suffix):
    v = float(v)
    if v != v or v in (float('inf'), float('-inf')):
        raise CodegenError("non-finite literal")
    s = repr(v)
    if 'e' not in s and '.' not in s:
        s += '.0'
    return s + suffix


# ---------------------------------------------------------------------------
class Names(object):
    def __init__(self):
        self.used = {}
        self.of = {}

    def get(self, obj, base):
        if id(obj) in self.of:
            return self.of[id(obj)]
        b = re.sub(r'[^A-Za-z0-9_]', '_', base)
        n = b
        i = 1
        while n in self.used:
            i += 1
            n = "%s_%d" % (b, i)
        self.used[n] = obj
        self.of[id(obj)] = n
        return n


class ExprCtx(object):
    """Expression printer with scoped common-subexpression temps.

    ``reader(func, arg_asts)`` returns a C lvalue/expression for a producer
    value (a shared-memory or global read, or an inlined computation) and
    may emit statements; ``bind`` maps DSL variables to ASTs over the loop
    variables of the point being computed."""

    def __init__(self, w, mode, params, reader):
        self.w = w
        self.mode = mode              # 'device' | 'host'
        self.params = params          # Parameter -> C name
        self.reader = reader
        self.scopes = [{}]
        self.ntemp = 0
        # lower bounds of loop variables (C name -> int), for emitting
        # unsigned division/modulo where the numerator cannot be negative
        self.var_lo = {}
        # residues of loop variables known at compile time
        # (C name -> (residue, modulus)), for folding x % k and parity
        # Selects on interior tiles
        self.var_res = {}
        # interior tiles whose clamped indices provably do not clamp: a
        # min/max of an index with a bound free of loop variables prints
        # as its unclamped arm (only inside index expressions)
        self.fold_clamps = False
        self._in_index = 0

    def temp(self):
        self.ntemp += 1
        return "t%d" % self.ntemp

    def lookup(self, key):
        for s in reversed(self.scopes):
            if key in s:
                return s[key]
        return None

    def define(self, key, name):
        self.scopes[-1][key] = name

    def push(self):
        self.scopes.append({})

    def pop(self):
        self.scopes.pop()

    # ---- printing ----------------------------------------------------------
    def lit(self, v):
        t = v.typ
        x = v.value
        if t is C.Rational:
            if x.denominator == 1:
                return str(int(x))
            return "(%s)" % _float_lit(float(x), '' if self.mode == 'host'
                                       else 'f')
        if t in _INT_T:
            x = int(x)
            s = str(x)
            if abs(x) >= (1 << 31):
                s += "LL"
            return "(%s)" % s if x < 0 else s
        if t is C.Float:
            s = _float_lit(x, '' if self.mode == 'host' else 'f')
        else:
            s = _float_lit(x, '')
        return "(%s)" % s if s.startswith('-') else s

    def expr(self, e, bind):
        e = Value.numericToValue(e)
        if isinstance(e, Value):
            return self.lit(e)
        if isinstance(e, C.Parameter):
            if e not in self.params:
                raise CodegenError("unknown parameter %s" % e.name)
            return self.params[e]
        if isinstance(e, C.Variable):
            if e in bind:
                b = bind[e]
                if isinstance(b, str):
                    return b
                return self.expr(b, {})
            if hasattr(e, '_cname'):
                return e._cname
            raise CodegenError("unbound variable %s" % e.name)
        if isinstance(e, C.Reference):
            args = [_subst(a, bind) for a in e.arguments]
            return self.reader(e.objectRef, args, self)
        if isinstance(e, AbstractBinaryOpNode):
            if e.op == '%':
                sm = self._static_mod(e, bind)
                if sm is not None:
                    return str(sm)
            if e.op == '/':
                sd = self._static_div(e, bind)
                if sd is not None:
                    return sd
            if e.op in ('/', '%') and self._unsigned_ok(e, bind):
                # truncating division of a non-negative int by a positive
                # constant equals unsigned division (a shift or mask for
                # powers of two); C semantics are unchanged
                return "((int)((unsigned)(%s) %s %du))" % (
                    self.expr(e.left, bind), e.op, int(e.right.value))
            return "(%s %s %s)" % (self.expr(e.left, bind), e.op,
                                   self.expr(e.right, bind))
        if isinstance(e, AbstractUnaryOpNode):
            return "(%s%s)" % (e.op, self.expr(e.child, bind))
        if isinstance(e, C.Cast):
            return "((%s)(%s))" % (ctype(e.typ), self.expr(e.expression, bind))
        if isinstance(e, C.Select):
            if self.fold_clamps and self._in_index:
                arm = _clamp_arm(e)
                if arm is not None:
                    return self.expr(arm, bind)
            sv = self._static_cond(e.condition, bind)
            if sv is not None:
                # the condition is known here: only the taken arm is
                # evaluated (the arms have no side effects)
                return self.expr(e.true_expression if sv else
                                 e.false_expression, bind)
            c = self.cond(e.condition, bind)
            a = self.expr(e.true_expression, bind)
            b = self.expr(e.false_expression, bind)
            return "(%s ? %s : %s)" % (c, a, b)
        if isinstance(e, (C.Pow, C.Powf)) and self.mode == 'device' and \
                self._int_power_of_two(e):
            # 2^n for an integer n is exact either way; ldexp scales by the
            # exponent instead of evaluating a general power
            n = self.expr(e.arguments[1], bind)
            if isinstance(e, C.Powf):
                return "ldexpf(1.0f, (int)(%s))" % n
            return "ldexp(1.0, (int)(%s))" % n
        if isinstance(e, InbuiltFunction):
            args = []
            for a in e.arguments:
                t = self.expr(a, bind)
                # C promotes an integer argument of a math function to
                # double (to float for the f-suffixed ones); CUDA has no
                # device overload taking an integer, so the conversion is
                # written out
                if self.mode == 'device' and not isinstance(e, C.Abs):
                    try:
                        it = getType(a) in _INT_T
                    except Exception:
                        it = False
                    if it:
                        t = "((%s)(%s))" % (
                            "float" if isinstance(e, (C.Powf, C.Sqrtf))
                            else "double", t)
                args.append(t)
            return "%s(%s)" % (self._fname(e), ", ".join(args))
        raise CodegenError("cannot print %r" % (e,))

    @staticmethod
    def _int_power_of_two(e):
        """Whether ``e`` is Pow(2, n) with n of a type whose every value
        converts to int unchanged."""
        b = Value.numericToValue(e.arguments[0])
        if not (isinstance(b, Value) and b.value == 2):
            return False
        try:
            t = getType(e.arguments[1])
        except Exception:
            return False
        return t in (C.Int, C.Short, C.UShort, C.Char, C.UChar)

    def _fname(self, e):
        if isinstance(e, C.RandomFloat):
            raise CodegenError("RandomFloat is not supported")
        if self.mode == 'host':
            return {C.Pow: 'pow', C.Powf: 'powf', C.Log: 'log',
                    C.Exp: 'std::exp', C.Sin: 'std::sin', C.Cos: 'std::cos',
                    C.Sqrt: 'std::sqrt', C.Sqrtf: 'sqrtf',
                    C.Abs: 'std::abs'}[type(e)]
        return {C.Pow: 'pow', C.Powf: 'powf', C.Log: 'log', C.Exp: 'exp',
                C.Sin: 'sin', C.Cos: 'cos', C.Sqrt: 'sqrt', C.Sqrtf: 'sqrtf',
                C.Abs: 'pm_abs'}[type(e)]

    def _unsigned_ok(self, e, bind):
        if not self.var_lo:
            return False
        r = e.right
        if not (isinstance(r, Value) and r.typ in _INT_T and r.typ is not
                C.Long and r.typ is not C.ULong and int(r.value) > 0):
            return False
        try:
            if getType(e.left) is not C.Int:
                return False
        except Exception:
            return False
        f = affine_form(_subst(e.left, bind))
        if f is None:
            return False
        low = f[1]
        for v, c in f[0].items():
            lo = self.var_lo.get(getattr(v, '_cname', None))
            if lo is None or c < 0:
                return False
            low += c * lo
        return low >= 0

    def _static_mod(self, e, bind):
        """Value of ``x % k`` when the residues of its loop variables are
        known and x cannot be negative; else None."""
        if not self.var_res:
            return None
        r = e.right
        if not (isinstance(r, Value) and r.typ in _INT_T and
                int(r.value) > 0) or not self._unsigned_ok(e, bind):
            return None
        m = int(r.value)
        f = affine_form(_subst(e.left, bind))
        if f is None:
            return None
        total = f[1]
        for v, c in f[0].items():
            rm = self.var_res.get(getattr(v, '_cname', None))
            if rm is None or rm[1] % m:
                return None
            total += c * rm[0]
        return total % m

    def _static_div(self, e, bind):
        """``(q + c) / k`` as ``q / k + d`` when the residue of loop variable
        ``q`` modulo ``k`` is known and the numerator cannot be negative
        (then q / k + (q % k + c) / k with the second term a constant), so
        that the consecutive points of a thread that fall into the same
        cell of a decimated producer index it by the same text; else
        None."""
        if not self.var_res:
            return None
        r = e.right
        if not (isinstance(r, Value) and r.typ in _INT_T and
                int(r.value) > 0) or not self._unsigned_ok(e, bind):
            return None
        k = int(r.value)
        f = affine_form(_subst(e.left, bind))
        if f is None or len(f[0]) != 1:
            return None
        (v, c), = f[0].items()
        name = getattr(v, '_cname', None)
        rm = self.var_res.get(name)
        lo = self.var_lo.get(name)
        if c != 1 or rm is None or rm[1] % k or lo is None or lo < 0:
            return None
        d = (rm[0] % k + f[1]) // k
        base = "((int)((unsigned)(%s) / %du))" % (name, k)
        return base if d == 0 else "(%s + %d)" % (base, d)

    def _static_int(self, e, bind):
        e = Value.numericToValue(e)
        if isinstance(e, Value):
            return int(e.value) if e.typ in _INT_T else None
        if isinstance(e, AbstractBinaryOpNode) and e.op == '%':
            return self._static_mod(e, bind)
        return None

    def _static_cond(self, c, bind):
        """True/False when condition ``c`` is decided by known residues."""
        if not self.var_res:
            return None
        op = c.conditional
        if op in ('&&', '||'):
            a = self._static_cond(c.lhs, bind)
            b = self._static_cond(c.rhs, bind)
            if op == '&&':
                if a is False or b is False:
                    return False
                return True if (a and b) else None
            if a is True or b is True:
                return True
            return False if (a is False and b is False) else None
        a = self._static_int(c.lhs, bind)
        b = self._static_int(c.rhs, bind)
        if a is None or b is None:
            return None
        return {'==': a == b, '!=': a != b, '<': a < b, '<=': a <= b,
                '>': a > b, '>=': a >= b}.get(op)

    def cond(self, c, bind):
        op = c.conditional
        if op in ('&&', '||'):
            return "(%s %s %s)" % (self.cond(c.lhs, bind), op,
                                   self.cond(c.rhs, bind))
        return "(%s %s %s)" % (self.expr(c.lhs, bind), op,
                               self.expr(c.rhs, bind))

    def index(self, e):
        """Canonical C text of an index AST over loop variables."""
        saved = self._in_index
        # clamps fold only in an index monotone in one loop variable and
        # free of data: the indices whose clamps the interior test checks
        self._in_index = 0
        if self.fold_clamps and not is_data_dependent(e):
            vs = dict((id(v), v) for v in e.collect(C.Variable)
                      if not isinstance(v, C.Parameter))
            if len(vs) == 1 and monotone_dir(
                    e, list(vs.values())[0]) in (1, -1):
                self._in_index = 1
        try:
            return self._index(e)
        finally:
            self._in_index = saved

    def unclamped(self, e, bind):
        """C text of index ``e`` with its clamps (min/max against bounds
        free of loop variables) dropped."""
        saved = (self.fold_clamps, self._in_index)
        self.fold_clamps, self._in_index = True, 1
        try:
            return self.expr(e, bind)
        finally:
            self.fold_clamps, self._in_index = saved

    def _index(self, e):
        f = affine_form(e)
        if f is not None:
            parts = []
            for k, c in sorted(f[0].items(), key=lambda kv: self.expr(
                    kv[0], {})):
                n = self.expr(k, {})
                if c == 1:
                    parts.append(n)
                elif c == -1:
                    parts.append("-" + n)
                else:
                    parts.append("%d*%s" % (c, n))
            if f[1] or not parts:
                parts.append(str(f[1]))
            s = " + ".join(parts).replace("+ -", "- ")
            return "(%s)" % s
        return self.expr(e, {})


def _inner_parity(f, var):
    """Whether a stage's definition divides or takes the remainder of an
    expression of ``var`` by 2 (an upsampling by 2 along that dimension)."""
    from .pipe import body_parts
    stack = []
    for cond, expr, red in body_parts(f):
        stack.append(expr)
        if cond is not None:
            stack.append(cond)
    while stack:
        x = stack.pop()
        x = Value.numericToValue(x)
        if isinstance(x, AbstractBinaryOpNode) and x.op in ('/', '%') and \
                isinstance(x.right, Value) and x.right.typ in _INT_T and \
                int(x.right.value) == 2 and \
                any(v is var for v in x.left.collect(C.Variable)):
            return True
        if isinstance(x, C.Condition):
            stack += [x.lhs, x.rhs]
        elif hasattr(x, 'children'):
            stack.extend(x.children())
        elif isinstance(x, C.Select):
            stack += [x.condition, x.true_expression, x.false_expression]
    return False


def _top_level_decls(lines):
    """(type, name) of the ``int`` / ``bool`` variables that generated
    statements declare outside any braces, in order (declarator lists are
    split at commas outside parentheses)."""
    out = []
    depth = 0
    for raw in lines:
        s = raw.strip()
        if depth == 0:
            m = re.match(r'(?:const )?(int|bool) (.*);$', s)
            if m:
                typ, rest = m.group(1), m.group(2)
                par, cur, parts = 0, [], []
                for ch in rest:
                    if ch == '(':
                        par += 1
                    elif ch == ')':
                        par -= 1
                    if ch == ',' and par == 0:
                        parts.append("".join(cur))
                        cur = []
                    else:
                        cur.append(ch)
                parts.append("".join(cur))
                for p in parts:
                    out.append((typ, p.split('=')[0].strip()))
        depth += s.count('{') - s.count('}')
    return out


def _opt(pipeline, name, default=None):
    from .tiling import _option
    return _option(pipeline, name, default)


def _vn(v):
    return "v_" + re.sub(r'[^A-Za-z0-9_]', '_', v.name)


def _has_loop_var(e):
    return any(not isinstance(v, C.Parameter)
               for v in e.collect(C.Variable))


def _clamp_arm(e):
    """The unclamped arm of a clamp ``min/max(v, bound)`` in index
    arithmetic (``bound`` free of loop variables, no data), else None."""
    if not is_min_max(e) or is_data_dependent(e):
        return None
    t, f = e.true_expression, e.false_expression
    tv, fv = _has_loop_var(t), _has_loop_var(f)
    if tv and not fv:
        return t
    if fv and not tv:
        return f
    return None


def _has_clamp(e):
    stack = [e]
    while stack:
        n = stack.pop()
        if _clamp_arm(n) is not None:
            return True
        if hasattr(n, 'children'):
            stack.extend(n.children())
    return False


def _fixed_cells(f, cond, red):
    """{cell coordinate: constant} that a Reduction part's condition fixes:
    conjuncts ``v == k`` where ``v`` is the part's target argument at that
    coordinate (a reduction variable used as the cell index) or the
    function variable of that coordinate (which stands for the target
    cell's index)."""
    out = {}
    if cond is None:
        return out
    pos = {}
    for d, (fv, ta) in enumerate(zip(f.variables, red.accumulate_ref.arguments)):
        pos.setdefault(id(fv), d)
        if isinstance(ta, C.Variable):
            pos.setdefault(id(ta), d)
    stack = [cond]
    while stack:
        c = stack.pop()
        if c.conditional == '&&':
            stack.extend([c.lhs, c.rhs])
        elif c.conditional == '==':
            for v, k in ((c.lhs, c.rhs), (c.rhs, c.lhs)):
                k = Value.numericToValue(k)
                if isinstance(v, C.Variable) and id(v) in pos and \
                        isinstance(k, Value) and isinstance(k.value, int):
                    out[pos[id(v)]] = int(k.value)
    return out


def _disjoint_parts(f, parts):
    """Whether every two parts of a Reduction update disjoint cells: each
    fixes some cell coordinate to a constant the other fixes to a
    different value (the per-channel operators of a histogram)."""
    fixed = [_fixed_cells(f, cond, red) for cond, _, red in parts]
    for i in range(len(parts)):
        for j in range(i + 1, len(parts)):
            if not any(k in fixed[j] and fixed[j][k] != v
                       for k, v in fixed[i].items()):
                return False
    return True


def _subst(a, bind):
    """Substitute a variable binding (values are ASTs) into an index AST."""
    if not bind:
        return a
    m = dict((k, v) for k, v in bind.items() if not isinstance(v, str))
    if not m:
        return a
    return substitute_vars(a, m)


def tbind_of(f, rvars, red, rbind):
    """Binding for a reduction part: reduction variables to the loop
    variables, and every other function variable to the part's target
    index (a condition on it restricts the target cell)."""
    tb = dict(rbind)
    for fv, ta in zip(f.variables, red.accumulate_ref.arguments):
        if all(fv is not rv for rv in rvars):
            tb[fv] = _subst(ta, rbind)
    return tb


def _cond_const_true(c, bind):
    """True when condition ``c`` holds whatever the loop variables are
    (after substituting ``bind``; e.g. ``c == 0`` with c bound to 0)."""
    from .evaluate import try_eval_int
    op = c.conditional
    if op == '&&':
        return _cond_const_true(c.lhs, bind) and _cond_const_true(c.rhs, bind)
    if op == '||':
        return _cond_const_true(c.lhs, bind) or _cond_const_true(c.rhs, bind)
    a = try_eval_int(_subst(c.lhs, bind), {})
    b = try_eval_int(_subst(c.rhs, bind), {})
    if a is None or b is None:
        return False
    return {'==': a == b, '!=': a != b, '<': a < b, '<=': a <= b,
            '>': a > b, '>=': a >= b}.get(op, False)


def _cond_static(c, bind):
    """True / False when condition ``c`` has that value whatever the loop
    variables are (after substituting ``bind``), else None."""
    from .evaluate import try_eval_int
    op = c.conditional
    if op in ('&&', '||'):
        a = _cond_static(c.lhs, bind)
        b = _cond_static(c.rhs, bind)
        if op == '&&':
            if a is False or b is False:
                return False
            return True if (a and b) else None
        if a is True or b is True:
            return True
        return False if (a is False and b is False) else None
    a = try_eval_int(_subst(c.lhs, bind), {})
    b = try_eval_int(_subst(c.rhs, bind), {})
    if a is None or b is None:
        return None
    return {'==': a == b, '!=': a != b, '<': a < b, '<=': a <= b,
            '>': a > b, '>=': a >= b}.get(op)


def _const_int(e):
    """The value of an integer constant expression, else None."""
    try:
        f = affine_form(e)
    except Exception:
        return None
    if f is None or f[0]:
        return None
    return int(f[1])


def _loop_vars(n, prefix="q"):
    vs = []
    for i in range(n):
        v = C.Variable(C.Int, "%s%d" % (prefix, i))
        v._cname = "%s%d" % (prefix, i)
        vs.append(v)
    return vs


# ---------------------------------------------------------------------------
class PipelineGen(object):
    def __init__(self, pipeline):
        self.p = pipeline
        self.names = Names()
        self.pname = re.sub(r'[^A-Za-z0-9_]', '_', pipeline.name)
        self.params, self.inputs, self.outputs = pipeline.ordered_params()
        self.pmap = {}
        for prm in self.params:
            self.pmap[prm] = "p_" + self.names.get(prm, prm.name)
        self.iparams = [q for q in self.params
                        if q.typ not in (C.Float, C.Double)]
        self.fparams = [q for q in self.params
                        if q.typ in (C.Float, C.Double)]
        self.fname = {}
        all_funcs = list(self.inputs) + [c.func for c in pipeline.comps]
        for f in all_funcs:
            self.fname[id(f)] = self.names.get(f, f.name)
        self.w = W()
        self.hw = W()                 # host .cpp for const tables
        self.kernels = []
        self.meta = {'groups': []}

    def fn(self, f):
        return self.fname[id(f)]

    def ptype(self, prm):
        return 'float' if prm in self.fparams else 'int'

    # ---- expressions common to kernels and host ---------------------------
    def dom_exprs(self, f, ctx):
        out = []
        for d in f.domain:
            out.append((ctx.expr(d.lowerBound, {}), ctx.expr(d.upperBound,
                                                            {})))
        return out

    def declare_params(self, w, src):
        for prm in self.params:
            w("const %s %s = %s.%s;" % (self.ptype(prm), self.pmap[prm], src,
                                        self.pmap[prm]))

    def storage_perm(self, f):
        """Dimensions of an intermediate array, outermost to innermost in
        memory, when option ``('storage_order', ((name, dims), ...))``
        reorders it (a gather that varies another dimension across a
        warp then reads contiguous words); None for the domain's order.
        Caller-owned inputs and outputs and const tables keep theirs."""
        v = _opt(self.p, 'storage_order')
        if not v or any(f is x for x in self.inputs + self.outputs) or \
                getattr(f, 'is_const_func', False):
            return None
        for name, dims in v:
            if name != f.name:
                continue
            dims = tuple(int(d) for d in dims)
            if sorted(dims) != list(range(len(f.domain))):
                raise CodegenError("storage_order of %s: %r is not a "
                                   "permutation of its %d dimensions" % (
                                       f.name, dims, len(f.domain)))
            return None if dims == tuple(range(len(f.domain))) else dims
        return None

    def row_pitch(self, f):
        """Elements the innermost rows of ``f`` are padded to a multiple
        of in memory: 16 bytes' worth for an intermediate array of two or
        more dimensions in the workspace (so that its rows are 16-byte
        aligned and TMA can stage it), 1 for caller-owned inputs and
        outputs, for const tables, which are dense, and for reordered
        intermediates (never staged by TMA)."""
        if any(f is x for x in self.inputs + self.outputs) or \
                getattr(f, 'is_const_func', False) or \
                len(f.domain) < 2 or f.typ.size() >= 16 or \
                'no_row_pad' in self.p.options or \
                self.storage_perm(f) is not None:
            return 1
        return 16 // f.typ.size()

    def declare_domain(self, w, f, ctx, need_strides):
        n = self.fn(f)
        dom = self.dom_exprs(f, ctx)
        for d, (lo, hi) in enumerate(dom):
            w("const int d_%s_lo%d = %s, d_%s_hi%d = %s;" % (n, d, lo, n, d,
                                                            hi))
        perm = self.storage_perm(f) if need_strides else None
        if perm is not None:
            # reordered: the strides follow the memory order ``perm``
            w("const long long s_%s_%d = 1;" % (n, perm[-1]))
            for j in range(len(perm) - 2, -1, -1):
                d, dn = perm[j], perm[j + 1]
                w("const long long s_%s_%d = s_%s_%d * (long long)(d_%s_hi%d"
                  " - d_%s_lo%d + 1);" % (n, d, n, dn, n, dn, n, dn))
        elif need_strides:
            nd = len(dom)
            pitch = self.row_pitch(f)
            w("const long long s_%s_%d = 1;" % (n, nd - 1))
            for d in range(nd - 2, -1, -1):
                ext = "(long long)(d_%s_hi%d - d_%s_lo%d + 1)" % (
                    n, d + 1, n, d + 1)
                if d == nd - 2 and pitch > 1:
                    # rows padded to 16 bytes (row_pitch)
                    ext = "((%s + %d) / %d * %d)" % (ext, pitch - 1, pitch,
                                                     pitch)
                w("const long long s_%s_%d = s_%s_%d * %s;" % (
                    n, d, n, d + 1, ext))

    def gindex(self, f, args, ctx, clamp_dd=True, clamp_all=False):
        """Linear index into a dense array of ``f`` at index ASTs ``args``;
        data-dependent components are clamped into the domain."""
        n = self.fn(f)
        terms = []
        nd = len(args)
        # the innermost dimension has stride 1 unless the array is
        # reordered in memory (option storage_order)
        unit = self.storage_perm(f) is None
        for d, a in enumerate(args):
            s = ctx.index(a)
            if clamp_all or (clamp_dd and is_data_dependent(a)):
                s = "pm_clampi(%s, d_%s_lo%d, d_%s_hi%d)" % (s, n, d, n, d)
            if d == nd - 1 and unit:
                terms.append("(long long)(%s - d_%s_lo%d)" % (s, n, d))
            else:
                terms.append("(long long)(%s - d_%s_lo%d) * s_%s_%d" % (
                    s, n, d, n, d))
        return " + ".join(terms)

    def oob_guard(self, f, args, ctx):
        """Under option 'oob_zero': the C condition that a read of ``f``
        at ``args`` lies inside its domain along the dimensions the bounds
        check found it can leave (None when no guard is needed); the read
        yields 0 where the condition fails."""
        dims = getattr(self.p, '_oob_dims', {}).get(f)
        if not dims:
            return None
        n = self.fn(f)
        conds = []
        for d in sorted(dims):
            a = args[d]
            t = ctx.index(a) if not is_data_dependent(a) else \
                ctx.expr(a, {})
            conds.append("(%s) >= d_%s_lo%d && (%s) <= d_%s_hi%d" % (
                t, n, d, t, n, d))
        return " && ".join(conds)

    def host_text(self):
        if not self.hw.lines:
            return None
        return ("// const tables of pipeline %s -- generated by polymage_b200"
                "\n#include <cmath>\n#include <cstdlib>\n#include <cstring>"
                "\n#define isl_min(x,y) ((x) < (y) ? (x) : (y))\n"
                "#define isl_max(x,y) ((x) > (y) ? (x) : (y))\n"
                "static inline int pm_clampi(int v, int lo, int hi) "
                "{ return v < lo ? lo : (v > hi ? hi : v); }\n" %
                self.p.name) + self.hw.text()

    def gen_args_struct(self):
        w = self.w
        w.open("struct pm_args")
        for prm in self.params:
            w("%s %s;" % (self.ptype(prm), self.pmap[prm]))
        for f in self.inputs + self.outputs:
            w("void* b_%s;" % self.fn(f))
        w("char* ws;")
        w("char* ctab;")
        w.close("};")
        w("")

    # ---- per-call validation ------------------------------------------------
    def gen_validate(self):
        w = self.w
        ctx = ExprCtx(w, 'device', self.pmap, None)
        w("// Bounds checks of the spec, repeated for this call's parameters")
        w("// (a call whose references would leave a producer's domain is")
        w("// refused instead of reading out of bounds).")
        w.open("static int pm_validate(const pm_args& A)")
        self.declare_params(w, "A")
        for f in self.inputs + self.outputs:
            for d, (lo, hi) in enumerate(self.dom_exprs(f, ctx)):
                w("if ((long long)(%s) - (long long)(%s) + 1 < 0) "
                  "return PM_ERR_PARAMS;" % (hi, lo))
        checks = getattr(self.p, '_bounds_checks', [])
        seen = set()
        for (comp, box, arg, g, dim, is_target, restr) in checks:
            key = (id(comp), id(box), str(arg), id(g), dim,
                   tuple((id(v), k, r) for v, k, r in restr))
            if key in seen:
                continue
            seen.add(key)
            vs = [v for v in arg.collect(C.Variable)
                  if not isinstance(v, C.Parameter)]
            w.open("")
            ok = True
            for v in box.variables:
                los = [ctx.expr(e, {}) for e in box.lo[v]]
                his = [ctx.expr(e, {}) for e in box.hi[v]]
                lo = los[0]
                for x in los[1:]:
                    lo = "isl_max_i(%s, %s)" % (lo, x)
                hi = his[0]
                for x in his[1:]:
                    hi = "isl_min_i(%s, %s)" % (hi, x)
                for (rv, k, r) in restr:
                    if rv is v:
                        # the Select arm only runs on v = r (mod k)
                        lo = "pm_next_res(%s, %d, %d)" % (lo, k, r)
                        hi = "pm_prev_res(%s, %d, %d)" % (hi, k, r)
                w("const int %s_lo = %s, %s_hi = %s;" % (_vn(v), lo, _vn(v),
                                                          hi))
            empt = " || ".join("%s_lo > %s_hi" % (_vn(v), _vn(v))
                               for v in box.variables)
            w("bool empty = %s;" % (empt or "false"))
            lo_b = {}
            hi_b = {}
            for v in vs:
                dd = monotone_dir(arg, v)
                if dd is None:
                    ok = False
                    break
                if dd >= 0:
                    lo_b[v], hi_b[v] = _vn(v) + "_lo", _vn(v) + "_hi"
                else:
                    lo_b[v], hi_b[v] = _vn(v) + "_hi", _vn(v) + "_lo"
            if ok:
                glo = ctx.expr(g.domain[dim].lowerBound, {})
                ghi = ctx.expr(g.domain[dim].upperBound, {})
                a_lo = ctx.expr(arg, lo_b)
                a_hi = ctx.expr(arg, hi_b)
                w("if (!empty && ((%s) < (%s) || (%s) > (%s))) return "
                  "PM_ERR_PARAMS;" % (a_lo, glo, a_hi, ghi))
            w.close()
        w("return PM_OK;")
        w.close()
        w("")

    # ---- workspace layout -----------------------------------------------------
    def gen_workspace(self):
        w = self.w
        ctx = ExprCtx(w, 'device', self.pmap, None)
        slots = getattr(self.p, '_storage_slots', [])
        self.slot_of = getattr(self.p, '_storage_assign', {})
        w("// Intermediate arrays: one slot per storage class occupant chain,")
        w("// sized per call (bytes = max over the slot's occupants).")
        w.open("static void pm_ws_layout(const pm_args& A, size_t* off, "
               "size_t* total)")
        self.declare_params(w, "A")
        w("size_t o = 0;")
        for i, occ in enumerate(slots):
            w("{ size_t b = 0;")
            for comp in occ:
                f = comp.func
                exts = ["(size_t)pm_nonneg((%s) - (%s) + 1)" % (
                    ctx.expr(d.upperBound, {}), ctx.expr(d.lowerBound, {}))
                    for d in f.domain]
                pitch = self.row_pitch(f)
                if pitch > 1:
                    exts[-1] = "((%s + %d) / %d * %d)" % (
                        exts[-1], pitch - 1, pitch, pitch)
                ext = " * ".join(exts)
                w("  { size_t e = (size_t)%d * %s; if (e > b) b = e; }" % (
                    f.typ.size(), ext))
            w("  off[%d] = o; o += pm_align256(b); }" % i)
        w("*total = o;")
        w.close()
        w("")
        self.nslots = len(slots)

    def buf_expr(self, f, src="A"):
        """C expression of the device pointer of a full array."""
        if any(f is x for x in self.inputs + self.outputs):
            return "%s.b_%s" % (src, self.fn(f))
        comp = self.p.func_map.get(f)
        if comp is not None and comp in self.slot_of:
            return "(%s.ws + wsoff[%d])" % (src, self.slot_of[comp])
        if f.is_const_func:
            return "ctab_ptr_%s" % self.fn(f)
        raise CodegenError("no buffer for %s" % f.name)

    def buf_key(self, f):
        """Identity of the HBM buffer holding ``f`` (None for stages kept
        in shared memory or registers)."""
        if any(f is x for x in self.inputs):
            return ('in', id(f))
        if any(f is x for x in self.outputs):
            return ('out', id(f))
        comp = self.p.func_map.get(f)
        if comp is not None and comp in self.slot_of:
            return ('slot', self.slot_of[comp])
        if getattr(f, 'is_const_func', False):
            return ('ctab', id(f))
        return None

    def group_rw(self, g):
        """(buffers read, buffers written) by one group's launch."""
        from .pipe import body_refs
        funcs = [c.func for c in g.comps]
        ids = set(id(f) for f in funcs)
        reads, writes = set(), set()
        for f in funcs:
            k = self.buf_key(f)
            if k is not None:
                writes.add(k)
            for r in body_refs(f):
                x = r.objectRef
                if id(x) in ids:
                    continue
                k = self.buf_key(x)
                if k is not None:
                    reads.add(k)
        return reads, writes

    def schedule(self, batch=False):
        """(stream of each launch, waits, recorded launches) of the
        concurrent schedule (polymage_b200.streams).  ``batch``: the
        batched entries' launches, one per group (no chains)."""
        key = '_bsched' if batch else '_sched'
        if getattr(self, key, None) is None:
            from . import streams
            nst = int(_opt(self.p, 'streams', DEFAULT_STREAMS))
            rw, main = (self.group_launch_rw, self.group_launch_main) \
                if batch else (self.launch_rw, self.launch_main)
            setattr(self, key, streams.schedule(rw, nst, main_only=main))
        return getattr(self, key)

    def emit_calls(self, w, calls, ret, batch=False):
        """Every group's launch in program order, spread over concurrent
        streams when groups are independent.  ``calls[j]``: the C call of
        launch j with ``{s}`` where its stream goes (it returns a status);
        ``ret``: the statement that returns a failed ``st``.  The caller's
        stream ``s`` forks to the side streams first and joins them at the
        end, also when a launch fails.  ``batch``: the calls are the
        batched entries' per-group launches."""
        sof, waits, records = self.schedule(batch)
        used = sorted(set(sof) - {0})
        if not used:
            for c in calls:
                w("if ((st = %s)) %s" % (c.format(s="s"), ret))
            return
        ev = {}
        for i in sorted(records):
            ev[i] = len(ev) + 1
        join = dict((k, len(ev) + 1 + n) for n, k in enumerate(used))
        nev = 1 + len(ev) + len(used)
        self.conc_streams = max(self.conc_streams, max(used))
        self.conc_events = max(self.conc_events, nev)
        w("// %d launches on %d streams: independent groups run "
          "concurrently" % (len(sof), len(used) + 1))
        w.open("")
        w("cudaStream_t ss[%d]; ss[0] = s;" % (max(used) + 1))
        w("cudaEvent_t* ev = nullptr;")
        w("if ((st = pm_conc_get(ss, %d, %d, &ev))) %s" % (max(used), nev,
                                                          ret))
        w("if (cudaEventRecord(ev[0], s) != cudaSuccess) { st = "
          "PM_ERR_CUDA; %s }" % ret)
        for k in used:
            w("if (cudaStreamWaitEvent(ss[%d], ev[0], 0) != cudaSuccess) { st "
              "= PM_ERR_CUDA; %s }" % (k, ret))
        w.open("do")
        for j, c in enumerate(calls):
            for i in waits[j]:
                w("if (cudaStreamWaitEvent(ss[%d], ev[%d], 0) != cudaSuccess)"
                  " { st = PM_ERR_CUDA; break; }" % (sof[j], ev[i]))
            w("if ((st = %s)) break;" % c.format(s="ss[%d]" % sof[j]))
            if j in records:
                w("if (cudaEventRecord(ev[%d], ss[%d]) != cudaSuccess) "
                  "{ st = PM_ERR_CUDA; break; }" % (ev[j], sof[j]))
        w.close("} while (0);")
        w("// join: the caller's stream follows every side stream")
        for k in used:
            w("if (cudaEventRecord(ev[%d], ss[%d]) != cudaSuccess || "
              "cudaStreamWaitEvent(s, ev[%d], 0) != cudaSuccess) st = st ? "
              "st : PM_ERR_CUDA;" % (join[k], k, join[k]))
        w("if (st) %s" % ret)
        w.close()

    # ---- entry points -----------------------------------------------------------
    def abi_params(self):
        ps = ["%s %s" % (self.ptype(q), q.name) for q in self.params]
        ps += ["void* %s" % f.name for f in self.inputs]
        ps += ["void* %s" % f.name for f in self.outputs]
        return ps

    def gen_entries(self):
        w = self.w
        name = self.pname
        w("static pm_arena pm_ws_arena;")
        w("static pm_arena pm_ctab_arena;")
        w("")
        # ---- single image, device pointers ----
        w.open("static int pm_run(pm_args& A, cudaStream_t s)")
        w("int st = pm_validate(A);")
        w("if (st) return st;")
        w("size_t wsoff[%d + 1]; size_t wstotal = 0;" % max(self.nslots, 1))
        w("pm_ws_layout(A, wsoff, &wstotal);")
        w("void* ws = nullptr;")
        w("if ((st = pm_arena_get(&pm_ws_arena, wstotal, &ws))) return st;")
        w("A.ws = (char*)ws;")
        self.emit_calls(w, ["%s(A, wsoff, {s})" % f for f in self.launch_fns],
                        "return st;")
        w("return PM_OK;")
        w.close()
        w("")
        sig = ", ".join(self.abi_params())
        call_fill = []
        for q in self.params:
            call_fill.append("A.%s = %s;" % (self.pmap[q], q.name))
        for f in self.inputs + self.outputs:
            call_fill.append("A.b_%s = %s;" % (self.fn(f), f.name))
        w.open('extern "C" int pipeline_%s_dev(%s, void* stream)' % (name,
                                                                    sig))
        w("pm_args A; memset(&A, 0, sizeof(A));")
        for line in call_fill:
            w(line)
        w("pm_status = pm_run(A, (cudaStream_t)stream);")
        w("return pm_status;")
        w.close()
        w("")
        # ---- graph replay ----
        w("// per device: the graph, its arguments, workspace and stream")
        w("static cudaGraphExec_t pm_graph_exec[64];")
        w("static pm_args pm_graph_key[64];")
        w("static void* pm_graph_ws[64];")
        w("static cudaStream_t pm_graph_stream[64];")
        w("// Replays a CUDA graph of the whole pipeline; the graph is")
        w("// (re)captured when the arguments or the workspace change.")
        w.open('extern "C" int pipeline_%s_graph(%s, void* stream)' % (name,
                                                                      sig))
        if any(img for _, img in self.const_replay):
            w("// a const table is computed on the host from input image")
            w("// contents, which a captured graph would not see change")
            for q in self.params:
                w("(void)%s;" % q.name)
            for f in self.inputs + self.outputs:
                w("(void)%s;" % f.name)
            w("(void)stream;")
            w("return pm_status = PM_ERR_UNSUPPORTED;")
            w.close()
            w("")
            return self._gen_entries_tail(sig, call_fill)
        w("pm_args A; memset(&A, 0, sizeof(A));")
        for line in call_fill:
            w(line)
        w("const int dev = pm_cur_dev();")
        w("void* wsnow = pm_ws_arena.ptr[dev];")
        w.open("if (!pm_graph_exec[dev] || wsnow != pm_graph_ws[dev] || "
               "memcmp(&A, &pm_graph_key[dev], sizeof(A)) != 0)")
        w("pm_args B = A;")
        w("int st = pm_run(B, (cudaStream_t)stream);  // sizes workspace, "
          "uploads tables")
        w("if (st) return pm_status = st;")
        w("if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) "
          "return pm_status = PM_ERR_CUDA;")
        w("if (!pm_graph_stream[dev] && cudaStreamCreateWithFlags("
          "&pm_graph_stream[dev], cudaStreamNonBlocking) != cudaSuccess) "
          "return pm_status = PM_ERR_CUDA;")
        w("if (pm_graph_exec[dev]) { cudaGraphExecDestroy("
          "pm_graph_exec[dev]); pm_graph_exec[dev] = nullptr; }")
        w("cudaGraph_t g = nullptr;")
        w("if (cudaStreamBeginCapture(pm_graph_stream[dev], "
          "cudaStreamCaptureModeThreadLocal) != cudaSuccess) return "
          "pm_status = PM_ERR_CUDA;")
        w("pm_args Cc = A;")
        w("st = pm_run(Cc, pm_graph_stream[dev]);")
        w("cudaError_t e = cudaStreamEndCapture(pm_graph_stream[dev], &g);")
        w("if (st || e != cudaSuccess) { if (g) cudaGraphDestroy(g); "
          "cudaGetLastError(); return pm_status = st ? st : PM_ERR_CUDA; }")
        w("e = cudaGraphInstantiate(&pm_graph_exec[dev], g, 0);")
        w("cudaGraphDestroy(g);")
        w("if (e != cudaSuccess) { pm_graph_exec[dev] = nullptr; return "
          "pm_status = PM_ERR_CUDA; }")
        w("pm_graph_key[dev] = A;")
        w("pm_graph_ws[dev] = pm_ws_arena.ptr[dev];")
        w.close()
        w("if (cudaGraphLaunch(pm_graph_exec[dev], (cudaStream_t)stream) != "
          "cudaSuccess) return pm_status = PM_ERR_CUDA;")
        w("return pm_status = PM_OK;")
        w.close()
        w("")
        self._gen_entries_tail(sig, call_fill)

    def _gen_entries_tail(self, sig, call_fill):
        w = self.w
        name = self.pname
        # ---- host pointers (the reference's ABI) ----
        self.gen_host_entry(sig, call_fill)
        # ---- batch ----
        self.gen_batch_entry()
        # ---- status ----
        w('extern "C" int pipeline_%s_status(void) { return pm_status; }'
          % name)
        w.open('extern "C" int pipeline_%s_check(void)' % name)
        w("unsigned v = 0;")
        w("if (cudaDeviceSynchronize() != cudaSuccess) return PM_ERR_CUDA;")
        w("if (cudaMemcpyFromSymbol(&v, pm_err_word, sizeof(v)) != "
          "cudaSuccess) return PM_ERR_CUDA;")
        w("return v ? PM_ERR_KERNEL : PM_OK;")
        w.close()
        w('extern "C" void pipeline_%s_clear_error(void) { unsigned z = 0; '
          'cudaMemcpyToSymbol(pm_err_word, &z, sizeof(z)); pm_status = 0; }'
          % name)
        w("")

    def gen_host_entry(self, sig, call_fill):
        w = self.w
        name = self.pname
        ctx = ExprCtx(w, 'device', self.pmap, None)
        nin, nout = len(self.inputs), len(self.outputs)
        w("static pm_arena pm_host_in[%d];" % max(nin, 1))
        w("static pm_arena pm_host_out[%d];" % max(nout, 1))
        w("static cudaStream_t pm_host_stream[64];")
        if self.band_group() is not None:
            w("// row-band overlap of copies and compute (host entry)")
            w("#define PM_MAX_BANDS 128")
            w("static cudaStream_t pm_band_in[64], pm_band_out[64];")
            w("static cudaEvent_t pm_band_ev[64][PM_MAX_BANDS * 2 + 1];")
            w("static bool pm_band_ready[64];")
            w("// bands to aim for: PM_HOST_BANDS (0 disables banding), else 12")
            w.open("static int pm_target_bands()")
            w("static int v = -1;")
            w("if (v < 0) { const char* e = getenv(\"PM_HOST_BANDS\"); "
              "v = e ? atoi(e) : 12; if (v < 0) v = 0; if (v > 64) v = 64; }")
            w("return v;")
            w.close()
        w.open('extern "C" void pipeline_%s(%s)' % (name, sig))
        w("pm_args A; memset(&A, 0, sizeof(A));")
        for line in call_fill:
            w(line)
        w("int dev = 0; cudaGetDevice(&dev);")
        w("if (dev < 0 || dev >= 64) { pm_status = PM_ERR_CUDA; return; }")
        w("if (!pm_host_stream[dev] && cudaStreamCreateWithFlags("
          "&pm_host_stream[dev], cudaStreamNonBlocking) != cudaSuccess) "
          "{ pm_status = PM_ERR_CUDA; return; }")
        w("cudaStream_t s = pm_host_stream[dev];")
        self.declare_params(w, "A")
        w("int st = pm_validate(A);")
        w("if (st) { pm_status = st; return; }")
        for i, f in enumerate(self.inputs + self.outputs):
            n = self.fn(f)
            arena = "pm_host_in[%d]" % i if i < nin else \
                "pm_host_out[%d]" % (i - nin)
            ext = " * ".join("(size_t)pm_nonneg((%s) - (%s) + 1)" % (hi, lo)
                             for lo, hi in self.dom_exprs(f, ctx))
            w("const size_t nb_%s = (size_t)%d * %s;" % (n, f.typ.size(), ext))
            w("void* dv_%s = nullptr;" % n)
            w("if (pm_arena_get(&%s, nb_%s, &dv_%s)) { pm_status = "
              "PM_ERR_CUDA; return; }" % (arena, n, n))
        sg = self.band_group()
        if sg is not None:
            self.gen_banded(sg, ctx)
        for f in self.inputs:
            n = self.fn(f)
            w("if (nb_%s && cudaMemcpyAsync(dv_%s, %s, nb_%s, "
              "cudaMemcpyHostToDevice, s) != cudaSuccess) { pm_status = "
              "PM_ERR_CUDA; return; }" % (n, n, f.name, n))
        for f in self.outputs:
            n = self.fn(f)
            box = self.written_box(f)
            if box is None:
                # coverage is not a box: keep the caller's untouched points
                w("if (nb_%s && cudaMemcpyAsync(dv_%s, %s, nb_%s, "
                  "cudaMemcpyHostToDevice, s) != cudaSuccess) { pm_status = "
                  "PM_ERR_CUDA; return; }" % (n, n, f.name, n))
        for f in self.inputs + self.outputs:
            n = self.fn(f)
            w("A.b_%s = dv_%s;" % (n, n))
        w("st = pm_run(A, s);")
        w("if (st) { pm_status = st; cudaStreamSynchronize(s); return; }")
        for f in self.outputs:
            self.gen_d2h(f, ctx)
        w("if (cudaStreamSynchronize(s) != cudaSuccess) { pm_status = "
          "PM_ERR_CUDA; return; }")
        w("unsigned kerr = 0;")
        w("cudaMemcpyFromSymbol(&kerr, pm_err_word, sizeof(kerr));")
        w("pm_status = kerr ? PM_ERR_KERNEL : PM_OK;")
        w.close()
        w("")

    def band_group(self):
        """The stencil group of a pipeline that the host entry can run in
        row bands: the pipeline is that one group (no reductions, no const
        tables), its anchor is the pipeline's only output, and the output's
        written points form a box."""
        if len(self.launch_fns) != 1 or len(self.band_groups) != 1 or \
                len(self.outputs) != 1 or self.const_ptrs:
            return None
        sg = self.band_groups[0]
        out = self.outputs[0]
        if sg.plan.anchor is not out or out.ndims < 2 or \
                self.written_box(out) is None:
            return None
        return sg

    def gen_banded(self, sg, ctx):
        """Host buffers in pinned memory: split the tile grid into row bands
        and overlap, on three streams, the input copy of the next band, the
        kernel on this band and the output copy of the previous band.  A
        band's input need is the prefix of each input up to the largest
        offset its corner tiles read (footprints are monotone in the tile
        coordinates); its output copy is the written box clipped to the
        band's anchor region."""
        w = self.w
        k = sg.k
        plan = sg.plan
        na = plan.anchor.ndims
        nin = len(self.inputs)
        out = self.outputs[0]
        w("bool pm_band = pm_target_bands() > 0 && (%s) >= ((size_t)16 << 20);" %
          " + ".join("nb_%s" % self.fn(f) for f in self.inputs + self.outputs))
        w.open("if (pm_band)")
        w("cudaPointerAttributes pa;")
        for f in self.inputs + self.outputs:
            w("if (cudaPointerGetAttributes(&pa, %s) != cudaSuccess || pa.type "
              "!= cudaMemoryTypeHost) { pm_band = false; cudaGetLastError(); }"
              % f.name)
        w.close()
        w("%s_launch L; memset(&L, 0, sizeof(L));" % k)
        w("L.nimg = 1;")
        w("long long nt = 0, nrow = 0, ninner = 0, nouter = 0;")
        w.open("if (pm_band)")
        for f in self.inputs + self.outputs:
            n = self.fn(f)
            w("A.b_%s = dv_%s;" % (n, n))
        w("size_t wsoff[%d + 1]; size_t wstotal = 0;" % max(self.nslots, 1))
        w("pm_ws_layout(A, wsoff, &wstotal);")
        w("void* ws = nullptr;")
        w("if (pm_arena_get(&pm_ws_arena, wstotal, &ws)) { pm_status = "
          "PM_ERR_CUDA; return; }")
        w("A.ws = (char*)ws;")
        w("if ((st = fill_%s(L.d0, A, wsoff, &nt))) { pm_status = st; return; }"
          % k)
        w("nrow = L.d0.gn[%d]; ninner = L.d0.gn[%d];" % (na - 2, na - 1))
        w("nouter = (nrow && ninner) ? nt / (nrow * ninner) : 0;")
        w("if (nt == 0 || nt > 0x7fffffffLL || nouter > 40) pm_band = false;")
        w.close()
        w.open("if (pm_band)")
        w("const %s_desc& D = L.d0;" % k)
        w.open("if (!pm_band_ready[dev])")
        w("if (cudaStreamCreateWithFlags(&pm_band_in[dev], "
          "cudaStreamNonBlocking) != cudaSuccess || cudaStreamCreateWithFlags("
          "&pm_band_out[dev], cudaStreamNonBlocking) != cudaSuccess) "
          "{ pm_status = PM_ERR_CUDA; return; }")
        w("for (int i = 0; i < PM_MAX_BANDS * 2 + 1; ++i) if (cudaEventCreate"
          "WithFlags(&pm_band_ev[dev][i], cudaEventDisableTiming) != "
          "cudaSuccess) { pm_status = PM_ERR_CUDA; return; }")
        w("pm_band_ready[dev] = true;")
        w.close()
        w("cudaStream_t sin = pm_band_in[dev], sout = pm_band_out[dev];")
        w.open("if (!%s_attr[pm_cur_dev()])" % k)
        w("if (cudaFuncSetAttribute(%s, cudaFuncAttributeMaxDynamicShared"
          "MemorySize, %d) != cudaSuccess) { pm_status = PM_ERR_CUDA; "
          "return; }" % (k, plan.smem_bytes))
        w("%s_attr[pm_cur_dev()] = true;" % k)
        w.close()
        w("// the kernel's first band must not start before earlier work on s")
        w("cudaEventRecord(pm_band_ev[dev][PM_MAX_BANDS * 2], s);")
        w("cudaStreamWaitEvent(sin, pm_band_ev[dev][PM_MAX_BANDS * 2], 0);")
        w("cudaStreamWaitEvent(sout, pm_band_ev[dev][PM_MAX_BANDS * 2], 0);")
        w("long long rb = (nrow * nouter + pm_target_bands() - 1) / "
          "pm_target_bands();")
        w("if (rb < 1) rb = 1;")
        w("if (rb > nrow) rb = nrow;")
        w("size_t copied[%d] = {0};" % max(nin, 1))
        w("int bi = 0;")
        w.open("for (long long o = 0; o < nouter; ++o)")
        w.open("for (long long a = 0; a < nrow; a += rb)")
        w("const long long b = a + rb < nrow ? a + rb : nrow;")
        w("const long long tf = (o * nrow + a) * ninner, tl = (o * nrow + b) "
          "* ninner;")
        w("long long need[%d] = {0};" % max(nin, 1))
        w("int blo[%d], bhi[%d];" % (na, na))
        w("for (int d = 0; d < %d; ++d) { blo[d] = 0x3fffffff; bhi[d] = "
          "-0x3fffffff; }" % na)
        w("const long long corner[4] = {tf, tf + ninner - 1, tl - ninner, "
          "tl - 1};")
        w.open("for (int c = 0; c < 4; ++c)")
        w("long long e[%d]; int alo[%d], ahi[%d];" % (max(nin, 1), na, na))
        w("%s_footprint(D, (int)corner[c], e, alo, ahi);" % k)
        w("for (int j = 0; j < %d; ++j) if (e[j] > need[j]) need[j] = e[j];"
          % nin)
        w("for (int d = 0; d < %d; ++d) { blo[d] = pm_imin(blo[d], alo[d]); "
          "bhi[d] = pm_imax(bhi[d], ahi[d]); }" % na)
        w.close()
        for j, f in enumerate(self.inputs):
            n = self.fn(f)
            w.open("")
            w("size_t nb = (size_t)need[%d] * %d;" % (j, f.typ.size()))
            w("if (nb > nb_%s) nb = nb_%s;" % (n, n))
            w("if (nb > copied[%d] && cudaMemcpyAsync((char*)dv_%s + copied[%d],"
              " (const char*)%s + copied[%d], nb - copied[%d], "
              "cudaMemcpyHostToDevice, sin) != cudaSuccess) { pm_status = "
              "PM_ERR_CUDA; return; }" % (j, n, j, f.name, j, j))
            w("if (nb > copied[%d]) copied[%d] = nb;" % (j, j))
            w.close()
        w("if (bi >= PM_MAX_BANDS) { cudaStreamSynchronize(s); pm_status = "
          "PM_ERR_UNSUPPORTED; return; }")
        w("cudaEvent_t ein = pm_band_ev[dev][2 * bi], ek = "
          "pm_band_ev[dev][2 * bi + 1];")
        w("if (cudaEventRecord(ein, sin) != cudaSuccess || "
          "cudaStreamWaitEvent(s, ein, 0) != cudaSuccess) { pm_status = "
          "PM_ERR_CUDA; return; }")
        w("L.first = (int)tf; L.total = (int)tl; L.queue = nullptr;")
        w("%s<<<(unsigned)(tl - tf), %d, %d, s>>>(L);" % (k, plan.threads,
                                                         plan.smem_bytes))
        w("if (cudaGetLastError() != cudaSuccess || cudaEventRecord(ek, s) != "
          "cudaSuccess || cudaStreamWaitEvent(sout, ek, 0) != cudaSuccess) "
          "{ pm_status = PM_ERR_CUDA; return; }")
        clip = [("blo[%d]" % d, "bhi[%d]" % d) for d in range(na)]
        self.gen_d2h(out, ctx, stream="sout",
                     fail="{ pm_status = PM_ERR_CUDA; return; }", clip=clip)
        w("++bi;")
        w.close()
        w.close()
        w("if (cudaEventRecord(pm_band_ev[dev][PM_MAX_BANDS * 2], sout) != "
          "cudaSuccess || cudaStreamWaitEvent(s, pm_band_ev[dev][PM_MAX_BANDS "
          "* 2], 0) != cudaSuccess) { pm_status = PM_ERR_CUDA; return; }")
        w("if (cudaStreamSynchronize(s) != cudaSuccess) { pm_status = "
          "PM_ERR_CUDA; return; }")
        w("unsigned kerr = 0;")
        w("cudaMemcpyFromSymbol(&kerr, pm_err_word, sizeof(kerr));")
        w("pm_status = kerr ? PM_ERR_KERNEL : PM_OK;")
        w("return;")
        w.close()

    def written_box(self, f):
        """Per-dim (lo, hi) expressions of the points of output ``f`` that
        the pipeline writes, when they form a box; None otherwise."""
        parts = part_boxes(f)
        if not parts or any(not b.exact for b, _, _, _ in parts):
            return None
        env = self.p.int_env()
        try:
            vals = [b.evaluate(env) for b, _, _, _ in parts]
        except Exception:
            return None
        vs = f.variables
        if len(parts) > 1:
            # union is a box when all parts agree except on one dim where
            # their intervals are disjoint and contiguous
            diff = [v for v in vs if len(set(val[v] for val in vals)) > 1]
            if len(diff) > 1:
                return None
            if diff:
                v = diff[0]
                iv = sorted(val[v] for val in vals)
                for (a0, a1), (b0, b1) in zip(iv, iv[1:]):
                    if b0 != a1 + 1:
                        return None
        out = []
        for d, v in enumerate(vs):
            los, his = [], []
            for b, _, _, _ in parts:
                lo = b.lo[v][0]
                for e in b.lo[v][1:]:
                    lo = C.Max(lo, e, typeCheck=False)
                hi = b.hi[v][0]
                for e in b.hi[v][1:]:
                    hi = C.Min(hi, e, typeCheck=False)
                los.append(lo)
                his.append(hi)
            lo = los[0]
            for e in los[1:]:
                lo = C.Min(lo, e, typeCheck=False)
            hi = his[0]
            for e in his[1:]:
                hi = C.Max(hi, e, typeCheck=False)
            out.append((lo, hi))
        return out

    def gen_d2h(self, f, ctx, stream="s",
                fail="{ pm_status = PM_ERR_CUDA; return; }", clip=None):
        """Copy the written points of output ``f`` back to the caller's
        buffer (pm_copy_box_d2h: contiguous spans where the box covers
        the inner dimensions whole, 2-D copies otherwise); ``clip`` optionally
        intersects the written box with per-dim (lo, hi) C expressions."""
        w = self.w
        n = self.fn(f)
        box = self.written_box(f)
        es = f.typ.size()
        if box is None:
            w("if (nb_%s && cudaMemcpyAsync(%s, dv_%s, nb_%s, "
              "cudaMemcpyDeviceToHost, %s) != cudaSuccess) %s" % (
                  n, f.name, n, n, stream, fail))
            return
        nd = len(f.domain)
        w.open("")
        for d, dom in enumerate(f.domain):
            w("const long long D%d_lo = %s, D%d_hi = %s;" % (
                d, ctx.expr(dom.lowerBound, {}), d,
                ctx.expr(dom.upperBound, {})))
            lo = "pm_llmax(D%d_lo, %s)" % (d, ctx.expr(box[d][0], {}))
            hi = "pm_llmin(D%d_hi, %s)" % (d, ctx.expr(box[d][1], {}))
            if clip is not None:
                lo = "pm_llmax(%s, (long long)(%s))" % (lo, clip[d][0])
                hi = "pm_llmin(%s, (long long)(%s))" % (hi, clip[d][1])
            w("const long long B%d_lo = %s, B%d_hi = %s;" % (d, lo, d, hi))
        w("long long Dl[%d] = {%s}, Dh[%d] = {%s};" % (
            nd, ", ".join("D%d_lo" % d for d in range(nd)), nd,
            ", ".join("D%d_hi" % d for d in range(nd))))
        w("long long Bl[%d] = {%s}, Bh[%d] = {%s};" % (
            nd, ", ".join("B%d_lo" % d for d in range(nd)), nd,
            ", ".join("B%d_hi" % d for d in range(nd))))
        w("if (pm_copy_box_d2h(%s, dv_%s, %d, %d, Dl, Dh, Bl, Bh, %s)) %s" % (
            f.name, n, es, nd, stream, fail))
        w.close()

    def gen_batch_entry(self):
        w = self.w
        name = self.pname
        nin, nout = len(self.inputs), len(self.outputs)
        w("static pm_arena pm_batch_arena;")
        w("static char* pm_batch_pinned = nullptr;")
        w("static size_t pm_batch_pinned_cap = 0;")
        w("// Batched execution: n images (each with its own parameters) run")
        w("// through each group in one launch; a CTA maps its block index to")
        w("// (image, tile) through the per-image tile prefix.")
        w("// A call repeating the previous call's arguments (same images,")
        w("// parameters and workspace) relaunches the kernels with the")
        w("// descriptors already on the device: no host copies, so it can be")
        w("// captured in a CUDA graph (pipeline_<name>_batch_graph).")
        w("static std::vector<char> pm_batch_key;")
        w("static void* pm_batch_ws = nullptr;")
        image_tables = any(img for _, img in self.const_replay)
        w("// const tables still those the last batch uploaded (a single-image")
        w("// call in between may have replaced them)")
        w.open("static bool pm_batch_tables_current()")
        if image_tables:
            w("return false;   // a table depends on input image contents")
        else:
            for fnm, _ in self.const_replay:
                w("if (ctab_key_%s != pm_bctab_key_%s || ctab_ptr_%s != "
                  "pm_bctab_ptr_%s) return false;" % (fnm, fnm, fnm, fnm))
            w("return true;")
        w.close()
        w.open('extern "C" int pipeline_%s_batch(int n, const int* iparams, '
               'const float* fparams, void* const* inputs, void* const* '
               'outputs, void* stream)' % name)
        w("cudaStream_t s = (cudaStream_t)stream;")
        w("if (n <= 0) return pm_status = PM_OK;")
        w("std::vector<char> key;")
        w("pm_key_add(key, &n, sizeof(n));")
        w("pm_key_add(key, iparams, sizeof(int) * (size_t)n * %d);" %
          len(self.iparams))
        w("pm_key_add(key, fparams, sizeof(float) * (size_t)n * %d);" %
          len(self.fparams))
        w("pm_key_add(key, inputs, sizeof(void*) * (size_t)n * %d);" % nin)
        w("pm_key_add(key, outputs, sizeof(void*) * (size_t)n * %d);" % nout)
        w("const int dev = pm_cur_dev();")
        w.open("if (key == pm_batch_key && pm_batch_ws && "
               "pm_batch_arena.ptr[dev] == pm_batch_ws && "
               "pm_batch_tables_current())")
        w("int st = 0;")
        self.emit_calls(w, ["%s(nullptr, nullptr, 0, n, nullptr, nullptr, "
                            "nullptr, {s}, 1)" % f for f in self.batch_fns],
                        "return pm_status = st;", batch=True)
        w("return pm_status = PM_OK;")
        w.close()
        w("pm_batch_key.clear(); pm_batch_ws = nullptr;")
        w("std::vector<pm_args> As(n);")
        w("std::vector<size_t> wsoffs((size_t)n * %d);" % max(self.nslots, 1))
        w("size_t total = 0;")
        w.open("for (int i = 0; i < n; ++i)")
        w("pm_args& A = As[i]; memset(&A, 0, sizeof(A));")
        for j, q in enumerate(self.iparams):
            w("A.%s = iparams[(size_t)i * %d + %d];" % (
                self.pmap[q], len(self.iparams), j))
        for j, q in enumerate(self.fparams):
            w("A.%s = fparams[(size_t)i * %d + %d];" % (
                self.pmap[q], len(self.fparams), j))
        for j, f in enumerate(self.inputs):
            w("A.b_%s = inputs[(size_t)i * %d + %d];" % (self.fn(f), nin, j))
        for j, f in enumerate(self.outputs):
            w("A.b_%s = outputs[(size_t)i * %d + %d];" % (self.fn(f), nout,
                                                          j))
        w("int st = pm_validate(A); if (st) return pm_status = st;")
        w("size_t t = 0; pm_ws_layout(A, &wsoffs[(size_t)i * %d], &t);" %
          max(self.nslots, 1))
        w("for (int k = 0; k < %d; ++k) wsoffs[(size_t)i * %d + k] += total;"
          % (self.nslots, max(self.nslots, 1)))
        w("total += pm_align256(t);")
        w.close()
        w("size_t descs_bytes = pm_batch_desc_bytes(n);")
        w("void* ws = nullptr;")
        w("if (pm_arena_get(&pm_batch_arena, total + descs_bytes, &ws)) "
          "return pm_status = PM_ERR_CUDA;")
        w("for (int i = 0; i < n; ++i) As[i].ws = (char*)ws;")
        w("char* ddesc = (char*)ws + total;")
        w("if (!pm_batch_event[dev] && cudaEventCreateWithFlags("
          "&pm_batch_event[dev], cudaEventDisableTiming) != cudaSuccess) "
          "return pm_status = PM_ERR_CUDA;")
        w("cudaEventSynchronize(pm_batch_event[dev]);  // previous upload "
          "done")
        w.open("if (pm_batch_pinned_cap < descs_bytes)")
        w("if (pm_batch_pinned) cudaFreeHost(pm_batch_pinned);")
        w("pm_batch_pinned = nullptr; pm_batch_pinned_cap = 0;")
        w("if (cudaMallocHost((void**)&pm_batch_pinned, descs_bytes) != "
          "cudaSuccess) return pm_status = PM_ERR_CUDA;")
        w("pm_batch_pinned_cap = descs_bytes;")
        w.close()
        w("size_t doff = 0; int st = 0;")
        self.emit_calls(w, ["%s(As.data(), wsoffs.data(), %d, n, "
                            "pm_batch_pinned, ddesc, &doff, {s}, 0)" % (
                                f, max(self.nslots, 1))
                            for f in self.batch_fns],
                        "return pm_status = st;", batch=True)
        w("// the pinned descriptors are free once every stream's upload is")
        w("cudaEventRecord(pm_batch_event[dev], s);")
        w("pm_batch_key = key; pm_batch_ws = ws;")
        w("return pm_status = PM_OK;")
        w.close()
        w("")
        w("// per device: the batch graph, its arguments, workspace, stream")
        w("static cudaGraphExec_t pm_bgraph_exec[64];")
        w("static std::vector<char> pm_bgraph_key[64];")
        w("static void* pm_bgraph_ws[64];")
        w("static cudaStream_t pm_bgraph_stream[64];")
        w("// The batch as one CUDA graph: captured on first use (after one")
        w("// ordinary call has sized the workspace and uploaded descriptors),")
        w("// re-captured when the arguments change.")
        w.open('extern "C" int pipeline_%s_batch_graph(int n, const int* '
               'iparams, const float* fparams, void* const* inputs, void* '
               'const* outputs, void* stream)' % name)
        if image_tables:
            w("// a const table is computed on the host from input image")
            w("// contents, which a captured graph would not see change")
            w("return pm_status = PM_ERR_UNSUPPORTED;")
            w.close()
            w("")
            return
        w("cudaStream_t s = (cudaStream_t)stream;")
        w("std::vector<char> key;")
        w("pm_key_add(key, &n, sizeof(n));")
        w("pm_key_add(key, iparams, sizeof(int) * (size_t)n * %d);" %
          len(self.iparams))
        w("pm_key_add(key, fparams, sizeof(float) * (size_t)n * %d);" %
          len(self.fparams))
        w("pm_key_add(key, inputs, sizeof(void*) * (size_t)n * %d);" % nin)
        w("pm_key_add(key, outputs, sizeof(void*) * (size_t)n * %d);" % nout)
        w("const int dev = pm_cur_dev();")
        w("void* wsnow = pm_batch_arena.ptr[dev];")
        w.open("if (!pm_bgraph_exec[dev] || key != pm_bgraph_key[dev] || "
               "wsnow != pm_bgraph_ws[dev] || !pm_batch_tables_current())")
        w("int st = pipeline_%s_batch(n, iparams, fparams, inputs, outputs, "
          "stream);" % name)
        w("if (st) return st;")
        w("if (cudaStreamSynchronize(s) != cudaSuccess) return pm_status = "
          "PM_ERR_CUDA;")
        w("if (!pm_bgraph_stream[dev] && cudaStreamCreateWithFlags("
          "&pm_bgraph_stream[dev], cudaStreamNonBlocking) != cudaSuccess) "
          "return pm_status = PM_ERR_CUDA;")
        w("if (pm_bgraph_exec[dev]) { cudaGraphExecDestroy("
          "pm_bgraph_exec[dev]); pm_bgraph_exec[dev] = nullptr; }")
        w("cudaGraph_t g = nullptr;")
        w("if (cudaStreamBeginCapture(pm_bgraph_stream[dev], "
          "cudaStreamCaptureModeThreadLocal) != cudaSuccess) return "
          "pm_status = PM_ERR_CUDA;")
        w("st = pipeline_%s_batch(n, iparams, fparams, inputs, outputs, "
          "pm_bgraph_stream[dev]);   // replays: kernels only" % name)
        w("cudaError_t e = cudaStreamEndCapture(pm_bgraph_stream[dev], &g);")
        w("if (st || e != cudaSuccess) { if (g) cudaGraphDestroy(g); "
          "cudaGetLastError(); return pm_status = st ? st : PM_ERR_CUDA; }")
        w("e = cudaGraphInstantiate(&pm_bgraph_exec[dev], g, 0);")
        w("cudaGraphDestroy(g);")
        w("if (e != cudaSuccess) { pm_bgraph_exec[dev] = nullptr; return "
          "pm_status = PM_ERR_CUDA; }")
        w("pm_bgraph_key[dev] = key; pm_bgraph_ws[dev] = "
          "pm_batch_arena.ptr[dev];")
        w.close()
        w("if (cudaGraphLaunch(pm_bgraph_exec[dev], s) != cudaSuccess) return "
          "pm_status = PM_ERR_CUDA;")
        w("return pm_status = PM_OK;")
        w.close()
        w("")

    def gen_header(self):
        name = self.pname
        sig = ", ".join(self.abi_params())
        lines = [
            "/* pipeline_%s -- C ABI of the PolyMage pipeline '%s' built for "
            "NVIDIA B200 (sm_100a)." % (name, self.p.name),
            " * Generated by polymage_b200; argument order: parameters, then "
            "inputs, then",
            " * outputs, each sorted by name.  pipeline_%s replaces the "
            "function of the same" % name,
            " * name the reference generates (signature built at "
            "sandbox/codegen.py:957-1007,",
            " * sandbox/targetc.py:344-366; called through ctypes as in "
            "sandbox/apps/python/",
            " * img_proc/harris/exec_pipe.py:13-35); the other entry points "
            "are additions. */",
            "#pragma once",
            "#ifdef __cplusplus",
            'extern "C" {',
            "#endif",
            "/* host buffers, synchronous (reference ABI) */",
            "void pipeline_%s(%s);" % (name, sig),
            "/* device buffers, asynchronous on `stream` (cudaStream_t); "
            "returns a PM status */",
            "int pipeline_%s_dev(%s, void* stream);" % (name, sig),
            "/* same as _dev through a CUDA graph captured on first use */",
            "int pipeline_%s_graph(%s, void* stream);" % (name, sig),
            "/* n images; iparams: n x %d int params, fparams: n x %d float "
            "params, each row in" % (len(self.iparams), len(self.fparams)),
            " * name order; inputs: n x %d device pointers, outputs: n x %d "
            "device pointers */" % (len(self.inputs), len(self.outputs)),
            "int pipeline_%s_batch(int n, const int* iparams, const float* "
            "fparams, void* const* inputs, void* const* outputs, void* "
            "stream);" % name,
            "/* same as _batch through a CUDA graph captured on first use "
            "(re-captured when",
            " * the arguments change); a repeated _batch call with unchanged "
            "arguments",
            " * relaunches kernels only */",
            "int pipeline_%s_batch_graph(int n, const int* iparams, const "
            "float* fparams, void* const* inputs, void* const* outputs, void* "
            "stream);" % name,
            "/* status of the last call: 0 ok, 1 bad parameters, 2 CUDA "
            "error, 3 kernel error */",
            "int pipeline_%s_status(void);" % name,
            "/* synchronizes and reports the device error word */",
            "int pipeline_%s_check(void);" % name,
            "void pipeline_%s_clear_error(void);" % name,
            "#ifdef __cplusplus",
            "}",
            "#endif",
        ]
        return "\n".join(lines) + "\n"


# ---------------------------------------------------------------------------
class StencilGen(object):
    """Kernel + launcher of one fused stencil group."""

    def __init__(self, pg, group):
        self.pg = pg
        self.fast = False
        self.clamp = False
        self.inside = False
        self.has_inside = False
        self.fold_ok = False
        self.g = group
        self.plan = group.plan
        self.k = "pm_%s_g%d" % (pg.pname, group.level_time)
        self.vec = 1                  # points per thread along the inner dim
        self.vec_stats = None

    def node_name(self, n):
        return self.pg.fn(n.func)

    def generate(self):
        pg = self.pg
        plan = self.plan
        w = pg.w
        k = self.k
        anchor = plan.anchor
        na = anchor.ndims
        stage_nodes = [n for n in plan.nodes if n.role == 'stage']
        glob_ext = [x for x in plan.externals
                    if plan.ext_role[x] == 'global']
        outs = [n for n in plan.nodes if n.role == 'out']
        self.outs = outs
        self.stage_nodes = stage_nodes
        # buffers the kernel touches
        bufs = []
        for n in stage_nodes:
            bufs.append(n.func)
        for x in glob_ext:
            bufs.append(x)
        for n in outs:
            bufs.append(n.func)
        self.bufs = bufs
        pg.meta['groups'].append({
            'kernel': k, 'kind': 'stencil', 'threads': plan.threads,
            'smem': plan.smem_bytes, 'tile': plan.tile,
            'stages': [f.name for f in plan.funcs],
            'materialized': [f.name for f in plan.steps],
            'staged': [n.name for n in stage_nodes],
            'features': plan.features()})
        # ---- descriptor -------------------------------------------------------
        w("// ---- group %d: %s (anchor %s, tile %s, %d threads, %d B smem)"
          % (self.g.level_time, ", ".join(f.name for f in plan.funcs),
             anchor.name, plan.tile, plan.threads, plan.smem_bytes))
        w.open("struct __align__(64) %s_desc" % k)
        for n in stage_nodes:
            w("CUtensorMap tm_%s;" % self.node_name(n))
        for prm in pg.params:
            w("%s %s;" % (pg.ptype(prm), pg.pmap[prm]))
        for f in bufs:
            w("%s%s* b_%s;" % ("" if any(f is n.func for n in outs)
                               else "const ", ctype(f.typ), pg.fn(f)))
        w("int glo[%d], ghi[%d], gn[%d];" % (na, na, na))
        w("int tile_base;")
        for n in stage_nodes:
            w("int tma_%s;" % self.node_name(n))
        w.close("};")
        w.open("struct %s_launch" % k)
        w("%s_desc d0;" % k)
        w("const %s_desc* descs;" % k)
        w("int nimg;")
        w("int first;           // tiles [first, total) of this launch")
        w("int total;           // tiles over all images")
        w("int* queue;          // tile queue counter (persistent launch)")
        w("int stride;          // no queue: a CTA's tiles are gridDim.x apart")
        w.close("};")
        w("")
        self.gen_kernel()
        self.gen_launcher()
        self.gen_footprint()

    def gen_footprint(self):
        """Host function ``<k>_footprint(D, tile, in_end, a_lo, a_hi)``: the
        same region inference as the kernel, for one tile, reduced to what
        the banded host entry needs: per pipeline input, one past the
        largest element offset the tile reads (0 when it reads none), and
        the tile's anchor region."""
        pg = self.pg
        plan = self.plan
        k = self.k
        na = plan.anchor.ndims
        saved_w, saved_ctx = pg.w, getattr(self, 'ctx', None)
        saved_inside = self.has_inside
        w = W()
        pg.w = w
        self.ctx = ExprCtx(w, 'device', pg.pmap, None)
        w.open("static void %s_footprint(const %s_desc& D, int tile, "
               "long long* in_end, int* a_lo, int* a_hi)" % (k, k))
        pg.declare_params(w, "D")
        w("int rem = tile - D.tile_base;")
        for d in range(na - 1, 0, -1):
            w("const int t%d = rem %% D.gn[%d]; rem /= D.gn[%d];" % (d, d, d))
        w("const int t0 = rem;")
        for d in range(na):
            w("const int a_lo%d = D.glo[%d] + t%d * %d;" % (d, d, d,
                                                           plan.tile[d]))
            w("const int a_hi%d = pm_imin(a_lo%d + %d, D.ghi[%d]);" % (
                d, d, plan.tile[d] - 1, d))
        seen = set()
        for n in plan.nodes:
            if id(n.func) not in seen:
                seen.add(id(n.func))
                pg.declare_domain(w, n.func, self.ctx, False)
        self.gen_regions()
        w("(void)t0;")
        for j, f in enumerate(pg.inputs):
            w("in_end[%d] = 0;" % j)
            n = plan.node_of.get(f)
            if n is None or n.role not in ('stage', 'global'):
                continue
            nm = self.node_name(n)
            fnm = pg.fn(f)
            nd = n.ndims
            w.open("")
            empty = []
            for d in range(nd):
                w("const int h%d = pm_imin(r_%s_hi%d, d_%s_hi%d), l%d = "
                  "pm_imax(r_%s_lo%d, d_%s_lo%d);" % (d, nm, d, fnm, d, d, nm,
                                                      d, fnm, d))
                empty.append("l%d > h%d" % (d, d))
            w("long long o = 0, s = 1;")
            for d in range(nd - 1, -1, -1):
                w("o += (long long)(h%d - d_%s_lo%d) * s; s *= (long long)"
                  "(d_%s_hi%d - d_%s_lo%d + 1);" % (d, fnm, d, fnm, d, fnm, d))
            w("if (!(%s)) in_end[%d] = o + 1;" % (" || ".join(empty), j))
            w.close()
        an = self.node_name(plan.node_of[plan.anchor])
        for d in range(na):
            w("a_lo[%d] = r_%s_lo%d; a_hi[%d] = r_%s_hi%d;" % (d, an, d, d, an,
                                                              d))
        w.close()
        w("")
        pg.w = saved_w
        self.ctx = saved_ctx
        self.has_inside = saved_inside
        pg.w.lines.extend(w.lines)
        pg.band_groups.append(self)

    # ---- kernel -------------------------------------------------------------
    def gen_kernel(self):
        pg = self.pg
        plan = self.plan
        w = pg.w
        k = self.k
        nt = plan.threads
        # option 'min_blocks=N': ask ptxas for N resident CTAs per SM
        # (caps registers per thread)
        mb = int(_opt(pg.p, 'min_blocks', 0) or 0)
        lb = "%d, %d" % (nt, mb) if mb > 0 else "%d" % nt
        self.launch_bounds = lb
        # The group's work is a device function over the launch's tiles
        # [first, total): CTA ``pm_bid`` of ``pm_nb`` takes tile first +
        # pm_bid, then every pm_nb-th (stride) or the queue's next.  The
        # group's own kernel calls it with PM_CH false; a chain kernel
        # (several groups in one launch) with PM_CH true.
        w("template <bool PM_CH>")
        w("static __device__ __forceinline__ void %s_body(const %s_launch& L,"
          " const int pm_bid, const int pm_nb)" % (k, k))
        w.open("")
        self.gen_body()
        w.close()
        w('extern "C" __global__ void __launch_bounds__(%s) %s(const '
          '__grid_constant__ %s_launch L)' % (lb, k, k))
        w.open("")
        w("%s_body<false>(L, (int)blockIdx.x, (int)gridDim.x);" % k)
        w.close()
        w("")

    def gen_body(self):
        pg = self.pg
        plan = self.plan
        w = pg.w
        w("extern __shared__ __align__(128) unsigned char pm_smem[];")
        # option 'prefetch': the next tile's staged inputs are loaded into
        # a second copy of their buffers while this tile computes
        pre = bool(self.stage_nodes) and 'prefetch' in pg.p.options and \
            getattr(plan, 'stage_delta', 0) > 0
        self.prefetch = pre
        if 'pdl' in pg.p.options:
            # option 'pdl': launched with programmatic stream serialization;
            # nothing earlier kernels wrote is read before this wait
            w("pm_grid_dep_wait();")
            w("pm_grid_dep_launch();")
        if self.stage_nodes:
            # one mbarrier per copy of the staged inputs, initialized once;
            # each tile that issues TMA loads completes one phase of the
            # barrier of its copy (bit k of pm_phase: parity of barrier k)
            w("uint64_t* pm_bar = reinterpret_cast<uint64_t*>(pm_smem + %d);"
              % (plan.smem_bytes - 128))
            w.open("if (threadIdx.x == 0)")
            w("pm_mbar_init(pm_bar, 1);")
            if pre:
                w("pm_mbar_init(pm_bar + 1, 1);")
            w("pm_fence_barrier_init();")
            w.close()
            w("__syncthreads();")
            w("uint32_t pm_phase = 0;")
        w("__shared__ int pm_next_tile;")
        if not pre:
            w("// Tiles: pm_bid first; with a tile queue (persistent "
              "launch)")
            w("// each CTA then takes the next index from the device "
              "counter.")
            w.open("for (int tile = L.first + pm_bid; tile < L.total; )")
            self.gen_tile_setup("tile")
            self.gen_buffers(None)
            if self.stage_nodes:
                self.gen_issue("pm_bar")
                self.gen_coop_loads()
                self.gen_wait("pm_bar", "0", None)
            for f in plan.steps:
                self.gen_step(f)
            w("if (!L.queue && !L.stride) break;")
            if self.stage_nodes:
                w("pm_fence_proxy_async();   // the next tile's TMA rewrites "
                  "smem")
            w("__syncthreads();      // shared memory is reused by the next "
              "tile")
            w.open("if (L.queue)")
            w("if (threadIdx.x == 0) pm_next_tile = L.first + pm_nb + "
              "atomicAdd(L.queue, 1);")
            w("__syncthreads();")
            w("tile = pm_next_tile;")
            w.close()
            w("else tile += pm_nb;")
            w.close()
            self.gen_body_end()
            return
        # Prefetching tile loop: the staged inputs of a CTA's tiles
        # alternate between two copies; the loads of tile n+1 are issued
        # (thread 0) before tile n is computed.  The next index is drawn
        # from the queue one tile ahead.
        w("int pm_buf = 0;          // copy of the staged inputs this tile "
          "reads")
        w("int tile = L.first + pm_bid;")
        w("bool pm_pend = false;    // loads in flight into the other copy")
        w.open("if (tile < L.total)")
        self.gen_tile_setup("tile")
        self.gen_stage_ptrs("0")
        self.gen_issue("pm_bar")
        w.close()
        w.open("while (tile < L.total)")
        w("int pm_nt = L.total;")
        w.open("if (L.queue)")
        w("if (threadIdx.x == 0) pm_next_tile = L.first + pm_nb + "
          "atomicAdd(L.queue, 1);")
        w("__syncthreads();")
        w("pm_nt = pm_next_tile;")
        w.close()
        w("else if (L.stride) pm_nt = tile + pm_nb;")
        w("pm_pend = false;")
        w.open("if (pm_nt < L.total)")
        self.gen_tile_setup("pm_nt")
        self.gen_stage_ptrs("pm_buf ^ 1")
        self.gen_issue("pm_bar + (pm_buf ^ 1)")
        w("pm_pend = any_tma;")
        w.close()
        w.open("")
        self.gen_tile_setup("tile")
        self.gen_buffers("pm_buf")
        self.gen_coop_loads()
        self.gen_wait("pm_bar + pm_buf", "pm_buf", "pm_bar + (pm_buf ^ 1)")
        for f in plan.steps:
            self.gen_step(f)
        w.close()
        w("pm_fence_proxy_async();   // a later tile's TMA rewrites this copy")
        w("__syncthreads();")
        w("pm_buf ^= 1;")
        w("tile = pm_nt;")
        w.close()
        self.gen_body_end()

    def gen_body_end(self):
        """In a chain kernel the next group lays out shared memory
        differently: the mbarriers of this body are invalidated first."""
        w = self.pg.w
        if not self.stage_nodes:
            return
        w.open("if (PM_CH)")
        w("__syncthreads();")
        w.open("if (threadIdx.x == 0)")
        w("pm_mbar_inval(pm_bar);")
        if self.prefetch:
            w("pm_mbar_inval(pm_bar + 1);")
        w.close()
        w.close()

    def gen_tile_setup(self, tile):
        """Descriptor, parameters, tile box, domains and region inference of
        tile index ``tile`` (emitted into the current scope)."""
        pg = self.pg
        plan = self.plan
        w = pg.w
        k = self.k
        na = plan.anchor.ndims
        w("const %s_desc* Dp = &L.d0;" % k)
        w("if (L.nimg > 1) Dp = L.descs + pm_find_image(L.descs, L.nimg, "
          "%s);" % tile)
        w("const %s_desc& D = *Dp;" % k)
        pg.declare_params(w, "D")
        ctx = ExprCtx(w, 'device', pg.pmap, self.reader)
        self.ctx = ctx
        # tile coordinates
        w("int rem = %s - D.tile_base;" % tile)
        for d in range(na - 1, 0, -1):
            w("const int t%d = rem %% D.gn[%d]; rem /= D.gn[%d];" % (d, d, d))
        w("const int t0 = rem;")
        for d in range(na):
            w("const int a_lo%d = D.glo[%d] + t%d * %d;" % (d, d, d,
                                                           plan.tile[d]))
            w("const int a_hi%d = pm_imin(a_lo%d + %d, D.ghi[%d]);" % (
                d, d, plan.tile[d] - 1, d))
        # domains and strides of everything we touch
        need_stride = set(id(f) for f in self.bufs)
        for n in plan.nodes:
            pg.declare_domain(w, n.func, ctx, id(n.func) in need_stride)
        for f in self.bufs:
            if f not in plan.node_of:
                pg.declare_domain(w, f, ctx, True)
        # region inference: the same values for every thread of the CTA.
        # By default every thread computes them (a few hundred integer
        # instructions for a group of many stages); with option
        # 'shared_regions' thread 0 computes them and hands them to the
        # others through shared memory, at the cost of a CTA barrier and
        # the single thread's latency (faster only for the L=4 pyramid)
        if 'shared_regions' not in pg.p.options:
            self.gen_regions()
            return
        tmp = W()
        tmp.ind = w.ind + 1
        pg.w = ctx.w = tmp
        try:
            self.gen_regions()
        finally:
            pg.w = ctx.w = w
        names = _top_level_decls(tmp.lines)
        self.nshared = getattr(self, 'nshared', 0) + 1
        arr = "pm_ts%d" % self.nshared
        w("__shared__ int %s[%d];   // this tile's regions" % (arr,
                                                             len(names)))
        w.open("if (threadIdx.x == 0)")
        w.lines.extend(tmp.lines)
        for i, (typ, nm) in enumerate(names):
            w("%s[%d] = (int)%s;" % (arr, i, nm))
        w.close()
        w("__syncthreads();")
        for i, (typ, nm) in enumerate(names):
            w("const %s %s = %s%s[%d];" % (
                typ, nm, "(bool)" if typ == "bool" else "", arr, i))

    def gen_buffers(self, buf):
        """HBM buffer pointers and shared-memory buffers of the current
        tile; ``buf``: the copy of the staged inputs (prefetch) or None."""
        pg = self.pg
        w = pg.w
        for f in self.bufs:
            w("%s%s* __restrict__ b_%s = D.b_%s;" % (
                "" if any(f is n.func for n in self.outs) else "const ",
                ctype(f.typ), pg.fn(f), pg.fn(f)))
        for n in self.plan.nodes:
            if n.in_smem:
                if n.role == 'stage' and buf is not None:
                    self.gen_stage_ptrs(buf, [n])
                    continue
                nm = self.node_name(n)
                w("%s* sm_%s = reinterpret_cast<%s*>(pm_smem + %d);" % (
                    ctype(n.func.typ), nm, ctype(n.func.typ), n.smem_off))
                self.decl_smem_origin(n)

    def gen_stage_ptrs(self, buf, nodes=None):
        """Shared-memory pointers and origins of the staged inputs in copy
        ``buf`` (0 or 1) of their buffers."""
        w = self.pg.w
        for n in (self.stage_nodes if nodes is None else nodes):
            nm = self.node_name(n)
            t = ctype(n.func.typ)
            w("%s* sm_%s = reinterpret_cast<%s*>(pm_smem + %d + (%s) * %d);"
              % (t, nm, t, n.smem_off, buf, self.plan.stage_delta))
            self.decl_smem_origin(n)

    def empty_expr(self, n, kind="r"):
        nm = self.node_name(n)
        return " || ".join("%s_%s_lo%d > %s_%s_hi%d" % (kind, nm, d, kind,
                                                        nm, d)
                           for d in range(n.ndims))

    def gen_regions(self):
        pg = self.pg
        plan = self.plan
        w = pg.w
        ctx = self.ctx
        na = plan.anchor.ndims
        big = "0x3fffffff"
        for n in plan.nodes:
            nm = self.node_name(n)
            fnm = pg.fn(n.func)
            nd = n.ndims
            if n.func is plan.anchor:
                for d in range(nd):
                    w("const int r_%s_lo%d = pm_imax(a_lo%d, d_%s_lo%d), "
                      "r_%s_hi%d = pm_imin(a_hi%d, d_%s_hi%d);" % (
                          nm, d, d, fnm, d, nm, d, d, fnm, d))
                self.effective_bounds(n)
                continue
            if n.role == 'out':
                owner = " && ".join("t%d == 0" % kk
                                    for kk in range(na - nd)) or "true"
                for d in range(nd):
                    kk = n.owned_map[d]
                    w("int o_%s_lo%d = (%s) ? pm_imax(a_lo%d, d_%s_lo%d) : "
                      "%s;" % (nm, d, owner, kk, fnm, d, big))
                    w("int o_%s_hi%d = (%s) ? pm_imin(a_hi%d, d_%s_hi%d) : "
                      "-%s;" % (nm, d, owner, kk, fnm, d, big))
                    w("int r_%s_lo%d = o_%s_lo%d, r_%s_hi%d = o_%s_hi%d;" % (
                        nm, d, nm, d, nm, d, nm, d))
            else:
                for d in range(nd):
                    w("int r_%s_lo%d = %s, r_%s_hi%d = -%s;" % (nm, d, big,
                                                                nm, d, big))
            for m, per_dim in self.distinct_uses(n):
                mn = self.node_name(m)
                w.open("if (!(%s))" % self.empty_expr(m, "e"))
                for d, fns in enumerate(per_dim):
                    for fn in fns:
                        if fn.kind == 'mono':
                            a = ctx.expr(fn.expr, {fn.var: "e_%s_lo%d" % (
                                mn, fn.cdim)})
                            b = ctx.expr(fn.expr, {fn.var: "e_%s_hi%d" % (
                                mn, fn.cdim)})
                        elif fn.kind == 'const':
                            a = b = ctx.expr(fn.expr, {})
                        else:
                            a, b = ("d_%s_lo%d" % (fnm, d),
                                    "d_%s_hi%d" % (fnm, d))
                        w("{ const int ea = %s, eb = %s; r_%s_lo%d = "
                          "pm_imin(r_%s_lo%d, pm_imin(ea, eb)); r_%s_hi%d = "
                          "pm_imax(r_%s_hi%d, pm_imax(ea, eb)); }" % (
                              a, b, nm, d, nm, d, nm, d, nm, d))
                w.close()
            if n.role not in ('global', 'inline'):
                # footprint-only nodes stay unclamped (used by pm_inside)
                for d in range(nd):
                    w("r_%s_lo%d = pm_imax(r_%s_lo%d, d_%s_lo%d); r_%s_hi%d ="
                      " pm_imin(r_%s_hi%d, d_%s_hi%d);" % (
                          nm, d, nm, d, fnm, d, nm, d, nm, d, fnm, d))
            self.effective_bounds(n)
        # Interior tile: every region is its full static box (nothing was
        # clamped), HBM reads stay in their buffers, and every stage's single
        # box-shaped Case holds on its whole region, so the stages can be
        # evaluated without conditions, guards or clamped reads.
        conds = []
        for n in plan.nodes:
            nm = self.node_name(n)
            fnm = pg.fn(n.func)
            if n.role == 'global':
                for d in range(n.ndims):
                    if all(fns[d].kind != 'full' for _, fns in n.uses):
                        conds.append("r_%s_lo%d >= d_%s_lo%d && r_%s_hi%d <= "
                                     "d_%s_hi%d" % (nm, d, fnm, d, nm, d,
                                                    fnm, d))
                continue
            if n.role == 'inline':
                continue
            for d, e in enumerate(self.loop_ext(n)):
                conds.append("r_%s_hi%d - r_%s_lo%d + 1 == %d" % (nm, d, nm,
                                                                  d, e))
        inside = self.inside_conds()
        self.has_inside = inside is not None and \
            'no_inside' not in pg.p.options
        # clamped indices (min/max against bounds free of loop variables)
        # that do not clamp at either end of their consumer's region do
        # not clamp anywhere in it (the clamp is monotone in a monotone
        # index): interior tiles then read them unclamped
        unclamp = []
        if 'no_fold_clamps' not in pg.p.options:
            for n in plan.nodes:
                for m, per_dim in self.distinct_uses(n):
                    mn = self.node_name(m)
                    for fns in per_dim:
                        for fn in fns:
                            if fn.kind != 'mono' or not _has_clamp(fn.expr):
                                continue
                            for end in ("lo", "hi"):
                                b = {fn.var: "r_%s_%s%d" % (mn, end,
                                                            fn.cdim)}
                                c = "(%s) == (%s)" % (ctx.expr(fn.expr, b),
                                                      ctx.unclamped(fn.expr,
                                                                    b))
                                if c not in unclamp:
                                    unclamp.append(c)
        self.fold_ok = bool(unclamp)
        if self.has_inside:
            # the clamp checks come last: && evaluates them only on tiles
            # whose regions are full (no overflow on empty regions)
            w("const bool pm_inside = %s;" % (
                " && ".join(conds + inside + unclamp) or "true"))

    def effective_bounds(self, n):
        """Bounds of the points of a node that read their producers: the
        region intersected with the node's Case box."""
        w = self.pg.w
        nm = self.node_name(n)
        cb = getattr(n, 'case_box', None)
        for d in range(n.ndims):
            lo = "r_%s_lo%d" % (nm, d)
            hi = "r_%s_hi%d" % (nm, d)
            if cb:
                for e in cb[d][0]:
                    lo = "pm_imax(%s, %s)" % (lo, self.ctx.expr(e, {}))
                for e in cb[d][1]:
                    hi = "pm_imin(%s, %s)" % (hi, self.ctx.expr(e, {}))
            w("const int e_%s_lo%d = %s, e_%s_hi%d = %s;" % (nm, d, lo, nm,
                                                             d, hi))

    def inside_conds(self):
        """Tile-level conditions under which every stage's Case holds on the
        stage's whole region; None when some stage is piecewise or its
        condition is not a box."""
        pg = self.pg
        plan = self.plan
        ctx = self.ctx
        out = []
        for f in plan.funcs:
            parts = body_parts(f)
            if len(parts) == 1 and parts[0][0] is None:
                continue
            if len(parts) != 1:
                # several box-shaped Cases (e.g. one per channel): evaluated
                # per point by a branch chain in the interior path
                boxes = part_boxes(f)
                if len(boxes) != len(parts) or \
                        not all(b[0].exact for b in boxes):
                    return None
                continue
            boxes = part_boxes(f)
            if len(boxes) != 1 or not boxes[0][0].exact:
                return None
            n = plan.node_of.get(f)
            if n is None:
                continue              # never evaluated in this group
            box = boxes[0][0]
            nm = self.node_name(n)
            for d, v in enumerate(f.variables):
                for e in box.lo[v]:
                    c = "r_%s_lo%d >= %s" % (nm, d, ctx.expr(e, {}))
                    if c not in out:
                        out.append(c)
                for e in box.hi[v]:
                    c = "r_%s_hi%d <= %s" % (nm, d, ctx.expr(e, {}))
                    if c not in out:
                        out.append(c)
        return out

    def distinct_uses(self, n):
        """Uses of a node grouped by consumer, with per-dimension index
        functions deduplicated; of affine functions ``a*v + c`` differing
        only in ``c`` just the smallest and largest ``c`` are kept (the
        others cannot extend the union)."""
        from .expression import affine_form
        out = []
        for m in [u[0] for u in n.uses]:
            if any(m is o[0] for o in out):
                continue
            per_dim = []
            for d in range(n.ndims):
                fns = [fns_[d] for mm, fns_ in n.uses if mm is m]
                keep = []
                seen = set()
                groups = {}
                for fn in fns:
                    k = fn.key()
                    if k in seen:
                        continue
                    seen.add(k)
                    f = affine_form(fn.expr) if fn.kind == 'mono' else None
                    if f is not None and all(not isinstance(v, C.Parameter)
                                             for v in f[0]):
                        gk = tuple(sorted((v.name, c) for v, c in
                                          f[0].items()))
                        lo, hi = groups.get(gk, (None, None))
                        if lo is None or f[1] < lo[1]:
                            lo = (fn, f[1])
                        if hi is None or f[1] > hi[1]:
                            hi = (fn, f[1])
                        groups[gk] = (lo, hi)
                    else:
                        keep.append(fn)
                for lo, hi in groups.values():
                    keep.append(lo[0])
                    if hi[0] is not lo[0]:
                        keep.append(hi[0])
                per_dim.append(keep)
            out.append((m, per_dim))
        return out

    def loop_ext(self, n):
        """Static extents of the box a node is computed (or staged) over."""
        if n.role == 'out' and not n.in_smem:
            na = self.plan.anchor.ndims
            return [min(e, t) for e, t in zip(n.ext,
                                              self.plan.tile[na - n.ndims:])]
        return list(n.ext)

    def decl_smem_origin(self, n):
        """Smem layout of a node: dense [E0][E1]..[E_inner] (inner padded
        for staged inputs); sb_<n> is the linear offset of the origin."""
        w = self.pg.w
        nm = self.node_name(n)
        fnm = self.pg.fn(n.func)
        ext = list(n.ext)
        if n.role != 'stage' and n.pad_inner:
            ext[-1] = n.pad_inner
        if n.role == 'stage':
            es = n.func.typ.size()
            al = max(1, 16 // es)
            ext[-1] = n.pad_inner
            nd = n.ndims
            if getattr(n, 'tight', False):
                # the whole innermost dimension, narrower than one 16-byte
                # chunk: the rounded-down origin offset is always 0
                w("const int so_%s_%d = 0;" % (nm, nd - 1))
            else:
                w("const int so_%s_%d = (r_%s_lo%d - d_%s_lo%d) & ~%d;" % (
                    nm, nd - 1, nm, nd - 1, fnm, nd - 1, al - 1))
            org = ["r_%s_lo%d" % (nm, d) for d in range(nd - 1)] + \
                ["(d_%s_lo%d + so_%s_%d)" % (fnm, nd - 1, nm, nd - 1)]
        else:
            org = ["r_%s_lo%d" % (nm, d) for d in range(n.ndims)]
        strides = []
        s = 1
        for e in reversed(ext):
            strides.insert(0, s)
            s *= e
        n._sm_strides = strides
        n._sm_ext = ext
        terms = ["%s * %d" % (o, st) for o, st in zip(org, strides)]
        w("const int sb_%s = %s;" % (nm, " + ".join(terms)))
        for d in range(n.ndims):
            w("(void)r_%s_hi%d;" % (nm, d))

    def smem_index(self, n, args):
        ctx = self.ctx
        nm = self.node_name(n)
        fnm = self.pg.fn(n.func)
        terms = []
        for d, (a, st) in enumerate(zip(args, n._sm_strides)):
            s = ctx.index(a)
            if is_data_dependent(a):
                if n.role == 'stage':
                    s = "pm_clampi(%s, d_%s_lo%d, d_%s_hi%d)" % (s, fnm, d,
                                                                fnm, d)
                else:
                    s = "pm_clampi(%s, r_%s_lo%d, r_%s_hi%d)" % (s, nm, d,
                                                                nm, d)
            terms.append(s if st == 1 else "%s * %d" % (s, st))
        return "%s - sb_%s" % (" + ".join(terms), nm)

    # ---- producer reads ------------------------------------------------------
    def reader(self, f, args, ctx):
        pg = self.pg
        plan = self.plan
        key = (pg.fn(f), tuple(ctx.index(a) if not is_data_dependent(a)
                                else ctx.expr(a, {}) for a in args))
        hit = ctx.lookup(key)
        if hit is not None:
            return hit
        w = pg.w
        node = plan.node_of.get(f)
        t = ctx.temp()
        guard = pg.oob_guard(f, args, ctx)
        if guard is not None:
            # reads outside the image's domain yield 0 (option 'oob_zero')
            if node is not None and node.in_smem:
                idx = self.smem_index(node, args)
                w("const %s %s = (%s) ? sm_%s[%s] : (%s)0;" % (
                    ctype(f.typ), t, guard, self.node_name(node), idx,
                    ctype(f.typ)))
            elif f in plan.role and plan.role[f] == 'inline':
                raise CodegenError("option oob_zero: %s is read outside "
                                   "its domain and computed inline; it "
                                   "must be materialized" % f.name)
            else:
                w("const %s %s = (%s) ? pm_ld<PM_CH>(b_%s + (%s)) : (%s)0;" % (
                    ctype(f.typ), t, guard, pg.fn(f),
                    pg.gindex(f, args, ctx, clamp_all=self.clamp),
                    ctype(f.typ)))
            ctx.define(key, t)
            return t
        if node is not None and node.in_smem and self.vec > 1 and \
                self.inside:
            vt = self.vec_read(node, f, args)
            if self.vec_stats is not None:
                self.vec_stats[0 if vt else 1] += 1
            if vt is not None:
                ctx.define(key, vt)
                return vt
        if node is not None and node.in_smem:
            idx = self.smem_index(node, args)
            if self.clamp:
                size = 1
                for e in node._sm_ext:
                    size *= e
                idx = "pm_clampi(%s, 0, %d)" % (idx, size - 1)
            w("const %s %s = sm_%s[%s];" % (ctype(f.typ), t,
                                            self.node_name(node), idx))
        elif f in plan.role and plan.role[f] == 'inline':
            self.emit_inline(f, args, t)
        elif f in plan.role:
            raise CodegenError("internal: %s read but not available" %
                               f.name)
        else:
            if self.vec_stats is not None:
                self.vec_stats[1] += 1      # a strided HBM read
            w("const %s %s = pm_ld<PM_CH>(b_%s + (%s));" % (
                ctype(f.typ), t, pg.fn(f),
                pg.gindex(f, args, ctx, clamp_all=self.clamp)))
        ctx.define(key, t)
        return t

    def emit_inline(self, f, args, t):
        """Compute an inlined stage's value at ``args`` into temp ``t``."""
        w = self.pg.w
        ctx = self.ctx
        w("%s %s = 0;" % (ctype(f.typ), t))
        bind = dict(zip(f.variables, args))
        self.emit_cases(f, bind, t, None)

    def emit_cases(self, f, bind, target, written_flag):
        """Evaluate ``f``'s definition at the bound point into ``target``
        (already 0); later cases take precedence, as in the reference
        where later parts' loops overwrite earlier ones."""
        w = self.pg.w
        ctx = self.ctx
        parts = body_parts(f)
        if len(parts) == 1 and parts[0][0] is None:
            e = ctx.expr(parts[0][1], bind)
            w("%s = (%s)(%s);" % (target, ctype(f.typ), e))
            if written_flag:
                w("%s = true;" % written_flag)
            return
        if self.inside and len(parts) == 1:
            # the single Case holds on the whole region of this tile
            e = ctx.expr(parts[0][1], bind)
            w("%s = (%s)(%s);" % (target, ctype(f.typ), e))
            if written_flag:
                w("%s = true;" % written_flag)
            return
        if self.fast and not self.inside:
            # unguarded: every case evaluated, later cases take precedence
            T = ctype(f.typ)
            val = "(%s)0" % T
            cs = []
            for cond, expr, red in parts:
                c = ctx.cond(cond, bind) if cond is not None else "true"
                e = ctx.expr(expr, bind)
                cs.append(c)
                val = "(%s ? (%s)(%s) : %s)" % (c, T, e, val)
            w("%s = %s;" % (target, val))
            if written_flag:
                w("%s = %s;" % (written_flag, " || ".join(cs)))
            return
        first = True
        for cond, expr, red in reversed(parts):
            known = True if cond is None else _cond_static(cond, bind)
            if known is False:
                continue            # never holds at this point
            if known is True and first:
                # the last part that can hold always holds: no branch, and
                # its reads stay in scope for the rest of the point (shared
                # with the other channels of a channel block)
                e = ctx.expr(expr, bind)
                w("%s = (%s)(%s);" % (target, ctype(f.typ), e))
                if written_flag:
                    w("%s = true;" % written_flag)
                return
            ctx.push()
            if known is True:
                w.open("else")
            else:
                c = ctx.cond(cond, bind)
                w.open("%sif (%s)" % ("" if first else "else ", c))
            e = ctx.expr(expr, bind)
            w("%s = (%s)(%s);" % (target, ctype(f.typ), e))
            if written_flag:
                w("%s = true;" % written_flag)
            w.close()
            ctx.pop()
            first = False
            if known is True:
                return

    # ---- staging of external producers ------------------------------------------
    def gen_issue(self, bar):
        """TMA loads of the staged inputs of the tile set up in this scope,
        completing on mbarrier ``bar`` (thread 0 issues them); declares
        ``any_tma``."""
        pg = self.pg
        w = pg.w
        conds = []
        for n in self.stage_nodes:
            nm = self.node_name(n)
            w("const bool use_tma_%s = D.tma_%s && !(%s);" % (
                nm, nm, self.empty_expr(n)))
            conds.append("use_tma_%s" % nm)
        w("const bool any_tma = %s;" % " || ".join(conds))
        w.open("if (any_tma && threadIdx.x == 0)")
        w("uint32_t bytes = 0;")
        for n in self.stage_nodes:
            nm = self.node_name(n)
            box = 1
            for e in n._sm_ext:
                box *= e
            w("if (use_tma_%s) bytes += %du;" % (nm, box * n.func.typ.size()))
        w("pm_mbar_arrive_expect_tx(%s, bytes);" % bar)
        for n in self.stage_nodes:
            nm = self.node_name(n)
            fnm = pg.fn(n.func)
            nd = n.ndims
            coords = ["so_%s_%d" % (nm, nd - 1)]
            for d in range(nd - 2, -1, -1):
                coords.append("r_%s_lo%d - d_%s_lo%d" % (nm, d, fnm, d))
            w("if (use_tma_%s) pm_tma_load_%dd(sm_%s, &D.tm_%s, %s, %s);"
              % (nm, nd, nm, nm, bar, ", ".join(coords)))
        w.close()

    def gen_coop_loads(self):
        """Cooperative loads of the staged inputs that have no tensor map
        (unaligned buffers), into the current tile's copy."""
        pg = self.pg
        plan = self.plan
        w = pg.w
        for n in self.stage_nodes:
            nm = self.node_name(n)
            fnm = pg.fn(n.func)
            nd = n.ndims
            ext = n._sm_ext
            tot = 1
            for e in ext:
                tot *= e
            w.open("if (!D.tma_%s && !(%s))" % (nm, self.empty_expr(n)))
            w.open("for (int i = threadIdx.x; i < %d; i += %d)" % (
                tot, plan.threads))
            self.decompose("i", ext, "j")
            inb = []
            coords = []
            for d in range(nd):
                if d == nd - 1:
                    c = "so_%s_%d + j%d" % (nm, d, d)
                else:
                    c = "r_%s_lo%d - d_%s_lo%d + j%d" % (nm, d, fnm, d, d)
                w("const int c%d = %s;" % (d, c))
                inb.append("c%d >= 0 && c%d <= d_%s_hi%d - d_%s_lo%d" % (
                    d, d, fnm, d, fnm, d))
                coords.append("(long long)c%d * s_%s_%d" % (d, fnm, d))
            w("sm_%s[i] = (%s) ? pm_ld<PM_CH>(b_%s + (%s)) : (%s)0;" % (
                nm, " && ".join(inb), fnm, " + ".join(coords),
                ctype(n.func.typ)))
            w.close()
            w.close()

    def gen_wait(self, bar, bit, other):
        """Wait for the current tile's TMA loads on ``bar`` (phase bit
        ``bit`` of pm_phase), then a CTA barrier.  If any thread's bounded
        wait ran out (the error word records it), the CTA computes nothing
        more: it waits, again bounded, for loads in flight into the other
        copy (``other``, prefetch), and returns."""
        pg = self.pg
        w = pg.w
        w("const bool any_tma_cur = %s;" % " || ".join(
            "(D.tma_%s && !(%s))" % (self.node_name(n), self.empty_expr(n))
            for n in self.stage_nodes))
        w("bool pm_fail = false;")
        w.open("if (any_tma_cur)")
        w("pm_fail = !pm_mbar_wait(%s, (pm_phase >> (%s)) & 1u, "
          "&pm_err_word);" % (bar, bit))
        w("pm_phase ^= 1u << (%s);" % bit)
        w.close()
        w.open("if (__syncthreads_or(pm_fail))")
        if other is not None:
            w("if (pm_pend) pm_mbar_wait(%s, (pm_phase >> (%s ^ 1)) & 1u, "
              "nullptr);" % (other, bit))
        w("return;")
        w.close()

    def decompose(self, iv, ext, prefix):
        w = self.pg.w
        nd = len(ext)
        if nd == 1:
            w("const int %s0 = %s;" % (prefix, iv))
            return
        w("int rr = %s;" % iv)
        for d in range(nd - 1, 0, -1):
            w("const int %s%d = rr %% %d; rr /= %d;" % (prefix, d, ext[d],
                                                       ext[d]))
        w("const int %s0 = rr;" % prefix)

    # ---- materialized stages -------------------------------------------------
    # ---- 4-wide interior loops ----------------------------------------------
    def inner_residues(self):
        """Per node, the residue mod 4 of the origin of its shared-memory
        rows (innermost dim) on interior tiles, when every tile has the
        same one (tile grids starting at a constant); None otherwise."""
        if hasattr(self, '_res4'):
            return self._res4
        from .tiling import infer_regions, _grid_lo
        plan = self.plan
        res = {}
        self._res4 = res
        self._loop_res = {}
        self._lo_res = {}
        glo = _grid_lo(plan)
        na = plan.anchor.ndims
        if glo[na - 1] is None:
            return res
        env = self.pg.p.int_env()
        big = 1 << 20
        # far interior tiles, 8 consecutive along every anchor dim (a full
        # period of any residue mod 8 of a region origin whose scale
        # factors divide the tile sizes; others show up as several values)
        grids = np.meshgrid(*[np.arange(8, dtype=np.int64)] * na,
                            indexing='ij')
        box = []
        for k, t in enumerate(plan.tile):
            lo = (glo[k] if glo[k] is not None else 0) + \
                (big + grids[k].ravel()) * t
            box.append((lo, lo + t - 1))
        try:
            reg = infer_regions(plan, box, env, clamp=False)
        except Exception:
            return res

        def residues(n, d, m):
            v = np.unique(np.asarray(reg[n.func][0][d]).ravel() % m)
            return int(v[0]) if len(v) == 1 else None
        for n in plan.nodes:
            if n.role in ('global', 'inline'):
                continue
            r4 = residues(n, n.ndims - 1, 4)
            if r4 is not None:
                self._loop_res[n.func] = r4
            self._lo_res[n.func] = [residues(n, d, 8)
                                    for d in range(n.ndims)]
            if not n.in_smem:
                continue
            if n.role == 'stage':
                lo = _const_int(n.func.domain[-1].lowerBound)
                if lo is not None:
                    res[n.func] = lo % 4      # origin d_lo + so, so % 4 == 0
            elif n.func in self._loop_res:
                res[n.func] = self._loop_res[n.func]
        return res

    def choose_vec(self, f, n, ext):
        """4 points per thread along the innermost dim when every read of
        the stage from shared memory can then be a 16-byte vector load and
        none is a strided HBM read (decided by generating the loop once
        into a scratch buffer)."""
        pg = self.pg
        if 'no_vec' in pg.p.options or ext[-1] % 4 or ext[-1] < 16:
            return 1
        self.inner_residues()
        if f not in self._loop_res:
            return 1
        saved = pg.w
        pg.w = self.ctx.w = W()
        self.ctx.push()
        self.vec = 4
        self.vec_stats = [0, 0]
        try:
            self.gen_fast_loop(f, n, ext)
            ok = self.vec_stats[0] > 0 and self.vec_stats[1] == 0
        finally:
            self.ctx.pop()
            pg.w = self.ctx.w = saved
            self.vec = 1
            self.vec_stats = None
        if ok:
            return 4
        # 2 points per thread when the stage decides something by the
        # parity of its innermost index (an upsampling by 2 reading x / 2
        # and selecting on x % 2): each of the two points then has a known
        # parity, only the taken arm is evaluated, and both read the same
        # coarse cells
        if 'no_vec2' not in pg.p.options and \
                _inner_parity(f, f.variables[-1]):
            return 2
        return 1

    def vec_read(self, node, f, args):
        """Text of a 16-byte-vector read covering point ``args`` of smem
        node ``node`` (one lane of a cached float4/int4), or None."""
        ctx = self.ctx
        if node.func.typ.size() != 4 or not node.in_smem or self.vec != 4:
            return None
        res = self.inner_residues()
        if node.func not in res or node._sm_ext[-1] % 4:
            return None
        a = args[-1]
        if is_data_dependent(a):
            return None
        fa = affine_form(a)
        if fa is None:
            return None
        coeffs, d = fa
        if len(coeffs) != 1:
            return None
        (v, c), = coeffs.items()
        if c != 1 or getattr(v, '_cname', None) != self.vec_var:
            return None
        vt = {'float': 'float4', 'int': 'int4'}.get(ctype(node.func.typ))
        if vt is None:
            return None
        rc = (self.vec_res + d - res[node.func]) % 4
        aligned = list(args[:-1]) + [a - rc if rc else a]
        idx = self.smem_index(node, aligned)
        key = ('v4', self.node_name(node), idx)
        t = ctx.lookup(key)
        if t is None:
            t = ctx.temp()
            self.pg.w("const %s %s = *reinterpret_cast<const %s*>(&sm_%s[%s]);"
                      % (vt, t, vt, self.node_name(node), idx))
            ctx.define(key, t)
        return "%s.%s" % (t, "xyzw"[rc])

    def gen_step(self, f):
        pg = self.pg
        plan = self.plan
        w = pg.w
        n = plan.node_of[f]
        ext = self.loop_ext(n)
        w("// stage %s (%s%s)" % (f.name, n.role,
                                  "+smem" if n.also_smem else ""))
        w.open("")
        if 'guarded' in pg.p.options:
            self.gen_guarded_loop(f, n, ext)
        else:
            if self.has_inside:
                w.open("if (pm_inside)")
                self.fast = self.inside = True
                self.ctx.fold_clamps = self.fold_ok
                self.vec = self.choose_vec(f, n, ext)
                self.gen_fast_loop(f, n, ext)
                self.vec = 1
                self.ctx.fold_clamps = False
                self.fast = self.inside = False
                w.close()
                w.open("else")
            # every point of the static box, select-based cases, clamped
            # reads: valid on any tile
            self.fast = self.clamp = True
            self.gen_fast_loop(f, n, ext)
            self.fast = self.clamp = False
            if self.has_inside:
                w.close()
        w.close()
        if n.in_smem:
            w("__syncthreads();")

    def _store(self, f, n, qs, val, flag, smem_idx, gidx=None,
               hbm=True):
        """Store one computed point: shared memory and/or HBM (owned
        points; pipeline outputs only where some case held)."""
        pg = self.pg
        plan = self.plan
        w = pg.w
        nm = self.node_name(n)
        fnm = pg.fn(f)
        nd = n.ndims
        if n.in_smem and smem_idx is not None:
            w("sm_%s[%s] = %s;" % (nm, smem_idx, val))
        if n.role == 'out' and hbm:
            own = ""
            if n.func is not plan.anchor and n.also_smem:
                own = " && ".join("%s >= o_%s_lo%d && %s <= o_%s_hi%d" % (
                    qs[d], nm, d, qs[d], nm, d) for d in range(nd))
            elif self.clamp:
                own = " && ".join("%s >= r_%s_lo%d && %s <= r_%s_hi%d" % (
                    qs[d], nm, d, qs[d], nm, d) for d in range(nd))
            cond = " && ".join(x for x in [own, flag or ""] if x)
            idx = gidx or " + ".join(
                ["(long long)(%s - d_%s_lo%d) * s_%s_%d" % (qs[d], fnm, d,
                                                            fnm, d)
                 for d in range(nd)])
            if cond:
                w("if (%s) b_%s[%s] = %s;" % (cond, fnm, idx, val))
            else:
                w("b_%s[%s] = %s;" % (fnm, idx, val))

    def gen_guarded_loop(self, f, n, ext):
        """Border tiles: one point per iteration, guarded by the region."""
        pg = self.pg
        plan = self.plan
        w = pg.w
        nm = self.node_name(n)
        nd = n.ndims
        comp = pg.p.func_map[f]
        tot = 1
        for e in ext:
            tot *= e
        w.open("for (int i = threadIdx.x; i < %d; i += %d)" % (
            tot, plan.threads))
        self.decompose("i", ext, "j")
        lv = _loop_vars(nd)
        for d in range(nd):
            w("const int q%d = r_%s_lo%d + j%d;" % (d, nm, d, d))
        w("if (%s) continue;" % " || ".join("q%d > r_%s_hi%d" % (d, nm, d)
                                           for d in range(nd)))
        ctx = self.ctx
        ctx.push()
        bind = dict(zip(f.variables, lv))
        w("%s v = 0;" % ctype(f.typ))
        flag = None
        if n.role == 'out' and comp.is_output:
            w("bool wr = false;")
            flag = "wr"
        self.emit_cases(f, bind, "v", flag)
        sidx = "i"
        if n.in_smem:
            sidx = " + ".join("j%d * %d" % (d, st) for d, st in
                              enumerate(n._sm_strides))
        self._store(f, n, ["q%d" % d for d in range(nd)], "v", flag, sidx)
        ctx.pop()
        w.close()

    def gen_fast_loop(self, f, n, ext):
        """Interior tiles: each thread computes a block of ``rb`` points
        along the second-innermost dimension (consecutive threads take
        consecutive innermost points, so shared-memory accesses stay
        conflict-free and HBM accesses coalesced); reads shared by the
        block's points are loaded once."""
        pg = self.pg
        plan = self.plan
        w = pg.w
        nm = self.node_name(n)
        nd = n.ndims
        comp = pg.p.func_map[f]
        rb_max = int(_opt(pg.p, 'rblock', 4))
        inner = ext[-1]
        if nd >= 2:
            outer = ext[-2]
            # block height: fewest rows loaded (block + a 2-row halo) per
            # row computed; a last partial block is shifted back to end at
            # the last row (its overlap is recomputed, same values)
            K, best = 1, None
            for k in range(min(rb_max, outer), 0, -1):
                cost = -(-outer // k) * (k + 2)
                if best is None or cost < best:
                    K, best = k, cost
        else:
            outer, K = 1, 1
        # a small outermost dimension (channels) is computed by the same
        # thread, so that reads and index arithmetic shared by the channels
        # of a point are done once
        cb = 1
        if nd >= 3 and ext[0] <= 4 and 'no_cblock' not in pg.p.options:
            cb = ext[0]
            while K > 1 and K * cb > 16:
                K -= 1
        V = self.vec if (self.inside and nd >= 2) else 1
        if V > 1:
            # 4 consecutive inner points per thread: shared-memory reads of
            # a row become 16-byte vector loads
            while K > 1 and K * cb * V > 16:
                K -= 1
            self.vec_var = "qb%d" % (nd - 1)
            self.vec_res = self._loop_res[f]
        nblk = -(-outer // K)
        rest = ext[:-2] if nd >= 2 else []
        total = nblk * (inner // V)
        for d, e in enumerate(rest):
            total *= 1 if (d == 0 and cb > 1) else e
        strides = []
        st = 1
        for e in reversed(ext):
            strides.insert(0, st)
            st *= e
        w.open("for (int it = threadIdx.x; it < %d; it += %d)" % (
            total, plan.threads))
        if V > 1:
            w("const int ji = (it %% %d) * %d; int rr = it / %d;" % (
                inner // V, V, inner // V))
        else:
            w("const int ji = it %% %d; int rr = it / %d;" % (inner, inner))
        if nd >= 2:
            if outer % K:
                w("const int jo = pm_imin((rr %% %d) * %d, %d); rr /= %d;" % (
                    nblk, K, outer - K, nblk))
            else:
                w("const int jo = (rr %% %d) * %d; rr /= %d;" % (nblk, K,
                                                                nblk))
        for d in range(len(rest) - 1, -1, -1):
            if d == 0:
                w("const int j0 = %s;" % ("0" if cb > 1 else "rr"))
            else:
                w("const int j%d = rr %% %d; rr /= %d;" % (d, rest[d],
                                                          rest[d]))
        base = _loop_vars(nd, "qb")
        for d in range(nd):
            if d == nd - 1:
                j = "ji"
            elif d == nd - 2:
                j = "jo"
            else:
                j = "j%d" % d
            w("const int qb%d = r_%s_lo%d + %s;" % (d, nm, d, j))
        if n.in_smem:
            strides = list(n._sm_strides)     # rows may be padded
        w("const int ib = %s;" % " + ".join(
            "(qb%d - r_%s_lo%d) * %d" % (d, nm, d, strides[d])
            for d in range(nd)))
        fnm = pg.fn(f)
        if n.role == 'out':
            w("const long long gb = %s;" % " + ".join(
                "(long long)(qb%d - d_%s_lo%d) * s_%s_%d" % (d, fnm, d, fnm, d)
                for d in range(nd)))
        ctx = self.ctx
        ctx.push()
        saved_lo = dict(ctx.var_lo)
        saved_res = dict(ctx.var_res)
        for d, dom in enumerate(f.domain):
            lo = _const_int(dom.lowerBound)
            if lo is not None:
                # regions are clamped to the domain: qb >= its lower bound
                ctx.var_lo["qb%d" % d] = lo
        if self.inside and 'no_static_res' not in pg.p.options:
            # interior tiles: region origins have fixed residues (mod 8),
            # and block starts are multiples of the block sizes
            self.inner_residues()
            lres = self._lo_res.get(f) or [None] * nd
            for d in range(nd):
                if lres[d] is None:
                    continue
                if d == nd - 1:
                    m = math.gcd(V, 8) if V > 1 else 1
                elif d == nd - 2 and outer % K == 0:
                    m = math.gcd(K, 8)
                else:
                    m = 1
                if m > 1:
                    ctx.var_res["qb%d" % d] = (lres[d] % m, m)
        flagged = n.role == 'out' and comp.is_output
        # 16-byte stores of the 4 inner points to HBM: the anchor's inner
        # index is 4-aligned on interior tiles; base and row strides are
        # checked at run time
        vst = None
        if V == 4 and n.role == 'out' and n.func is plan.anchor and \
                f.typ.size() == 4 and pg.storage_perm(f) is None:
            dlo = _const_int(f.domain[-1].lowerBound)
            if dlo is not None and (self._loop_res[f] - dlo) % 4 == 0:
                vst = {'float': 'float4', 'int': 'int4'}.get(ctype(f.typ))
                if vst:
                    w("const bool pm_v4 = ((unsigned long long)b_%s & 15) "
                      "== 0%s;" % (fnm, "".join(
                          " && (s_%s_%d & 3) == 0" % (fnm, d)
                          for d in range(nd - 1))))
        # channels tiled whole: on an interior tile the region spans the
        # domain's constant channel range, so the channel of block member
        # c is the literal lo + c and conditions on it fold at compile time
        # (the camera pipe's per-channel colour matrix rows)
        clo = None
        if cb > 1 and self.inside:
            from .tiling import _const_extent
            lo0 = _const_int(f.domain[0].lowerBound)
            if lo0 is not None and \
                    _const_extent(f.domain[0], pg.p.int_env()) == cb:
                clo = lo0
        group = []
        for c in range(cb):
            for k in range(K):
                for u in range(V):
                    pt = list(base)
                    qs = ["qb%d" % d for d in range(nd)]
                    if nd >= 2 and k:
                        pt[nd - 2] = base[nd - 2] + k
                        qs[nd - 2] = "(qb%d + %d)" % (nd - 2, k)
                    if clo is not None:
                        pt[0] = Value(clo + c, C.Int)
                    elif c:
                        pt[0] = base[0] + c
                    if c:
                        qs[0] = "(qb0 + %d)" % c
                    if u:
                        pt[nd - 1] = base[nd - 1] + u
                        qs[nd - 1] = "(qb%d + %d)" % (nd - 1, u)
                    bind = dict(zip(f.variables, pt))
                    v = "v%d_%d_%d" % (c, k, u)
                    w("%s %s = 0;" % (ctype(f.typ), v))
                    flag = None
                    if flagged:
                        flag = "wr%d_%d_%d" % (c, k, u)
                        w("bool %s = false;" % flag)
                    self.emit_cases(f, bind, v, flag)
                    off = k * strides[nd - 2] + c * strides[0] + u
                    idx = "ib" if off == 0 else "ib + %d" % off
                    gidx = None
                    if n.role == 'out':
                        terms = ["gb"]
                        if k:
                            terms.append("%d * s_%s_%d" % (k, fnm, nd - 2))
                        if c:
                            terms.append("%d * s_%s_0" % (c, fnm))
                        if u and pg.storage_perm(f) is not None:
                            terms.append("%d * s_%s_%d" % (u, fnm, nd - 1))
                        elif u:
                            terms.append("%d" % u)
                        gidx = " + ".join(terms)
                    self._store(f, n, qs, v, flag, idx, gidx,
                                hbm=vst is None)
                    if vst is None:
                        continue
                    group.append((qs, v, flag, gidx))
                    if u < V - 1:
                        continue
                    cond = " && ".join(["pm_v4"] + [g[2] for g in group
                                                    if g[2]])
                    w.open("if (%s)" % cond)
                    w("*reinterpret_cast<%s*>(&b_%s[%s]) = make_%s(%s);" % (
                        vst, fnm, group[0][3], vst,
                        ", ".join(g[1] for g in group)))
                    w.close()
                    w.open("else")
                    for gq, gv, gf, gi in group:
                        self._store(f, n, gq, gv, gf, None, gi)
                    w.close()
                    group = []
        ctx.var_lo = saved_lo
        ctx.var_res = saved_res
        ctx.pop()
        w.close()

    # ---- launcher -------------------------------------------------------------
    def gen_launcher(self):
        pg = self.pg
        plan = self.plan
        w = pg.w
        k = self.k
        anchor = plan.anchor
        na = anchor.ndims
        ctx = ExprCtx(w, 'device', pg.pmap, None)
        fill = "fill_" + k
        # descriptor filler shared by the single and batched launches
        w.open("static int %s(%s_desc& D, const pm_args& A, const size_t* "
               "wsoff, long long* ntiles)" % (fill, k))
        pg.declare_params(w, "A")
        for prm in pg.params:
            w("D.%s = %s;" % (pg.pmap[prm], pg.pmap[prm]))
        for f in self.bufs:
            w("D.b_%s = (%s%s*)(%s);" % (
                pg.fn(f), "" if any(f is n.func for n in self.outs)
                else "const ", ctype(f.typ), pg.buf_expr(f)))
        # grid: union of the out nodes' domains along the anchor dims
        for kk in range(na):
            w("long long glo%d = 0x3fffffff, ghi%d = -0x3fffffff;" % (kk, kk))
        for n in self.outs:
            for d, dom in enumerate(n.func.domain):
                kk = n.owned_map[d] if n.func is not anchor else d
                w("glo%d = pm_llmin(glo%d, %s); ghi%d = pm_llmax(ghi%d, %s);"
                  % (kk, kk, ctx.expr(dom.lowerBound, {}), kk, kk,
                     ctx.expr(dom.upperBound, {})))
        w("long long tot = 1;")
        for kk in range(na):
            w("if (ghi%d < glo%d) { *ntiles = 0; return PM_OK; }" % (kk, kk))
            w("D.glo[%d] = (int)glo%d; D.ghi[%d] = (int)ghi%d;" % (kk, kk, kk,
                                                                  kk))
            w("D.gn[%d] = (int)((ghi%d - glo%d + %d) / %d);" % (
                kk, kk, kk, plan.tile[kk], plan.tile[kk]))
            w("tot *= D.gn[%d];" % kk)
        w("*ntiles = tot;")
        for n in self.stage_nodes:
            nm = self.node_name(n)
            f = n.func
            nd = n.ndims
            dims = ", ".join("(long long)((%s) - (%s) + 1)" % (
                ctx.expr(d.upperBound, {}), ctx.expr(d.lowerBound, {}))
                for d in f.domain)
            box = ", ".join(str(e) for e in n._sm_ext)
            w("{ long long dims[%d] = {%s}; int box[%d] = {%s};" % (
                nd, dims, nd, box))
            pitch = pg.row_pitch(f)
            if pg.storage_perm(f) is not None:
                # a reordered array is staged by cooperative loads
                w("  D.tma_%s = 0; (void)dims; (void)box; }" % nm)
                continue
            w("  D.tma_%s = pm_use_tma() && pm_make_tmap(&D.tm_%s, D.b_%s, "
              "%d, dims, box, %d, %d, %s); }" % (
                  nm, nm, pg.fn(f), nd, f.typ.size(),
                  1 if f.typ in (C.Float, C.Double) else 0,
                  "(dims[%d] + %d) / %d * %d" % (nd - 1, pitch - 1, pitch,
                                                 pitch) if pitch > 1
                  else "dims[%d]" % (nd - 1)))
        w("return PM_OK;")
        w.close()
        w("")
        w("static bool %s_attr[64];     // per device" % k)
        w("static int %s_resident[64];  // per device" % k)
        w("// CTAs of this kernel resident on the current device at once")
        w.open("static long long %s_resident_now()" % k)
        w("const int dev = pm_cur_dev();")
        w.open("if (!%s_resident[dev])" % k)
        w("int per_sm = 0, sms = 0;")
        w("cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);")
        w("cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, %s, %d, %d);"
          % (k, plan.threads, plan.smem_bytes))
        w("%s_resident[dev] = (int)pm_llmax(1, (long long)per_sm * sms);" % k)
        w.close()
        w("return %s_resident[dev];" % k)
        w.close()
        w.open("static int launch_%s(pm_args& A, const size_t* wsoff, "
               "cudaStream_t s)" % k)
        w("%s_launch L; memset(&L, 0, sizeof(L));" % k)
        w("L.nimg = 1;")
        w("long long nt = 0;")
        w("int st = %s(L.d0, A, wsoff, &nt); if (st) return st;" % fill)
        w("if (nt == 0) return PM_OK;")
        w("if (nt > 0x7fffffffLL) return PM_ERR_UNSUPPORTED;")
        w("L.total = (int)nt; L.queue = nullptr; L.stride = 0;")
        w.open("if (!%s_attr[pm_cur_dev()])" % k)
        w("if (cudaFuncSetAttribute(%s, cudaFuncAttributeMaxDynamicShared"
          "MemorySize, %d) != cudaSuccess) return PM_ERR_CUDA;" % (
              k, plan.smem_bytes))
        w("%s_attr[pm_cur_dev()] = true;" % k)
        w.close()
        w("long long grid = nt;")
        if getattr(self, 'prefetch', False):
            # prefetching needs several tiles per CTA: as many CTAs as fit
            # on the GPU at once, each taking every gridDim.x-th tile
            w.open("if (pm_persistent())")
            w("const long long res = %s_resident_now();" % k)
            w("if (nt > res) { grid = res; L.stride = 1; }")
            w.close()
        if 'pdl' in pg.p.options:
            w("if (pm_launch_pdl(%s, (unsigned)grid, %d, %d, s, L) != "
              "cudaSuccess) return PM_ERR_CUDA;" % (k, plan.threads,
                                                   plan.smem_bytes))
        else:
            w("%s<<<(unsigned)grid, %d, %d, s>>>(L);" % (k, plan.threads,
                                                        plan.smem_bytes))
        w("return cudaGetLastError() == cudaSuccess ? PM_OK : PM_ERR_CUDA;")
        w.close()
        w("")
        # batched: descriptors for all images in one upload
        # The last batch launch is kept so that an unchanged batch can be
        # replayed (kernels only: descriptors already on the device).
        w("static %s_launch pm_bl_%s;" % (k, k))
        w("static long long pm_bgrid_%s = 0;" % k)
        w("static bool pm_bvalid_%s = false;" % k)
        w.open("static int batch_%s(pm_args* As, const size_t* wsoffs, int "
               "nslot, int n, char* pinned, char* ddesc, size_t* doff, "
               "cudaStream_t s, int replay)" % k)
        w.open("if (replay)")
        w("if (!pm_bvalid_%s) return PM_ERR_CUDA;" % k)
        w("if (pm_bgrid_%s == 0) return PM_OK;" % k)
        w("if (pm_bl_%s.queue && cudaMemsetAsync(pm_bl_%s.queue, 0, "
          "sizeof(int), s) != cudaSuccess) return PM_ERR_CUDA;" % (k, k))
        w("%s<<<(unsigned)pm_bgrid_%s, %d, %d, s>>>(pm_bl_%s);" % (
            k, k, plan.threads, plan.smem_bytes, k))
        w("return cudaGetLastError() == cudaSuccess ? PM_OK : PM_ERR_CUDA;")
        w.close()
        w("pm_bvalid_%s = false;" % k)
        w("size_t off = (*doff + 63) & ~size_t(63);")
        w("%s_desc* H = reinterpret_cast<%s_desc*>(pinned + off);" % (k, k))
        w("long long base = 0;")
        w.open("for (int i = 0; i < n; ++i)")
        w("long long nt = 0;")
        w("int st = %s(H[i], As[i], wsoffs + (size_t)i * nslot, &nt); if (st) "
          "return st;" % fill)
        w("H[i].tile_base = (int)base; base += nt;")
        w.close()
        w("*doff = off + sizeof(%s_desc) * n;" % k)
        w("size_t qoff = (*doff + 63) & ~size_t(63); *doff = qoff + 64;")
        w.open("if (base == 0)")
        w("pm_bgrid_%s = 0; pm_bvalid_%s = true;" % (k, k))
        w("return PM_OK;")
        w.close()
        w("if (base > 0x7fffffffLL) return PM_ERR_UNSUPPORTED;")
        w("if (cudaMemcpyAsync(ddesc + off, H, sizeof(%s_desc) * n, "
          "cudaMemcpyHostToDevice, s) != cudaSuccess) return PM_ERR_CUDA;" % k)
        w("cudaEventRecord(pm_batch_event[pm_cur_dev()], s);")
        w("%s_launch L; memset(&L, 0, sizeof(L));" % k)
        w("L.nimg = n; L.descs = reinterpret_cast<const %s_desc*>(ddesc + "
          "off);" % k)
        w("if (n == 1) L.d0 = H[0];")
        w("L.total = (int)base;")
        w.open("if (!%s_attr[pm_cur_dev()])" % k)
        w("if (cudaFuncSetAttribute(%s, cudaFuncAttributeMaxDynamicShared"
          "MemorySize, %d) != cudaSuccess) return PM_ERR_CUDA;" % (
              k, plan.smem_bytes))
        w("%s_attr[pm_cur_dev()] = true;" % k)
        w.close()
        w("// persistent launch: as many CTAs as fit on the GPU at once; they")
        w("// drain a device-side tile queue spanning every image of the batch")
        w("long long grid = base;")
        w.open("if (pm_persistent() && base > %s_resident_now())" % k)
        w("L.queue = reinterpret_cast<int*>(ddesc + qoff);")
        w("if (cudaMemsetAsync(L.queue, 0, sizeof(int), s) != cudaSuccess) "
          "return PM_ERR_CUDA;")
        w("grid = %s_resident_now();" % k)
        w.close()
        w("pm_bl_%s = L; pm_bgrid_%s = grid; pm_bvalid_%s = true;" % (k, k, k))
        w("%s<<<(unsigned)grid, %d, %d, s>>>(L);" % (k, plan.threads,
                                                    plan.smem_bytes))
        w("return cudaGetLastError() == cudaSuccess ? PM_OK : PM_ERR_CUDA;")
        w.close()
        w("")
        pg.launch_fns.append("launch_" + k)
        pg.batch_fns.append("batch_" + k)
        pg.desc_sizes.append("sizeof(%s_desc)" % k)


# ---------------------------------------------------------------------------
class ReductionGen(object):
    """Init + privatized accumulation kernels of a Reduction group."""

    def __init__(self, pg, group):
        self.pg = pg
        self.g = group
        self.plan = group.plan
        self.f = self.plan.func
        self.k = "pm_%s_g%d" % (pg.pname, group.level_time)

    def generate(self):
        pg = self.pg
        plan = self.plan
        f = self.f
        w = pg.w
        k = self.k
        fnm = pg.fn(f)
        rvars = f.reductionVariables
        nr = len(rvars)
        nd = f.ndims
        T = ctype(f.typ)
        parts = body_parts(f)
        reads = []
        for cond, expr, red in parts:
            for r in list(expr.collect(C.Reference)) + \
                    (cond.collect(C.Reference) if cond is not None else []):
                if all(r.objectRef is not q for q in reads) and \
                        r.objectRef is not f:
                    reads.append(r.objectRef)
            for a in red.accumulate_ref.arguments:
                for r in a.collect(C.Reference):
                    if all(r.objectRef is not q for q in reads):
                        reads.append(r.objectRef)
        self.reads = reads
        ops = set(red.op_type for _, _, red in parts)
        if len(ops) != 1 and not _disjoint_parts(f, parts):
            raise CodegenError("%s: reduction parts with different "
                               "operators may update the same cell" %
                               f.name)
        # one operator per part; with several, the parts update disjoint
        # cells (a condition fixing a non-reduced variable to different
        # constants) and accumulate straight into the output
        self.part_ops = [red.op_type for _, _, red in parts]
        self.op = parts[0][2].op_type
        self.mixed = len(ops) != 1
        pg.meta['groups'].append({
            'kernel': k, 'kind': 'reduction', 'threads': plan.threads,
            'smem': plan.smem_bytes, 'tile': plan.tile,
            'stages': [f.name], 'privatized': plan.privatize,
            'features': plan.features()})
        w("// ---- group %d: reduction %s (tile %s, privatized %s)" % (
            self.g.level_time, f.name, plan.tile, plan.privatize))
        w.open("struct __align__(64) %s_desc" % k)
        for prm in pg.params:
            w("%s %s;" % (pg.ptype(prm), pg.pmap[prm]))
        for x in reads:
            w("const %s* b_%s;" % (ctype(x.typ), pg.fn(x)))
        w("%s* b_%s;" % (T, fnm))
        w("int glo[%d], ghi[%d], gn[%d];" % (nr, nr, nr))
        w("int tile_base;")
        w("long long ncells;")
        w("long long nbytes;     // the array's bytes, row padding included")
        w.close("};")
        w.open("struct %s_launch" % k)
        w("%s_desc d0;" % k)
        w("const %s_desc* descs;" % k)
        w("int nimg;")
        w.close("};")
        ident = self.identity()
        # ---- init kernel: every cell to the default value ----
        ctx0 = ExprCtx(w, 'device', pg.pmap, self.reader)
        self.ctx = ctx0
        w('extern "C" __global__ void __launch_bounds__(256) %s_init(const '
          '__grid_constant__ %s_launch L)' % (k, k))
        w.open("")
        w.open("for (int im = 0; im < L.nimg; ++im)")
        w("const %s_desc& D = (L.nimg == 1) ? L.d0 : L.descs[im];" % k)
        pg.declare_params(w, "D")
        w("%s* __restrict__ out = D.b_%s;" % (T, fnm))
        pg.declare_domain(w, f, ctx0, True)
        lv = _loop_vars(nd)
        bind = dict(zip(f.variables, lv))
        dflt = ctx0.expr(f.default, bind)
        # cell index -> coordinates in 32-bit arithmetic when the domain
        # has fewer than 2^31 cells (the usual case; 64-bit division is
        # several times dearer), else in 64-bit
        for IT in ("unsigned", "long long"):
            if IT == "unsigned":
                w.open("if (D.ncells <= 0x7fffffffLL)")
            else:
                w.open("else")
            w.open("for (%s c = (%s)blockIdx.x * blockDim.x + threadIdx.x; "
                   "c < (%s)D.ncells; c += (%s)gridDim.x * blockDim.x)" % (
                       IT, IT, IT, IT))
            w("%s rr = c;" % IT)
            for d in range(nd - 1, -1, -1):
                w("const int q%d = (int)(rr %% (%s)(d_%s_hi%d - d_%s_lo%d + "
                  "1)) + d_%s_lo%d; rr /= (%s)(d_%s_hi%d - d_%s_lo%d + 1);"
                  % (d, IT, fnm, d, fnm, d, fnm, d, IT, fnm, d, fnm, d))
            w("out[%s] = (%s)(%s);" % (" + ".join(
                "(long long)(q%d - d_%s_lo%d) * s_%s_%d" % (d, fnm, d, fnm,
                                                             d)
                for d in range(nd)), T, dflt))
            w.close()
            w.close()
        w.close()
        w.close()
        w("")
        # ---- accumulation kernel ----
        w('extern "C" __global__ void __launch_bounds__(%d) %s(const '
          '__grid_constant__ %s_launch L)' % (plan.threads, k, k))
        w.open("")
        w("extern __shared__ __align__(128) unsigned char pm_smem[];")
        w("const int tile = blockIdx.x;")
        w("const %s_desc* Dp = &L.d0;" % k)
        w("if (L.nimg > 1) Dp = L.descs + pm_find_image(L.descs, L.nimg, "
          "tile);")
        w("const %s_desc& D = *Dp;" % k)
        pg.declare_params(w, "D")
        ctx = ExprCtx(w, 'device', pg.pmap, self.reader)
        self.ctx = ctx
        w("int rem = tile - D.tile_base;")
        for d in range(nr - 1, 0, -1):
            w("const int t%d = rem %% D.gn[%d]; rem /= D.gn[%d];" % (d, d, d))
        w("const int t0 = rem;")
        for d in range(nr):
            w("const int a_lo%d = D.glo[%d] + t%d * %d;" % (d, d, d,
                                                           plan.tile[d]))
            w("const int a_hi%d = pm_imin(a_lo%d + %d, D.ghi[%d]);" % (
                d, d, plan.tile[d] - 1, d))
        pg.declare_domain(w, f, ctx, True)
        for x in reads:
            pg.declare_domain(w, x, ctx, True)
            w("const %s* __restrict__ b_%s = D.b_%s;" % (ctype(x.typ),
                                                         pg.fn(x), pg.fn(x)))
        w("%s* __restrict__ out = D.b_%s;" % (T, fnm))
        if plan.gather is not None and not self.mixed:
            self.gen_gather(ctx, parts)
            w.close()
            w("")
            self.gen_launcher()
            return
        priv = plan.privatize and not self.mixed
        if priv:
            # privatized box: union of target footprints of this tile
            for d in range(nd):
                w("int p_lo%d = 0x3fffffff, p_hi%d = -0x3fffffff;" % (d, d))
            for fns in plan.target_fns:
                for d, fn in enumerate(fns):
                    if fn.kind == 'mono':
                        a = ctx.expr(fn.expr, {fn.var: "a_lo%d" % fn.cdim})
                        b = ctx.expr(fn.expr, {fn.var: "a_hi%d" % fn.cdim})
                    elif fn.kind == 'const':
                        a = b = ctx.expr(fn.expr, {})
                    else:
                        a, b = "d_%s_lo%d" % (fnm, d), "d_%s_hi%d" % (fnm, d)
                    w("{ const int ea = %s, eb = %s; p_lo%d = pm_imin(p_lo%d, "
                      "pm_imin(ea, eb)); p_hi%d = pm_imax(p_hi%d, pm_imax(ea, "
                      "eb)); }" % (a, b, d, d, d, d))
            for d in range(nd):
                w("p_lo%d = pm_imax(p_lo%d, d_%s_lo%d); p_hi%d = pm_imin("
                  "p_hi%d, d_%s_hi%d);" % (d, d, fnm, d, d, d, fnm, d))
            ptot = 1
            for e in plan.priv_ext:
                ptot *= e
            w("%s* acc = reinterpret_cast<%s*>(pm_smem);" % (T, T))
            w("for (int i = threadIdx.x; i < %d; i += %d) acc[i] = %s;" % (
                ptot, plan.threads, ident))
            w("__syncthreads();")
        # loop over the tile's reduction points; unrolled (option
        # 'red_unroll', default 4) so that the loads of several points are
        # in flight before their atomics
        tot = 1
        for t in plan.tile:
            tot *= t
        un = int(_opt(pg.p, 'red_unroll', 4) or 1)
        if un > 1:
            w("#pragma unroll %d" % un)
        w.open("for (int i = threadIdx.x; i < %d; i += %d)" % (tot,
                                                               plan.threads))
        spread = self.spread_factor()
        if spread:
            # option 'red_spread': consecutive threads take points k apart
            # along the innermost reduction variable (k = the divisor that
            # maps it to a target cell), so that a warp's 32 atomics go to
            # 32 different cells instead of 32/k threads per cell
            E = plan.tile[-1]
            m = E // spread
            w("const int pm_ii = i %% %d;" % E)
            w("const int pm_is = (i - pm_ii) + (pm_ii %% %d) * %d + "
              "pm_ii / %d;" % (m, spread, m))
            StencilGen.decompose(self, "pm_is", plan.tile, "j")
        else:
            StencilGen.decompose(self, "i", plan.tile, "j")
        lv = _loop_vars(nr)
        # A point past the tile's last one (a partial tile) is clamped onto
        # it and only its accumulation is skipped: its reads stay in
        # bounds and need no branch, so the unrolled iterations' loads can
        # all be issued before the first atomic
        w("const bool pm_pt = !(%s);" % " || ".join(
            "a_lo%d + j%d > a_hi%d" % (d, d, d) for d in range(nr)))
        for d in range(nr):
            w("const int q%d = pm_imin(a_lo%d + j%d, a_hi%d);" % (d, d, d, d))
        rbind = dict(zip(rvars, lv))
        saved_lo = dict(ctx.var_lo)
        for d, dom in enumerate(f.reductionDomain):
            lo = _const_int(dom.lowerBound)
            if lo is not None:
                # tiles start at the reduction domain's lower bound
                ctx.var_lo["q%d" % d] = lo
        for pi, (cond, expr, red) in enumerate(parts):
            tbind = tbind_of(f, rvars, red, rbind)
            # Parts whose condition holds everywhere read in bounds at every
            # point of the reduction domain (checked per call), so they
            # share one scope: values they have in common (e.g. an input
            # pixel) are read once.
            shared = cond is None or _cond_const_true(cond, tbind)
            if not shared:
                ctx.push()
                w.open("")
            tgt = red.accumulate_ref.arguments
            cn = ["c%d_%d" % (d, pi) for d in range(nd)]
            for d, ta in enumerate(tgt):
                w("const int %s = %s;" % (cn[d], ctx.expr(ta, rbind)))
            # target coordinates that do not depend on data are inside
            # the domain wherever the call passed the bounds validation;
            # only data-dependent ones (a bin index) are tested
            inb = " && ".join("%s >= d_%s_lo%d && %s <= d_%s_hi%d" % (
                cn[d], fnm, d, cn[d], fnm, d) for d in range(nd)
                if is_data_dependent(tgt[d])) or "true"
            cc = ctx.cond(cond, tbind) if cond is not None else "true"
            val = ctx.expr(expr, rbind) if shared else None
            w.open("if (pm_pt && (%s) && (%s))" % (inb, cc))
            if val is None:
                val = ctx.expr(expr, rbind)
            if priv:
                sidx = " + ".join("(%s - p_lo%d) * %d" % (
                    cn[d], d, _stride(plan.priv_ext, d)) for d in range(nd))
                w("%s(&acc[%s], (%s)(%s));" % (self.atomic(), sidx, T, val))
            else:
                gidx = " + ".join("(long long)(%s - d_%s_lo%d) * s_%s_%d" % (
                    cn[d], fnm, d, fnm, d) for d in range(nd))
                w("%s(&out[%s], (%s)(%s));" % (
                    self.atomic(self.part_ops[pi]), gidx, T, val))
            w.close()
            if not shared:
                w.close()
                ctx.pop()
        ctx.var_lo = saved_lo
        w.close()
        if priv:
            w("__syncthreads();")
            w.open("for (int i = threadIdx.x; i < %d; i += %d)" % (
                ptot, plan.threads))
            StencilGen.decompose(self, "i", plan.priv_ext, "j")
            for d in range(nd):
                w("const int c%d = p_lo%d + j%d;" % (d, d, d))
            w("if (%s) continue;" % " || ".join("c%d > p_hi%d" % (d, d)
                                               for d in range(nd)))
            w("const %s v = acc[i];" % T)
            w("if (v == %s) continue;" % ident)
            gidx = " + ".join("(long long)(c%d - d_%s_lo%d) * s_%s_%d" % (
                d, fnm, d, fnm, d) for d in range(nd))
            w("%s(&out[%s], v);" % (self.atomic(), gidx))
            w.close()
        w.close()
        w("")
        self.gen_launcher()

    def zero_default(self):
        """Whether the reduction's default is the constant 0 (all-zero
        bytes for every element type used here)."""
        d = Value.numericToValue(self.f.default)
        return isinstance(d, Value) and d.value == 0

    def spread_factor(self):
        """With option 'red_spread': the divisor k by which the innermost
        reduction variable indexes the target (a grid cell of k points),
        when the tile along it holds at least 32 cells of k; else 0."""
        if 'red_spread' not in self.pg.p.options:
            return 0
        from .evaluate import divisors_in
        plan = self.plan
        rv = self.f.reductionVariables[-1]
        ks = set()
        for fns in plan.target_fns:
            for fn in fns:
                if fn.kind == 'mono' and fn.var is rv:
                    ks.update(divisors_in(fn.expr))
        if len(ks) != 1:
            return 0
        k = ks.pop()
        E = plan.tile[-1]
        return k if k > 1 and E % k == 0 and E // k >= 32 else 0

    def gen_gather(self, ctx, parts):
        """Output-stationary accumulation (``plan.gather``): each thread
        owns target cells of the tile -- the points of the reduction
        variables that index the target -- and loops over the tile's range
        of the other reduction variables, combining in a register.  When
        the tile spans the whole range of those variables (one tile along
        them, the usual case) the thread is the cell's only writer and
        stores the default combined with its result; otherwise it combines
        into the cell with one atomic."""
        pg = self.pg
        w = pg.w
        plan = self.plan
        f = self.f
        fnm = pg.fn(f)
        T = ctype(f.typ)
        rvars = f.reductionVariables
        nr = len(rvars)
        tmap = plan.gather
        outer = [d for d in range(nr) if tmap[d] is not None]
        inner = [d for d in range(nr) if tmap[d] is None]
        lv = _loop_vars(nr)
        rbind = dict(zip(rvars, lv))
        op = self.op

        def combine(a, b):
            # a and b are names or literals (evaluated once each)
            if op == C.Op.Sum:
                return "%s + %s" % (a, b)
            if op == C.Op.Mul:
                return "%s * %s" % (a, b)
            # the atomics' rule: b replaces a when a < b (max), a > b (min)
            return "(%s %s %s) ? %s : %s" % (
                a, '<' if op == C.Op.Max else '>', b, b, a)

        whole = " && ".join("D.gn[%d] == 1" % d for d in inner) or "true"
        w("const bool pm_whole = %s;" % whole)
        otile = [plan.tile[d] for d in outer]
        tot = 1
        for t in otile:
            tot *= t
        saved_lo = dict(ctx.var_lo)
        for d, dom in enumerate(f.reductionDomain):
            lo = _const_int(dom.lowerBound)
            if lo is not None:
                ctx.var_lo["q%d" % d] = lo
        w.open("for (int i = threadIdx.x; i < %d; i += %d)" % (tot,
                                                               plan.threads))
        if outer:
            StencilGen.decompose(self, "i", otile, "o")
        for k, d in enumerate(outer):
            w("const int q%d = a_lo%d + o%d;" % (d, d, k))
        if outer:
            w("if (%s) continue;" % " || ".join("q%d > a_hi%d" % (d, d)
                                               for d in outer))
        w("%s acc = %s;" % (T, self.identity()))
        for d in inner:
            w.open("for (int q%d = a_lo%d; q%d <= a_hi%d; ++q%d)" % (
                d, d, d, d, d))
        for cond, expr, red in parts:
            tbind = tbind_of(f, rvars, red, rbind)
            ctx.push()
            w.open("")
            cc = ctx.cond(cond, tbind) if cond is not None and \
                not _cond_const_true(cond, tbind) else None
            if cc is not None:
                w.open("if (%s)" % cc)
            w("const %s v = (%s)(%s);" % (T, T, ctx.expr(expr, rbind)))
            w("acc = %s;" % combine("acc", "v"))
            if cc is not None:
                w.close()
            w.close()
            ctx.pop()
        for d in inner:
            w.close()
        # the cell: target dimension t is indexed by reduction variable d
        # with tmap[d] == t
        cell = dict((tmap[d], "q%d" % d) for d in outer)
        gidx = " + ".join("(long long)(%s - d_%s_lo%d) * s_%s_%d" % (
            cell[t], fnm, t, fnm, t) for t in range(f.ndims))
        dbind = dict((f.variables[tmap[d]], lv[d]) for d in outer)
        w.open("if (pm_whole)")
        w("const %s dflt = (%s)(%s);" % (T, T, ctx.expr(f.default, dbind)))
        w("out[%s] = %s;" % (gidx, combine("dflt", "acc")))
        w.close()
        w("else %s(&out[%s], acc);" % (self.atomic(), gidx))
        w.close()
        ctx.var_lo = saved_lo

    def atomic(self, op=None):
        return {C.Op.Sum: 'pm_atomic_add', C.Op.Mul: 'pm_atomic_mul',
                C.Op.Min: 'pm_atomic_min',
                C.Op.Max: 'pm_atomic_max'}[self.op if op is None else op]

    def identity(self):
        T = self.f.typ
        if self.op == C.Op.Sum:
            return "(%s)0" % ctype(T)
        if self.op == C.Op.Mul:
            return "(%s)1" % ctype(T)
        big = {C.Float: ("3.402823466e+38f", "-3.402823466e+38f"),
               C.Double: ("1.7976931348623157e+308", "-1.7976931348623157e+308"),
               C.Int: ("2147483647", "(-2147483647 - 1)"),
               C.UInt: ("4294967295u", "0u")}
        if T not in big:
            raise CodegenError("Min/Max reduction of %s unsupported" % T)
        return big[T][0] if self.op == C.Op.Min else big[T][1]

    def reader(self, f, args, ctx):
        pg = self.pg
        key = (pg.fn(f), tuple(ctx.index(a) if not is_data_dependent(a)
                                else ctx.expr(a, {}) for a in args))
        hit = ctx.lookup(key)
        if hit is not None:
            return hit
        t = ctx.temp()
        guard = pg.oob_guard(f, args, ctx)
        if guard is not None:
            # reads outside the image's domain yield 0 (option 'oob_zero')
            pg.w("const %s %s = (%s) ? __ldg(b_%s + (%s)) : (%s)0;" % (
                ctype(f.typ), t, guard, pg.fn(f), pg.gindex(f, args, ctx),
                ctype(f.typ)))
        else:
            pg.w("const %s %s = __ldg(b_%s + (%s));" % (
                ctype(f.typ), t, pg.fn(f), pg.gindex(f, args, ctx)))
        ctx.define(key, t)
        return t

    def gen_launcher(self):
        pg = self.pg
        plan = self.plan
        f = self.f
        w = pg.w
        k = self.k
        fnm = pg.fn(f)
        nr = len(f.reductionVariables)
        ctx = ExprCtx(w, 'device', pg.pmap, None)
        fill = "fill_" + k
        w.open("static int %s(%s_desc& D, const pm_args& A, const size_t* "
               "wsoff, long long* ntiles)" % (fill, k))
        pg.declare_params(w, "A")
        for prm in pg.params:
            w("D.%s = %s;" % (pg.pmap[prm], pg.pmap[prm]))
        for x in self.reads:
            w("D.b_%s = (const %s*)(%s);" % (pg.fn(x), ctype(x.typ),
                                             pg.buf_expr(x)))
        w("D.b_%s = (%s*)(%s);" % (fnm, ctype(f.typ), pg.buf_expr(f)))
        w("D.ncells = 1;")
        for d in f.domain:
            w("D.ncells *= (long long)pm_nonneg((%s) - (%s) + 1);" % (
                ctx.expr(d.upperBound, {}), ctx.expr(d.lowerBound, {})))
        pitch = pg.row_pitch(f)
        exts = ["(long long)pm_nonneg((%s) - (%s) + 1)" % (
            ctx.expr(d.upperBound, {}), ctx.expr(d.lowerBound, {}))
            for d in f.domain]
        if pitch > 1:
            exts[-1] = "((%s + %d) / %d * %d)" % (exts[-1], pitch - 1, pitch,
                                                  pitch)
        w("D.nbytes = (long long)%d * %s;" % (f.typ.size(), " * ".join(exts)))
        w("long long tot = 1;")
        for i, d in enumerate(f.reductionDomain):
            lo = ctx.expr(d.lowerBound, {})
            hi = ctx.expr(d.upperBound, {})
            w("D.glo[%d] = %s; D.ghi[%d] = %s;" % (i, lo, i, hi))
            w("if (D.ghi[%d] < D.glo[%d]) { *ntiles = 0; return PM_OK; }" % (
                i, i))
            w("D.gn[%d] = (D.ghi[%d] - D.glo[%d] + %d) / %d; tot *= D.gn[%d];"
              % (i, i, i, plan.tile[i], plan.tile[i], i))
        if plan.gather is not None and not self.mixed:
            # output-stationary: when the target variables' ranges cover
            # the domain and one tile spans the summed ones, every cell is
            # written once with its default folded in, and the init pass
            # is skipped
            cov = []
            for d, t in enumerate(plan.gather):
                if t is None:
                    cov.append("D.gn[%d] == 1" % d)
                else:
                    dom = f.domain[t]
                    cov.append("D.glo[%d] <= (%s) && D.ghi[%d] >= (%s)" % (
                        d, ctx.expr(dom.lowerBound, {}), d,
                        ctx.expr(dom.upperBound, {})))
            w("if (%s) D.ncells = 0;" % " && ".join(cov))
        w("*ntiles = tot;")
        w("return PM_OK;")
        w.close()
        w("")
        w("static bool %s_attr[64];     // per device" % k)
        w.open("static int launch_%s(pm_args& A, const size_t* wsoff, "
               "cudaStream_t s)" % k)
        w("%s_launch L; memset(&L, 0, sizeof(L));" % k)
        w("L.nimg = 1;")
        w("long long nt = 0;")
        w("int st = %s(L.d0, A, wsoff, &nt); if (st) return st;" % fill)
        if self.zero_default():
            # a default of 0: the init pass is a memset of the array (its
            # row padding included)
            w("if (L.d0.ncells > 0 && cudaMemsetAsync(L.d0.b_%s, 0, (size_t)"
              "L.d0.nbytes, s) != cudaSuccess) return PM_ERR_CUDA;" % fnm)
        else:
            w("if (L.d0.ncells > 0) %s_init<<<(unsigned)pm_llmin((L.d0.ncells"
              " + 255) / 256, 148LL * 16), 256, 0, s>>>(L);" % k)
        w("if (nt == 0) return cudaGetLastError() == cudaSuccess ? PM_OK : "
          "PM_ERR_CUDA;")
        w.open("if (!%s_attr[pm_cur_dev()])" % k)
        w("if (cudaFuncSetAttribute(%s, cudaFuncAttributeMaxDynamicShared"
          "MemorySize, %d) != cudaSuccess) return PM_ERR_CUDA;" % (
              k, max(plan.smem_bytes, 16)))
        w("%s_attr[pm_cur_dev()] = true;" % k)
        w.close()
        w("%s<<<(unsigned)nt, %d, %d, s>>>(L);" % (k, plan.threads,
                                                  max(plan.smem_bytes, 16)))
        w("return cudaGetLastError() == cudaSuccess ? PM_OK : PM_ERR_CUDA;")
        w.close()
        w("")
        w("static %s_launch pm_bl_%s;" % (k, k))
        w("static long long pm_bbase_%s = 0, pm_bcells_%s = 0;" % (k, k))
        w("static bool pm_bvalid_%s = false;" % k)
        w.open("static int batch_%s(pm_args* As, const size_t* wsoffs, int "
               "nslot, int n, char* pinned, char* ddesc, size_t* doff, "
               "cudaStream_t s, int replay)" % k)
        w.open("if (replay)")
        w("if (!pm_bvalid_%s) return PM_ERR_CUDA;" % k)
        w("if (pm_bcells_%s > 0) %s_init<<<(unsigned)pm_llmin((pm_bcells_%s + "
          "255) / 256, 148LL * 16), 256, 0, s>>>(pm_bl_%s);" % (k, k, k, k))
        w("if (pm_bbase_%s > 0) %s<<<(unsigned)pm_bbase_%s, %d, %d, s>>>"
          "(pm_bl_%s);" % (k, k, k, plan.threads, max(plan.smem_bytes, 16),
                           k))
        w("return cudaGetLastError() == cudaSuccess ? PM_OK : PM_ERR_CUDA;")
        w.close()
        w("pm_bvalid_%s = false;" % k)
        w("size_t off = (*doff + 63) & ~size_t(63);")
        w("%s_desc* H = reinterpret_cast<%s_desc*>(pinned + off);" % (k, k))
        w("long long base = 0, cells = 0;")
        w.open("for (int i = 0; i < n; ++i)")
        w("long long nt = 0;")
        w("int st = %s(H[i], As[i], wsoffs + (size_t)i * nslot, &nt); if (st) "
          "return st;" % fill)
        w("H[i].tile_base = (int)base; base += nt; cells += H[i].ncells;")
        w.close()
        w("*doff = off + sizeof(%s_desc) * n;" % k)
        w("if (cudaMemcpyAsync(ddesc + off, H, sizeof(%s_desc) * n, "
          "cudaMemcpyHostToDevice, s) != cudaSuccess) return PM_ERR_CUDA;" % k)
        w("cudaEventRecord(pm_batch_event[pm_cur_dev()], s);")
        w("%s_launch L; memset(&L, 0, sizeof(L));" % k)
        w("L.nimg = n; L.descs = reinterpret_cast<const %s_desc*>(ddesc + "
          "off);" % k)
        w("if (n == 1) L.d0 = H[0];")
        w("pm_bl_%s = L; pm_bbase_%s = base; pm_bcells_%s = cells; "
          "pm_bvalid_%s = base <= 0x7fffffffLL;" % (k, k, k, k))
        w("if (cells > 0) %s_init<<<(unsigned)pm_llmin((cells + 255) / 256, "
          "148LL * 16), 256, 0, s>>>(L);" % k)
        w("if (base == 0) return cudaGetLastError() == cudaSuccess ? PM_OK : "
          "PM_ERR_CUDA;")
        w("if (base > 0x7fffffffLL) return PM_ERR_UNSUPPORTED;")
        w.open("if (!%s_attr[pm_cur_dev()])" % k)
        w("if (cudaFuncSetAttribute(%s, cudaFuncAttributeMaxDynamicShared"
          "MemorySize, %d) != cudaSuccess) return PM_ERR_CUDA;" % (
              k, max(plan.smem_bytes, 16)))
        w("%s_attr[pm_cur_dev()] = true;" % k)
        w.close()
        w("%s<<<(unsigned)base, %d, %d, s>>>(L);" % (k, plan.threads,
                                                    max(plan.smem_bytes, 16)))
        w("return cudaGetLastError() == cudaSuccess ? PM_OK : PM_ERR_CUDA;")
        w.close()
        w("")
        pg.launch_fns.append("launch_" + k)
        pg.batch_fns.append("batch_" + k)
        pg.desc_sizes.append("sizeof(%s_desc)" % k)


def _stride(ext, d):
    s = 1
    for e in ext[d + 1:]:
        s *= e
    return s


# ---------------------------------------------------------------------------
class ConstGen(object):
    """Host tabulation + upload of a const function."""

    def __init__(self, pg, group):
        self.pg = pg
        self.g = group
        self.f = group.plan.func

    def generate(self):
        pg = self.pg
        f = self.f
        fnm = pg.fn(f)
        hw = pg.hw
        w = pg.w
        reads = []
        for r in f.getObjects(C.Reference):
            o = r.objectRef
            if o is not f and all(o is not q for q in reads):
                reads.append(o)
        for o in reads:
            if not (isinstance(o, C.Image) or o.is_const_func):
                raise CodegenError("const function %s reads non-const %s" % (
                    f.name, o.name))
        self.reads = reads
        pg.meta['groups'].append({'kernel': None, 'kind': 'const',
                                  'stages': [f.name]})
        pg.meta.setdefault('const', {})[f.name] = {
            'symbol': "pm_const_%s_%s" % (pg.pname, fnm),
            'params': [q.name for q in pg.params],
            'reads': [o.name for o in reads]}
        # ---- host C++ tabulation (compiled by g++ with the reference's
        # flags) ----
        hparams = ", ".join(["%s %s" % (pg.ptype(q), pg.pmap[q])
                             for q in pg.params] +
                            ["const %s* b_%s" % (ctype(o.typ), pg.fn(o))
                             for o in reads] +
                            ["%s* out" % ctype(f.typ)])
        hw('extern "C" void pm_const_%s_%s(%s)' % (pg.pname, fnm, hparams))
        hw.open("")
        ctx = ExprCtx(hw, 'host', pg.pmap, self.host_reader)
        self.ctx = ctx
        for o in reads + [f]:
            pg.declare_domain(hw, o, ctx, True)
        nd = f.ndims
        lv = _loop_vars(nd)
        for d in range(nd):
            hw.open("for (int q%d = d_%s_lo%d; q%d <= d_%s_hi%d; ++q%d)" % (
                d, fnm, d, d, fnm, d, d))
        ctx.push()
        bind = dict(zip(f.variables, lv))
        hw("%s v = 0;" % ctype(f.typ))
        parts = body_parts(f)
        if len(parts) == 1 and parts[0][0] is None:
            hw("v = (%s)(%s);" % (ctype(f.typ), ctx.expr(parts[0][1], bind)))
        else:
            first = True
            for cond, expr, red in reversed(parts):
                ctx.push()
                c = ctx.cond(cond, bind) if cond is not None else "true"
                hw.open("%sif (%s)" % ("" if first else "else ", c))
                hw("v = (%s)(%s);" % (ctype(f.typ), ctx.expr(expr, bind)))
                hw.close()
                ctx.pop()
                first = False
        idx = " + ".join("(long long)(q%d - d_%s_lo%d) * s_%s_%d" % (
            d, fnm, d, fnm, d) for d in range(nd))
        hw("out[%s] = v;" % idx)
        ctx.pop()
        for d in range(nd):
            hw.close()
        hw.close()
        hw("")
        # ---- device-side: cached upload -----------------------------------
        w('extern "C" void pm_const_%s_%s(%s);' % (pg.pname, fnm, hparams))
        dctx = ExprCtx(w, 'device', pg.pmap, None)
        ext = " * ".join("(size_t)pm_nonneg((%s) - (%s) + 1)" % (
            dctx.expr(d.upperBound, {}), dctx.expr(d.lowerBound, {}))
            for d in f.domain)
        w("static std::vector<char> ctab_key_%s;" % fnm)
        w("static std::vector<char> ctab_host_%s;" % fnm)
        w("static pm_arena ctab_dev_%s;" % fnm)
        w.open("static int launch_const_%s(pm_args& A, const size_t* wsoff, "
               "cudaStream_t s)" % fnm)
        pg.declare_params(w, "A")
        w("std::vector<char> key;")
        for q in pg.params:
            w("{ const char* p = (const char*)&%s; key.insert(key.end(), p, p "
              "+ sizeof(%s)); }" % (pg.pmap[q], pg.pmap[q]))
        hostbufs = []
        for o in reads:
            on = pg.fn(o)
            oext = " * ".join("(size_t)pm_nonneg((%s) - (%s) + 1)" % (
                dctx.expr(d.upperBound, {}), dctx.expr(d.lowerBound, {}))
                for d in o.domain)
            w("std::vector<char> hb_%s((size_t)%d * %s);" % (on, o.typ.size(),
                                                             oext))
            if isinstance(o, C.Image):
                w("if (!hb_%s.empty()) { if (pm_host_ptr(A.b_%s)) memcpy("
                  "hb_%s.data(), A.b_%s, hb_%s.size()); else if (cudaMemcpy"
                  "Async(hb_%s.data(), A.b_%s, hb_%s.size(), cudaMemcpyDevice"
                  "ToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != "
                  "cudaSuccess) return PM_ERR_CUDA; }" % (
                      on, on, on, on, on, on, on, on))
            else:
                w("hb_%s = ctab_host_%s;" % (on, on))
            w("key.insert(key.end(), hb_%s.begin(), hb_%s.end());" % (on, on))
            hostbufs.append("(const %s*)hb_%s.data()" % (ctype(o.typ), on))
        w("const size_t nb = (size_t)%d * %s;" % (f.typ.size(), ext))
        w.open("if (key != ctab_key_%s || ctab_host_%s.size() != nb)" % (
            fnm, fnm))
        w("ctab_host_%s.assign(nb, 0);" % fnm)
        args = [pg.pmap[q] for q in pg.params] + hostbufs + \
            ["(%s*)ctab_host_%s.data()" % (ctype(f.typ), fnm)]
        w("pm_const_%s_%s(%s);" % (pg.pname, fnm, ", ".join(args)))
        w("void* d = nullptr;")
        w("if (pm_arena_get(&ctab_dev_%s, nb, &d)) return PM_ERR_CUDA;" % fnm)
        w("if (cudaMemcpy(d, ctab_host_%s.data(), nb, cudaMemcpyHostToDevice)"
          " != cudaSuccess) return PM_ERR_CUDA;" % fnm)
        w("ctab_key_%s = key;" % fnm)
        w.close()
        w("void* d = nullptr;")
        w("if (pm_arena_get(&ctab_dev_%s, nb, &d)) return PM_ERR_CUDA;" % fnm)
        w("ctab_ptr_%s = (char*)d;" % fnm)
        w("return PM_OK;")
        w.close()
        w("")
        pg.const_ptrs.append(fnm)
        pg.launch_fns.append("launch_const_" + fnm)
        pg.batch_fns.append("batch_const_" + fnm)
        # A table computed from input images depends on their contents,
        # which a replayed batch does not look at: such pipelines never
        # replay.
        pg.const_replay.append((fnm, any(isinstance(o, C.Image)
                                         for o in reads)))
        w("static std::vector<char> pm_bctab_key_%s;" % fnm)
        w("static char* pm_bctab_ptr_%s = nullptr;" % fnm)
        w.open("static int batch_const_%s(pm_args* As, const size_t* wsoffs, "
               "int nslot, int n, char* pinned, char* ddesc, size_t* doff, "
               "cudaStream_t s, int replay)" % fnm)
        w("if (replay) return PM_OK;    // the table is already on the device")
        w("// one table for the batch: every image must use the same "
          "parameters")
        w.open("for (int i = 1; i < n; ++i)")
        for q in pg.params:
            w("if (As[i].%s != As[0].%s) return PM_ERR_UNSUPPORTED;" % (
                pg.pmap[q], pg.pmap[q]))
        w.close()
        w("int st = launch_const_%s(As[0], wsoffs, s);" % fnm)
        w("pm_bctab_key_%s = ctab_key_%s; pm_bctab_ptr_%s = ctab_ptr_%s;" % (
            fnm, fnm, fnm, fnm))
        w("return st;")
        w.close()
        w("")

    def host_reader(self, f, args, ctx):
        pg = self.pg
        t = ctx.temp()
        idx = pg.gindex(f, args, ctx)
        ctx.w("const %s %s = b_%s[%s];" % (ctype(f.typ), t, pg.fn(f), idx))
        return t


# ---------------------------------------------------------------------------
# ---------------------------------------------------------------------------
# Chain kernels: consecutive small stencil groups in one launch
CHAIN_DEFAULT_TILES = 512        # largest member group (tiles at estimates)
CHAIN_PARAM_BYTES = 28000        # kernel parameter budget of one chain


def _chain_limit(pipeline):
    """Option ``chain`` (``'chain'``, ``'chain=N'`` or ``('chain', N)``):
    runs of consecutive stencil groups of at most N tiles each (at the
    parameter estimates) become one launch; None when off."""
    v = _opt(pipeline, 'chain')
    if v is not None:
        return int(v)
    return CHAIN_DEFAULT_TILES if 'chain' in pipeline.options else None


def _launch_param_bytes(sg):
    """Upper estimate of sizeof(<k>_launch): tensor maps, parameters,
    buffer pointers, tile grid, launch fields."""
    pg = sg.pg
    na = sg.plan.anchor.ndims
    desc = 128 * len(sg.stage_nodes) + 8 * (len(pg.params) + len(sg.bufs)) \
        + 12 * na + 8 + 4 * len(sg.stage_nodes)
    desc = (desc + 63) // 64 * 64
    return desc + 64


def plan_chains(pg, pipeline):
    """Chains of launches: (member launch indices, phase of each member).

    A member is a stencil group's launch whose tile count at the parameter
    estimates is at most the option's limit (not prefetching, not launched
    with programmatic serialization, same CTA size as the others); members
    are consecutive in program order.  A member's phase is one more than
    the latest earlier member it has a read-after-write, write-after-read
    or write-after-write hazard with (0 without one): members of one phase
    run concurrently, a grid barrier separates phases."""
    limit = _chain_limit(pipeline)
    if limit is None or 'pdl' in pipeline.options:
        return []
    from .grouping import _comp_sizes
    sizes = _comp_sizes(pipeline)
    comp_of = pipeline.func_map

    def tiles(sg):
        s = sizes.get(comp_of.get(sg.plan.anchor))
        if s is None:
            return None
        return s / float(np.prod(sg.plan.tile))

    runs, cur = [], []
    for j in range(len(pg.launch_fns)):
        sg = pg.stencil_of.get(j)
        ok = sg is not None and not sg.prefetch and \
            j not in pg.launch_main and tiles(sg) is not None and \
            tiles(sg) <= limit
        if ok and cur:
            first = pg.stencil_of[cur[0]]
            size = sum(_launch_param_bytes(pg.stencil_of[i]) for i in cur)
            if sg.plan.threads != first.plan.threads or \
                    sg.launch_bounds != first.launch_bounds or \
                    size + _launch_param_bytes(sg) > CHAIN_PARAM_BYTES:
                runs.append(cur)
                cur = []
        if ok:
            cur.append(j)
        else:
            if cur:
                runs.append(cur)
            cur = []
    if cur:
        runs.append(cur)
    chains = []
    for run in runs:
        if len(run) < 2:
            continue
        phase = {}
        for j in run:
            rj, wj = pg.launch_rw[j]
            p = 0
            for i in run:
                if i >= j:
                    break
                ri, wi = pg.launch_rw[i]
                if (wi & rj) or (ri & wj) or (wi & wj):
                    p = max(p, phase[i] + 1)
            phase[j] = p
        chains.append((run, [phase[j] for j in run]))
    return chains


def gen_chains(pg, pipeline):
    """Emit one kernel per chain (``pm_<name>_chain<c>``) that runs its
    members' kernel bodies phase by phase, with a bounded grid barrier
    (``pm_grid_sync``) between phases, and its host launcher; the chain
    replaces its members in the launch list of the single-image entry
    points (batches keep the per-group kernels).  The grid is the largest
    phase's tile count, capped by the CTAs resident on the GPU at once, so
    every CTA of the launch is on the GPU together."""
    chains = plan_chains(pg, pipeline)
    if not chains:
        return
    w = pg.w
    w("// ---- chain kernels: consecutive small groups in one launch")
    w("__device__ unsigned pm_chain_ctr[%d];   // grid-barrier counters" %
      len(chains))
    w("// per device: the counters' address, looked up on the first chain")
    w("// launch (cudaDeviceReset reloads the module and invalidates it)")
    w("static unsigned* pm_chain_ctr_ptr[64];")
    w.open("static unsigned* pm_chain_counters()")
    w("const int dev = pm_cur_dev();")
    w.open("if (!pm_chain_ctr_ptr[dev])")
    w("void* p = nullptr;")
    w("if (cudaGetSymbolAddress(&p, pm_chain_ctr) != cudaSuccess) return "
      "nullptr;")
    w("pm_chain_ctr_ptr[dev] = static_cast<unsigned*>(p);")
    w.close()
    w("return pm_chain_ctr_ptr[dev];")
    w.close()
    w("")
    replace = {}
    pg.meta['chains'] = []
    for c, (run, phases) in enumerate(chains):
        sgs = [pg.stencil_of[j] for j in run]
        ck = "pm_%s_chain%d" % (pg.pname, c)
        nt = sgs[0].plan.threads
        smem = max(sg.plan.smem_bytes for sg in sgs)
        nph = max(phases) + 1
        w("// chain %d: %s in %d phases" % (
            c, ", ".join("%s (phase %d)" % (sg.k, p)
                         for sg, p in zip(sgs, phases)), nph))
        w.open("struct %s_launch" % ck)
        for m, sg in enumerate(sgs):
            w("%s_launch m%d;" % (sg.k, m))
        w("unsigned* ctr;        // grid-barrier counter, zeroed per launch")
        w("int rot[%d];          // CTA of each member's first tile" %
          len(sgs))
        w.close("};")
        w("static_assert(sizeof(%s_launch) <= 32000, \"chain parameters\");"
          % ck)
        w('extern "C" __global__ void __launch_bounds__(%s) %s(const '
          '__grid_constant__ %s_launch C)' % (sgs[0].launch_bounds, ck, ck))
        w.open("")
        w("const int nb = (int)gridDim.x, b = (int)blockIdx.x;")
        for p in range(nph):
            if p:
                w("if (!pm_grid_sync(C.ctr, %du * (unsigned)nb, "
                  "&pm_err_word)) return;" % p)
            w("// phase %d" % p)
            for m, (sg, q) in enumerate(zip(sgs, phases)):
                if q == p:
                    w("%s_body<true>(C.m%d, (b + nb - C.rot[%d]) %% nb, nb);"
                      % (sg.k, m, m))
        w.close()
        w("static bool %s_attr[64];     // per device" % ck)
        w("static int %s_resident[64];  // per device" % ck)
        w.open("static int launch_%s(pm_args& A, const size_t* wsoff, "
               "cudaStream_t s)" % ck)
        w("%s_launch C; memset(&C, 0, sizeof(C));" % ck)
        w("long long nt = 0, ph[%d] = {0};" % nph)
        w("int st = PM_OK;")
        for m, (sg, q) in enumerate(zip(sgs, phases)):
            w("if ((st = fill_%s(C.m%d.d0, A, wsoff, &nt))) return st;" % (
                sg.k, m))
            w("if (nt > 0x7fffffffLL) return PM_ERR_UNSUPPORTED;")
            w("C.m%d.nimg = 1; C.m%d.total = (int)nt; C.m%d.stride = 1;" % (
                m, m, m))
            w("C.rot[%d] = (int)(ph[%d] & 0x7fffffff); ph[%d] += nt;" % (
                m, q, q))
        w("long long need = 0;")
        w("for (int p = 0; p < %d; ++p) need = pm_llmax(need, ph[p]);" % nph)
        w("if (need == 0) return PM_OK;")
        w("const int dev = pm_cur_dev();")
        w.open("if (!%s_attr[dev])" % ck)
        w("if (cudaFuncSetAttribute(%s, cudaFuncAttributeMaxDynamicShared"
          "MemorySize, %d) != cudaSuccess) return PM_ERR_CUDA;" % (ck, smem))
        w("int per_sm = 0, sms = 0;")
        w("if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, "
          "dev) != cudaSuccess || cudaOccupancyMaxActiveBlocksPerMultiprocessor"
          "(&per_sm, %s, %d, %d) != cudaSuccess || per_sm < 1) return "
          "PM_ERR_CUDA;" % (ck, nt, smem))
        w("%s_resident[dev] = per_sm * sms;" % ck)
        w("%s_attr[dev] = true;" % ck)
        w.close()
        w("const long long grid = pm_llmin(need, %s_resident[dev]);" % ck)
        w("for (int m = 0; m < %d; ++m) C.rot[m] = (int)(C.rot[m] %% grid);"
          % len(sgs))
        w("unsigned* ctr = pm_chain_counters();")
        w("if (!ctr) return PM_ERR_CUDA;")
        w("C.ctr = ctr + %d;" % c)
        w("if (cudaMemsetAsync(C.ctr, 0, sizeof(unsigned), s) != cudaSuccess)"
          " return PM_ERR_CUDA;")
        w("%s<<<(unsigned)grid, %d, %d, s>>>(C);" % (ck, nt, smem))
        w("return cudaGetLastError() == cudaSuccess ? PM_OK : PM_ERR_CUDA;")
        w.close()
        w("")
        replace[run[0]] = ("launch_" + ck, run)
        pg.meta['chains'].append({
            'kernel': ck, 'members': [sg.k for sg in sgs],
            'phases': phases, 'smem': smem, 'threads': nt})
    # the chains take their members' places in the launch list
    fns, rw, main = [], [], []
    member = set(j for run, _ in chains for j in run)
    for j in range(len(pg.launch_fns)):
        if j in replace:
            fn, run = replace[j]
            reads, writes = set(), set()
            for i in run:
                reads |= pg.launch_rw[i][0]
                writes |= pg.launch_rw[i][1]
            fns.append(fn)
            rw.append((reads, writes))
        elif j not in member:
            if j in pg.launch_main:
                main.append(len(fns))
            fns.append(pg.launch_fns[j])
            rw.append(pg.launch_rw[j])
    pg.launch_fns, pg.launch_rw, pg.launch_main = fns, rw, main


def generate_code_for_pipeline(pipeline):
    pg = PipelineGen(pipeline)
    pg.slot_of = getattr(pipeline, '_storage_assign', {})
    pg.nslots = len(getattr(pipeline, '_storage_slots', []))
    pg.launch_fns = []
    pg.batch_fns = []
    pg.band_groups = []
    pg.desc_sizes = []
    pg.const_ptrs = []
    pg.const_replay = []
    # const tables are addressed through ctab pointers set by their launch
    pg.buf_expr_orig = pg.buf_expr
    body = W()
    pg_w = pg.w
    pg.w = body
    # generate groups into `body` first so helper declarations can precede
    pg.launch_rw = []
    pg.launch_main = []
    pg.stencil_of = {}
    pg.conc_streams = 0
    pg.conc_events = 0
    for g in pipeline.groups:
        plan = g.plan
        n0 = len(pg.launch_fns)
        if plan.kind == 'stencil':
            sg = StencilGen(pg, g)
            sg.generate()
            pg.stencil_of[n0] = sg
        elif plan.kind == 'reduction':
            ReductionGen(pg, g).generate()
        else:
            ConstGen(pg, g).generate()
            # const tables are computed and uploaded on the host, in
            # program order on the caller's stream
            pg.launch_main.append(n0)
        if len(pg.launch_fns) != n0 + 1:
            raise CodegenError("group %s: expected one launch" % (
                [c.func.name for c in g.comps],))
        pg.launch_rw.append(pg.group_rw(g))
    pg.group_launch_rw = list(pg.launch_rw)
    pg.group_launch_main = list(pg.launch_main)
    gen_chains(pg, pipeline)
    # kernel launches of one single-image call (a Reduction: its init
    # and accumulation; a chain: one for all its members)
    pg.meta['launches'] = sum(
        {'stencil': 1, 'reduction': 2}.get(g.plan.kind, 0)
        for g in pipeline.groups) - sum(
            len(ch['members']) - 1 for ch in pg.meta.get('chains', []))
    pg.w = pg_w
    w = pg.w
    w("// pipeline %s -- generated by polymage_b200 for sm_100a" %
      pipeline.name)
    w('#include "pm_runtime.cuh"')
    w("#include <vector>")
    w("")
    w("__device__ unsigned pm_err_word;")
    w("static int pm_status = 0;")
    w("static cudaEvent_t pm_batch_event[64];   // per device")
    w("static inline long long pm_nonneg(long long v) { return v < 0 ? 0 : v;"
      " }")
    w("static inline long long pm_llmin(long long a, long long b) { return a "
      "< b ? a : b; }")
    w("static inline long long pm_llmax(long long a, long long b) { return a "
      "> b ? a : b; }")
    w("static inline int isl_min_i(int a, int b) { return a < b ? a : b; }")
    w("static inline int pm_mod(int a, int k) { int m = a % k; return m < 0 "
      "? m + k : m; }")
    w("static inline int pm_next_res(int lo, int k, int r) { return lo + "
      "pm_mod(r - lo, k); }")
    w("static inline int pm_prev_res(int hi, int k, int r) { return hi - "
      "pm_mod(hi - r, k); }")
    w("static inline int isl_max_i(int a, int b) { return a > b ? a : b; }")
    w("static bool pm_use_tma() { static int v = -1; if (v < 0) { const char*"
      " e = getenv(\"PM_DISABLE_TMA\"); v = (e && e[0] == '1') ? 0 : 1; } "
      "return v == 1; }")
    w("static void pm_key_add(std::vector<char>& k, const void* p, size_t n)"
      " { if (n) k.insert(k.end(), (const char*)p, (const char*)p + n); }")
    w("static bool pm_persistent() { static int v = -1; if (v < 0) { const "
      "char* e = getenv(\"PM_PERSISTENT\"); v = (e && e[0] == '0') ? 0 : 1; }"
      " return v == 1; }")
    w("static bool pm_host_ptr(const void* p) { cudaPointerAttributes a; if "
      "(cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError();"
      " return true; } return a.type != cudaMemoryTypeDevice && a.type != "
      "cudaMemoryTypeManaged; }")
    for fnm in pg.const_ptrs:
        w("static char* ctab_ptr_%s = nullptr;" % fnm)
    w("")
    pg.gen_args_struct()
    pg.gen_validate()
    pg.gen_workspace()
    w.lines.extend(body.lines)
    # per group: up to 63 B of alignment before its descriptors, then up to
    # 63 B more and 64 B for its tile-queue counter
    w("static size_t pm_batch_desc_bytes(int n) { return (size_t)n * (%s) + "
      "192 * %d; }" % (" + ".join(pg.desc_sizes) or "0",
                       len(pg.desc_sizes) + 1))
    w("")
    ent = W()
    pg.w = ent
    pg.gen_entries()
    pg.w = w
    if pg.conc_streams:
        # per device: side streams and events of the concurrent schedule
        w("static cudaStream_t pm_side_stream[64][%d];" % pg.conc_streams)
        w("static cudaEvent_t pm_conc_event[64][%d];" % pg.conc_events)
        w.open("static int pm_conc_get(cudaStream_t* ss, int nside, int nev, "
               "cudaEvent_t** ev)")
        w("int dev = 0;")
        w("if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) "
          "return PM_ERR_CUDA;")
        w.open("for (int k = 0; k < nside; ++k)")
        w("if (!pm_side_stream[dev][k] && cudaStreamCreateWithFlags("
          "&pm_side_stream[dev][k], cudaStreamNonBlocking) != cudaSuccess) "
          "return PM_ERR_CUDA;")
        w("ss[k + 1] = pm_side_stream[dev][k];")
        w.close()
        w("for (int e = 0; e < nev; ++e)")
        w("  if (!pm_conc_event[dev][e] && cudaEventCreateWithFlags("
          "&pm_conc_event[dev][e], cudaEventDisableTiming) != cudaSuccess) "
          "return PM_ERR_CUDA;")
        w("*ev = pm_conc_event[dev];")
        w("return PM_OK;")
        w.close()
        w("")
    w.lines.extend(ent.lines)
    header = pg.gen_header()
    return CudaModule(pipeline.name, w.text(), pg.host_text(), header,
                      pg.meta)
