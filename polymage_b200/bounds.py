"""Bounds check: every affine reference must stay inside the producer's
domain (sandbox/bounds.py:36-118, which raises
``TypeError("Reference out of domain", ...)``).

The reference asks isl whether the set of referenced points leaves the
domain.  All pipelines this backend accepts have box domains, so a part's
iteration space is a box (its domain narrowed by the single-variable affine
conjuncts of its ``Case`` condition) and the referenced range of an index
expression that is monotone in each variable is attained at box corners.
Conditions that are not single-variable affine act as predicates and are
ignored, as the reference does for non-affine conditions
(sandbox/poly.py:656-683).

The same symbolic boxes are kept on the pipeline (``_bounds_checks``) so the
generated host code can repeat the check for the parameter values of each
call and refuse a call that would read out of bounds, instead of letting a
kernel read outside a buffer.
"""

import logging

from .expr_ast import Value
from . import constructs as C
from .expression import affine_form
from .evaluate import eval_int, EvalError, monotone_dir

LOG = logging.getLogger("polymage_b200.bounds")


class PartBox(object):
    """Iteration box of one definition piece.

    ``lo[v]`` / ``hi[v]`` are lists of expressions over parameters whose
    max / min bound variable ``v``; ``exact`` is False when some condition
    could not be expressed as variable bounds (the box over-approximates the
    piece)."""

    def __init__(self, variables):
        self.variables = list(variables)
        self.lo = dict((v, []) for v in variables)
        self.hi = dict((v, []) for v in variables)
        self.exact = True

    def copy(self):
        b = PartBox(self.variables)
        b.lo = dict((v, list(l)) for v, l in self.lo.items())
        b.hi = dict((v, list(l)) for v, l in self.hi.items())
        b.exact = self.exact
        return b

    def evaluate(self, env):
        out = {}
        for v in self.variables:
            lo = max(eval_int(e, env) for e in self.lo[v])
            hi = min(eval_int(e, env) for e in self.hi[v])
            out[v] = (lo, hi)
        return out


def _split_linear(e, variables):
    """(coeffs of loop variables, remainder) of ``e`` when ``e`` is a sum
    of integer multiples of loop variables and variable-free terms (which
    may be any parameter expression, divisions included); None otherwise."""
    e = Value.numericToValue(e)
    vs = [v for v in e.collect(C.Variable) if not isinstance(v, C.Parameter)]
    if not vs:
        return {}, e
    if isinstance(e, C.Variable):
        if any(e is v for v in variables):
            return {e: 1}, Value(0, C.Int)
        return None
    from .expr_ast import AbstractBinaryOpNode, AbstractUnaryOpNode
    if isinstance(e, AbstractUnaryOpNode):
        r = _split_linear(e.child, variables)
        if r is None:
            return None
        if e.op == '-':
            return dict((k, -c) for k, c in r[0].items()), 0 - r[1]
        return r
    if isinstance(e, AbstractBinaryOpNode):
        if e.op in ('+', '-'):
            a = _split_linear(e.left, variables)
            b = _split_linear(e.right, variables)
            if a is None or b is None:
                return None
            s = 1 if e.op == '+' else -1
            co = dict(a[0])
            for k, c in b[0].items():
                co[k] = co.get(k, 0) + s * c
            return co, (a[1] + b[1]) if s == 1 else (a[1] - b[1])
        if e.op == '*':
            for lin, k in ((e.left, e.right), (e.right, e.left)):
                k = Value.numericToValue(k)
                if isinstance(k, Value) and isinstance(k.value, int):
                    r = _split_linear(lin, variables)
                    if r is None:
                        return None
                    return (dict((v, c * k.value) for v, c in r[0].items()),
                            r[1] * k.value)
        return None
    return None


def _var_bound(cmp_cond, variables):
    """Translate ``a*v + rest (op) 0`` with a = +-1 into bounds on v.
    Returns ('lo'|'hi'|'eq', v, expr) items, or None if not of that form."""
    lf = _split_linear(cmp_cond.lhs, variables)
    rf = _split_linear(cmp_cond.rhs, variables)
    if lf is None or rf is None:
        return None
    coeffs = dict(lf[0])
    for k, c in rf[0].items():
        coeffs[k] = coeffs.get(k, 0) - c
    vs = [k for k, c in coeffs.items() if c != 0]
    if len(vs) != 1 or not any(vs[0] is v for v in variables):
        return None
    v = vs[0]
    a = coeffs[v]
    if a not in (1, -1):
        return None
    # condition: a*v + rest op 0
    rest = lf[1] - rf[1]
    # v op' (-rest)/a
    op = cmp_cond.conditional
    if a == -1:
        op = {'<': '>', '<=': '>=', '>': '<', '>=': '<=', '==': '==',
              '!=': '!='}[op]
        bound = rest            # -v + rest op 0  <=>  v op' rest
    else:
        bound = 0 - rest        # v + rest op 0   <=>  v op  -rest
    if op == '<':
        return [('hi', v, bound - 1)]
    if op == '<=':
        return [('hi', v, bound)]
    if op == '>':
        return [('lo', v, bound + 1)]
    if op == '>=':
        return [('lo', v, bound)]
    if op == '==':
        return [('lo', v, bound), ('hi', v, bound)]
    return None


def narrow_box(box, conjunct):
    """Apply a list of comparisons (one DNF conjunct) to a box."""
    b = box.copy()
    for cmp_cond in conjunct:
        items = _var_bound(cmp_cond, b.variables)
        if items is None:
            b.exact = False
            continue
        for kind, v, e in items:
            if kind == 'lo':
                b.lo[v].append(e)
            else:
                b.hi[v].append(e)
    return b


def domain_box(variables, domain):
    b = PartBox(variables)
    for v, d in zip(variables, domain):
        b.lo[v].append(d.lowerBound)
        b.hi[v].append(d.upperBound)
    return b


def part_boxes(func):
    """[(box, cond, expr, reduce)] for every DNF conjunct of every piece of
    ``func``'s definition."""
    from .pipe import body_parts
    out = []
    for cond, expr, red in body_parts(func):
        if red is not None:
            base = domain_box(func.reductionVariables, func.reductionDomain)
        else:
            base = domain_box(func.variables, func.domain)
        if cond is None:
            out.append((base, cond, expr, red))
            continue
        if cond.has(C.Reference) or not _affine_cond(cond):
            b = base.copy()
            b.exact = False
            out.append((b, cond, expr, red))
            continue
        for conj in cond.split_to_conjuncts():
            out.append((narrow_box(base, conj), cond, expr, red))
    return out


def _affine_cond(cond):
    from .expression import isAffine
    try:
        return isAffine(cond)
    except TypeError:
        return False


def expr_range(expr, ranges, env):
    """(lo, hi) of an integer expression over a box of variables, or None
    when the expression is not monotone in each of its variables."""
    vs = [v for v in expr.collect(C.Variable)
          if not isinstance(v, C.Parameter)]
    if expr.has(C.Reference):
        return None
    lo_env = dict(env)
    hi_env = dict(env)
    for v in vs:
        if v not in ranges:
            return None
        d = monotone_dir(expr, v)
        if d is None:
            return None
        lo, hi = ranges[v]
        if d >= 0:
            lo_env[v], hi_env[v] = lo, hi
        else:
            lo_env[v], hi_env[v] = hi, lo
    try:
        return eval_int(expr, lo_env), eval_int(expr, hi_env)
    except EvalError:
        return None


def modular_restriction(cond):
    """``(v, k, r)`` when ``cond`` is ``v % k == r`` (or ``!=`` with k = 2,
    i.e. the other residue) for a loop variable ``v`` and constants k > 0,
    0 <= r < k; else None.  The reference splits a Select on such a
    condition into one domain per arm (sandbox/poly.py:761-879)."""
    from .expr_ast import AbstractBinaryOpNode
    if cond.conditional not in ('==', '!='):
        return None
    lhs = Value.numericToValue(cond.lhs)
    rhs = Value.numericToValue(cond.rhs)
    if not (isinstance(lhs, AbstractBinaryOpNode) and lhs.op == '%'):
        return None
    v = lhs.left
    k = Value.numericToValue(lhs.right)
    if not (isinstance(v, C.Variable) and not isinstance(v, C.Parameter)):
        return None
    if not (isinstance(k, Value) and isinstance(k.value, int) and
            k.value > 0 and isinstance(rhs, Value) and
            isinstance(rhs.value, int) and 0 <= rhs.value < k.value):
        return None
    if cond.conditional == '==':
        return (v, k.value, rhs.value)
    if k.value == 2:
        return (v, 2, 1 - rhs.value)
    return None


def refs_with_residues(expr, restr=()):
    """[(reference, ((v, k, r), ...))]: every reference of ``expr`` with the
    residue classes its enclosing Select arms restrict variables to."""
    out = []
    if isinstance(expr, C.Reference):
        out.append((expr, tuple(restr)))
        for a in expr.arguments:
            out += refs_with_residues(a, restr)
        return out
    if isinstance(expr, C.Select):
        m = modular_restriction(expr.condition)
        out += refs_with_residues(expr.condition, restr)
        if m is not None:
            v, k, r = m
            other = (v, k, 1 - r) if k == 2 else None
            out += refs_with_residues(expr.true_expression,
                                      tuple(restr) + (m,))
            out += refs_with_residues(expr.false_expression,
                                      tuple(restr) + ((other,) if other
                                                      else ()))
            return out
    for ch in (expr.children() if hasattr(expr, 'children') else []):
        out += refs_with_residues(ch, restr)
    return out


def restrict_range(lo, hi, k, r):
    """[lo, hi] shrunk to its extreme members congruent to r mod k."""
    lo2 = lo + ((r - lo) % k)
    hi2 = hi - ((hi - r) % k)
    return lo2, hi2


def bounds_check_pass(pipeline):
    """Check every reference of every compute object at the parameter
    estimates; record the symbolic checks for the run-time validator.

    With option 'oob_zero' a read outside the producer's domain is not
    refused: the producer and dimension are recorded in
    ``pipeline._oob_dims`` ({producer: set of dims}) and the generated
    code reads 0 there (the convention of points nothing defines); such
    reads get no run-time check."""
    env = pipeline.int_env()
    checks = []
    oob_zero = 'oob_zero' in pipeline.options
    pipeline._oob_dims = {}
    for comp in pipeline.comps:
        f = comp.func
        for box, cond, expr, red in part_boxes(f):
            try:
                rng = box.evaluate(env)
            except EvalError:
                continue
            if any(lo > hi for lo, hi in rng.values()):
                continue
            refs = refs_with_residues(expr)
            if cond is not None:
                refs += [(r, ()) for r in cond.collect(C.Reference)]
            if red is not None:
                refs += [(red.accumulate_ref, ())]
                for a in red.accumulate_ref.arguments:
                    refs += [(r, ()) for r in a.collect(C.Reference)]
            for ref, restr in refs:
                g = ref.objectRef
                is_target = (red is not None and ref is red.accumulate_ref)
                rr = dict(rng)
                for (v, k, r) in restr:
                    if v in rr:
                        rr[v] = restrict_range(rr[v][0], rr[v][1], k, r)
                if any(lo > hi for lo, hi in rr.values()):
                    continue
                for dim, (arg, dom) in enumerate(zip(ref.arguments,
                                                     g.domain)):
                    r = expr_range(arg, rr, env)
                    if r is None:
                        continue
                    dlo = eval_int(dom.lowerBound, env)
                    dhi = eval_int(dom.upperBound, env)
                    if oob_zero and not is_target and \
                            (r[0] < dlo or r[1] > dhi):
                        pipeline._oob_dims.setdefault(g, set()).add(dim)
                        continue
                    checks.append((comp, box, arg, g, dim, is_target,
                                   restr))
                    if r[0] < dlo or r[1] > dhi:
                        LOG.error("Reference out of domain: %s in %s, dim %d"
                                  " referenced [%d, %d], domain [%d, %d]",
                                  ref, f.name, dim, r[0], r[1], dlo, dhi)
                        raise TypeError("Reference out of domain", f.name,
                                        str(ref), dim, r, (dlo, dhi))
    pipeline._bounds_checks = checks
