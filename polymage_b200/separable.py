"""Separable rewrite of rectangular weighted sums (option ``separable``).

A stage whose value is a sum of weighted reads of one producer over a
rectangle of offsets in two of its dimensions,

    S(x, y) = sum_{a in A, b in B} W[a][b] * P(x + a, y + b),

with a rank-one weight matrix W[a][b] = u[a] * v[b] (box sums, Sobel
derivatives, binomial blurs) is rewritten as

    S(x, y) = sum_a u[a] * R_a,   R_a = sum_b v[b] * P(x + a, y + b).

R_a at output row x is the same expression as R_{a-1} at row x + 1, so the
rows a thread computes in its register block share their row sums (nvcc
eliminates the repeated expressions): a 3x3 box sum costs 2 + 2 * 6 / 4
additions per output in a 4-row block instead of 8.  Only the
association of the sum changes (exactly representable weights, same
terms), so results differ from the spec's left-to-right order by rounding
only; the rewrite is applied to floating-point stages only (integer stages
keep their exact C semantics), and to rectangles of at least six terms
(smaller ones have no rows to share).

The reference evaluates the spec's expression as written
(sandbox/codegen.py:574-715); this pass has no counterpart there.
"""

from fractions import Fraction

from . import constructs as C
from .expr_ast import Value, AbstractBinaryOpNode, make_binop
from .expression import affine_form, rebuild

MIN_TERMS = 6


def _terms(e):
    if isinstance(e, AbstractBinaryOpNode) and e.op == '+':
        return _terms(e.left) + _terms(e.right)
    return [e]


def _weighted_ref(t):
    """(weight, reference) of ``ref`` or ``ref * c`` / ``c * ref``."""
    if isinstance(t, C.Reference):
        return Fraction(1), t
    if isinstance(t, AbstractBinaryOpNode) and t.op == '*':
        for r, c in ((t.left, t.right), (t.right, t.left)):
            if isinstance(r, C.Reference) and isinstance(c, Value) and \
                    isinstance(c.value, (int, float)) and \
                    c.typ in (C.Float, C.Double, C.Int):
                return Fraction(c.value), r
    return None


def _offsets(ref):
    """Per argument: (variable, offset) for ``v + c``, or None."""
    out = []
    for a in ref.arguments:
        f = affine_form(a)
        if f is None or len(f[0]) != 1:
            return None
        (v, k), = f[0].items()
        if k != 1 or not isinstance(v, C.Variable):
            return None
        out.append((v, f[1]))
    return out


def _factor(terms):
    """(pa, pb, {a: u}, {b: v}, {(a, b): ref}) of a rank-one rectangle of
    reads of one producer, or None."""
    if len(terms) < MIN_TERMS:
        return None
    wr = [_weighted_ref(t) for t in terms]
    if any(x is None for x in wr):
        return None
    prod = wr[0][1].objectRef
    if any(r.objectRef is not prod for _, r in wr):
        return None
    offs = [_offsets(r) for _, r in wr]
    if any(o is None for o in offs):
        return None
    nd = len(offs[0])
    if any(len(o) != nd for o in offs):
        return None
    # every argument reads the same variable in every term; exactly two
    # arguments vary
    vary = []
    for p in range(nd):
        if len(set(id(o[p][0]) for o in offs)) != 1:
            return None
        if len(set(o[p][1] for o in offs)) > 1:
            vary.append(p)
    if len(vary) != 2:
        return None
    pa, pb = vary
    W, refs = {}, {}
    for (w, r), o in zip(wr, offs):
        key = (o[pa][1], o[pb][1])
        if key in W:
            return None
        W[key] = w
        refs[key] = r
    A = sorted(set(a for a, _ in W))
    B = sorted(set(b for _, b in W))
    if len(A) < 2 or len(B) < 2 or len(W) != len(A) * len(B):
        return None
    a0, b0 = A[0], B[0]
    if W[(a0, b0)] == 0:
        return None
    v = dict((b, W[(a0, b)]) for b in B)
    u = dict((a, W[(a, b0)] / W[(a0, b0)]) for a in A)
    for a in A:
        for b in B:
            if u[a] * v[b] != W[(a, b)]:
                return None
    # weights exactly representable as doubles (the spec's own are)
    for x in list(u.values()) + list(v.values()):
        if Fraction(float(x)) != x:
            return None
    return pa, pb, u, v, refs


def _weight(w, e):
    if w == 1:
        return e
    return make_binop('*', e, Value(float(w), C.Float))


def _rewrite_sum(e):
    f = _factor(_terms(e))
    if f is None:
        return None
    pa, pb, u, v, refs = f
    total = None
    for a in sorted(u):
        r = None
        for b in sorted(v):
            t = _weight(v[b], rebuild(refs[(a, b)], lambda n: None))
            r = t if r is None else make_binop('+', r, t)
        if total is not None and u[a] == -1:
            total = make_binop('-', total, r)
            continue
        t = _weight(u[a], r)
        total = t if total is None else make_binop('+', total, t)
    return total


def _leaf(n):
    if isinstance(n, AbstractBinaryOpNode) and n.op == '+':
        return _rewrite_sum(n)
    return None


def separable_pass(pipeline):
    """Rewrite the rank-one rectangular sums of every floating-point stage
    of ``pipeline`` (its own cloned functions) in place; returns the names
    of the stages changed."""
    changed = []
    for comp in pipeline.comps:
        f = comp.func
        if f.typ not in (C.Float, C.Double) or isinstance(f, C.Reduction) \
                or f.is_const_func:
            continue
        parts, hit = [], False
        for p in f.defn:
            if isinstance(p, C.Case) and not isinstance(p.expression,
                                                        C.Reduce):
                e = rebuild(p.expression, _leaf)
                hit = hit or str(e) != str(p.expression)
                parts.append(C.Case(p.condition, e))
            elif not isinstance(p, (C.Case, C.Reduce)):
                e = rebuild(p, _leaf)
                hit = hit or str(e) != str(p)
                parts.append(e)
            else:
                parts.append(p)
        if hit:
            f._body = parts
            changed.append(f.name)
    return changed
