"""User-facing constructs of the PolyMage language.

Same names, constructor arguments and semantics as the reference front end
(sandbox/constructs.py): ``Variable``/``Parameter`` (:321, :343),
``Interval`` (:347), ``Reference`` (:383), ``Stencil`` (:544, macro expansion
:673), ``TStencil`` (:689), ``Condition`` (:722, ``split_to_conjuncts`` :767),
``Case`` (:806), ``Op``/``Reduce`` (:842, :848), ``Function`` (:907),
``Image`` (:1066), ``Reduction`` (:1092), the math builtins (:77-211),
``Cast`` (:213), ``Select`` (:256) and ``Max``/``Min`` as selects (:312-319).

Differences, all additive: every object keeps the same public properties, and
functions gain helpers the backend uses (``is_reduction``, ``dims`` ...).
"""

import math

from .expr_types import (Void, Float, Double, Int, UInt, Short, UShort, Char,
                         UChar, Long, ULong, Rational, result_type)
from .expr_ast import (AbstractExpression, Value, AbstractBinaryOpNode,
                       AbstractUnaryOpNode, InbuiltFunction, Add, Sub, Mul,
                       Div, Mod, LShift, RShift, LAnd, LOr, Xor, UnaryMinus,
                       UnaryPlus)

__all__ = [
    'Void', 'Float', 'Double', 'Int', 'UInt', 'Short', 'UShort', 'Char',
    'UChar', 'Long', 'ULong', 'Rational', 'result_type',
    'AbstractExpression', 'Value', 'Variable', 'Parameter', 'Interval',
    'Reference', 'Condition', 'Case', 'Op', 'Reduce', 'Function', 'Image',
    'Reduction', 'Select', 'Cast', 'Max', 'Min', 'Stencil', 'TStencil',
    'Pow', 'Powf', 'Log', 'Exp', 'Sin', 'Cos', 'Sqrt', 'Sqrtf', 'Abs',
    'RandomFloat', 'InbuiltFunction',
]


def _lift(v):
    return Value.numericToValue(v)


# ---------------------------------------------------------------------------
# Math builtins (sandbox/constructs.py:77-211).  ``result`` is the type the
# reference's type system assigns; the CUDA emitter prints ``c_name`` and lets
# C++ overloading pick the precision from the argument types, as the
# reference's generated C++ does.
# ---------------------------------------------------------------------------
class Pow(InbuiltFunction):
    c_name = 'pow'
    result = Double

    def __init__(self, left, right):
        InbuiltFunction.__init__(self, left, right)


class Powf(InbuiltFunction):
    c_name = 'powf'
    result = Float

    def __init__(self, left, right):
        InbuiltFunction.__init__(self, left, right)


class Log(InbuiltFunction):
    c_name = 'log'
    result = Double

    def __init__(self, e):
        InbuiltFunction.__init__(self, e)


class Exp(InbuiltFunction):
    c_name = 'exp'
    result = Double

    def __init__(self, e):
        InbuiltFunction.__init__(self, e)


class Sin(InbuiltFunction):
    c_name = 'sin'
    result = Double

    def __init__(self, e):
        InbuiltFunction.__init__(self, e)


class Cos(InbuiltFunction):
    c_name = 'cos'
    result = Double

    def __init__(self, e):
        InbuiltFunction.__init__(self, e)


class Sqrt(InbuiltFunction):
    c_name = 'sqrt'
    result = Double

    def __init__(self, e):
        InbuiltFunction.__init__(self, e)


class Sqrtf(InbuiltFunction):
    c_name = 'sqrtf'
    result = Float

    def __init__(self, e):
        InbuiltFunction.__init__(self, e)


class Abs(InbuiltFunction):
    c_name = 'abs'
    result = None      # type of the argument

    def __init__(self, e):
        InbuiltFunction.__init__(self, e)


class RandomFloat(InbuiltFunction):
    """Uniform float in [0, 1).  The reference calls libc ``rand()``
    (sandbox/constructs.py:120-131); the CUDA backend rejects it because a
    data-parallel kernel has no equivalent of a sequential libc generator."""
    c_name = 'random_float'
    result = Float

    def __init__(self):
        InbuiltFunction.__init__(self)


# ---------------------------------------------------------------------------
class Cast(AbstractExpression):
    """C cast of an expression to a scalar type (sandbox/constructs.py:213)."""

    def __init__(self, typ, expr):
        expr = _lift(expr)
        assert typ in [Float, Double, UChar, Char, UShort, Short, UInt, Int,
                       ULong, Long]
        assert isinstance(expr, AbstractExpression)
        self._typ = typ
        self._expr = expr

    @property
    def typ(self):
        return self._typ

    @property
    def expression(self):
        return self._expr

    def children(self):
        return [self._expr]

    def clone(self):
        return Cast(self._typ, self._expr.clone())

    def macro_expand(self):
        self._expr = self._expr.macro_expand()
        return self

    def __str__(self):
        return "(" + self._typ.c_decl() + ") (" + str(self._expr) + ")"


class Select(AbstractExpression):
    """``cond ? true_expr : false_expr`` (sandbox/constructs.py:256).
    Both arms must have the same type when ``typeCheck`` is on."""

    def __init__(self, cond, true_expr, false_expr, typeCheck=True):
        assert isinstance(cond, Condition)
        true_expr = _lift(true_expr)
        false_expr = _lift(false_expr)
        assert isinstance(true_expr, AbstractExpression)
        assert isinstance(false_expr, AbstractExpression)
        if typeCheck:
            from .expression import getType
            tt = getType(true_expr)
            ft = getType(false_expr)
            assert tt == ft, str(true_expr) + " == " + str(false_expr)
        self._cond = cond
        self._true_expr = true_expr
        self._false_expr = false_expr

    @property
    def condition(self):
        return self._cond

    @property
    def true_expression(self):
        return self._true_expr

    @property
    def false_expression(self):
        return self._false_expr

    def children(self):
        return [self._cond, self._true_expr, self._false_expr]

    def clone(self):
        return Select(self._cond.clone(), self._true_expr.clone(),
                      self._false_expr.clone(), typeCheck=False)

    def macro_expand(self):
        self._true_expr = self._true_expr.macro_expand()
        self._false_expr = self._false_expr.macro_expand()
        return self

    def __str__(self):
        return "(" + str(self._cond) + "? " + str(self._true_expr) + ": " + \
            str(self._false_expr) + ")"


class Max(Select):
    def __init__(self, left, right, typeCheck=True):
        Select.__init__(self, Condition(left, '>', right), left, right,
                        typeCheck)


class Min(Select):
    def __init__(self, left, right, typeCheck=True):
        Select.__init__(self, Condition(left, '<', right), left, right,
                        typeCheck)


# ---------------------------------------------------------------------------
class Variable(AbstractExpression):
    def __init__(self, typ, name):
        self._typ = typ
        self._name = name

    @property
    def name(self):
        return self._name

    @property
    def typ(self):
        return self._typ

    def clone(self):
        return self

    def __str__(self):
        return str(self._name)


class Parameter(Variable):
    """A scalar run-time argument of the compiled pipeline."""
    pass


class Interval(object):
    """Closed integer interval ``[lb, ub]``."""

    def __init__(self, typ, lb, ub):
        lb = _lift(lb)
        ub = _lift(ub)
        assert isinstance(lb, AbstractExpression)
        assert isinstance(ub, AbstractExpression)
        self._typ = typ
        self._lb = lb
        self._ub = ub

    @property
    def lowerBound(self):
        return self._lb

    @property
    def upperBound(self):
        return self._ub

    @property
    def typ(self):
        return self._typ

    def collect(self, objType):
        if type(self) is objType:
            return [self]
        out = self._lb.collect(objType)
        for o in self._ub.collect(objType):
            if all(o is not p for p in out):
                out.append(o)
        return out

    def clone(self):
        return Interval(self._typ, self._lb.clone(), self._ub.clone())

    def __str__(self):
        return '(' + str(self._lb) + ', ' + str(self._ub) + ')'


class Reference(AbstractExpression):
    """``f(args...)``: the value of function/image ``f`` at a point."""

    def __init__(self, obj, args):
        args = [_lift(a) for a in args]
        for a in args:
            assert isinstance(a, AbstractExpression)
        self._obj = obj
        self._args = args

    @property
    def objectRef(self):
        return self._obj

    def _replace_ref_object(self, obj):
        self._obj = obj

    @property
    def arguments(self):
        return self._args

    def children(self):
        return list(self._args)

    def clone(self):
        return Reference(self._obj, [a.clone() for a in self._args])

    def macro_expand(self):
        self._args = [a.macro_expand() for a in self._args]
        return self

    def __str__(self):
        return self._obj.name + "(" + ", ".join(str(a) for a in self._args) \
            + ")"


# ---------------------------------------------------------------------------
class Condition(object):
    """Comparison (``<, <=, >, >=, ==, !=``) of two expressions, or a
    conjunction/disjunction (``&&``/``||``, built with ``&``/``|``) of two
    conditions (sandbox/constructs.py:722-804)."""

    _CMP = ('<', '<=', '>', '>=', '==', '!=')

    def __init__(self, left, cond, right):
        left = _lift(left)
        right = _lift(right)
        assert cond in ['<', '<=', '>', '>=', '==', '!=', '&&', '||']
        if cond in self._CMP:
            assert isinstance(left, AbstractExpression)
            assert isinstance(right, AbstractExpression)
        else:
            assert isinstance(left, Condition)
            assert isinstance(right, Condition)
        self._left = left
        self._right = right
        self._cond = cond

    @property
    def lhs(self):
        return self._left

    @property
    def rhs(self):
        return self._right

    @property
    def conditional(self):
        return self._cond

    def children(self):
        return [self._left, self._right]

    def clone(self):
        return Condition(self._left.clone(), self._cond, self._right.clone())

    def collect(self, objType):
        if type(self) is objType:
            return [self]
        found = []
        for side in (self._left, self._right):
            for o in side.collect(objType):
                if all(o is not p for p in found):
                    found.append(o)
        return found

    def has(self, objType):
        return len(self.collect(objType)) > 0

    def split_to_conjuncts(self):
        """Disjunctive normal form as a list of lists of comparisons;
        ``!=`` becomes ``<`` or ``>`` (sandbox/constructs.py:767-786)."""
        if self._cond in ('<', '<=', '>', '>=', '=='):
            return [[self]]
        if self._cond == '!=':
            return [[Condition(self._left, '<', self._right)],
                    [Condition(self._left, '>', self._right)]]
        if self._cond == '||':
            return self._left.split_to_conjuncts() + \
                self._right.split_to_conjuncts()
        if self._cond == '&&':
            out = []
            for lc in self._left.split_to_conjuncts():
                for rc in self._right.split_to_conjuncts():
                    out.append(lc + rc)
            return out
        raise AssertionError(self._cond)

    def __and__(self, other):
        assert isinstance(other, Condition)
        return Condition(self, '&&', other)

    def __or__(self, other):
        assert isinstance(other, Condition)
        return Condition(self, '||', other)

    def __str__(self):
        return "(" + str(self._left) + " " + self._cond + " " + \
            str(self._right) + ")"


class Case(object):
    """One piece of a piecewise definition: ``expression`` where
    ``condition`` holds.  Stencils in the expression are macro-expanded at
    construction (sandbox/constructs.py:806-823)."""

    def __init__(self, cond, expr):
        expr = _lift(expr)
        assert isinstance(cond, Condition)
        assert isinstance(expr, (AbstractExpression, Reduce))
        self._cond = cond
        if isinstance(expr, AbstractExpression):
            self._expr = expr.macro_expand()
        else:
            self._expr = expr

    @property
    def condition(self):
        return self._cond

    @property
    def expression(self):
        return self._expr

    def collect(self, objType):
        if type(self) is objType:
            return [self]
        found = self._cond.collect(objType)
        for o in self._expr.collect(objType):
            if all(o is not p for p in found):
                found.append(o)
        return found

    def clone(self):
        return Case(self._cond.clone(), self._expr.clone())

    def __str__(self):
        return 'Case(' + str(self._cond) + '){ ' + str(self._expr) + ' }'


class Op(object):
    Sum = 0
    Mul = 1
    Min = 2
    Max = 3


class Reduce(object):
    """Accumulate ``expr`` into the reduction cell ``red_ref`` with
    ``op_typ`` (sandbox/constructs.py:848-906)."""

    def __init__(self, red_ref, expr, op_typ):
        assert isinstance(red_ref, Reference)
        assert isinstance(red_ref.objectRef, Reduction)
        expr = _lift(expr)
        assert isinstance(expr, AbstractExpression)
        assert op_typ in [Op.Sum, Op.Mul, Op.Min, Op.Max]
        self._red_ref = red_ref
        self._expr = expr
        self._op_typ = op_typ

    @property
    def accumulate_ref(self):
        return self._red_ref

    @property
    def expression(self):
        return self._expr

    @property
    def op_type(self):
        # The reference returns the expression here (a slip at
        # sandbox/constructs.py:866-868); the operator is what callers need.
        return self._op_typ

    def collect(self, objType):
        if type(self) is objType:
            return [self]
        found = self._red_ref.collect(objType)
        for o in self._expr.collect(objType):
            if all(o is not p for p in found):
                found.append(o)
        return found

    def clone(self):
        return Reduce(self._red_ref.clone(), self._expr.clone(), self._op_typ)

    def __str__(self):
        op_str, sep = {Op.Sum: ('', ' + '), Op.Mul: ('', ' * '),
                       Op.Min: ('Min', ', '), Op.Max: ('Max', ', ')}[
                           self._op_typ]
        r = str(self._red_ref)
        return 'Reduce [ ' + r + ' = ' + op_str + '(' + r + sep + \
            str(self._expr) + ') ]'


# ---------------------------------------------------------------------------
class Function(object):
    """A stage: a scalar-valued function over a box of integer points,
    defined piecewise by ``Case``s or by one expression
    (sandbox/constructs.py:907-1064).  ``Function(..., "const")`` marks a
    standalone constant function (a table that depends only on parameters
    and small inputs)."""

    def __init__(self, varDom, typ, name, const=""):
        self._name = name
        self._typ = typ
        self._const = (const == "const")
        assert len(varDom[0]) == len(varDom[1])
        for v, d in zip(varDom[0], varDom[1]):
            assert isinstance(v, Variable)
            assert isinstance(d, Interval)
            assert v.typ == d.typ
        self._variables = list(varDom[0])
        self._varDomain = list(varDom[1])
        self._ndims = len(self._variables)
        self._body = []

    @property
    def name(self):
        return self._name

    @property
    def typ(self):
        return self._typ

    @property
    def is_const_func(self):
        return self._const

    @property
    def variableDomain(self):
        return (self._variables, self._varDomain)

    @property
    def domain(self):
        return self._varDomain

    @property
    def variables(self):
        return self._variables

    @property
    def ndims(self):
        return self._ndims

    @property
    def is_reduction(self):
        return False

    @property
    def defn(self):
        return self._body

    @defn.setter
    def defn(self, parts):
        assert self._body == []
        assert len(parts) > 0, str(parts) + " " + str(self._name)
        n_case = 0
        n_expr = 0
        for p in parts:
            p = _lift(p)
            assert isinstance(p, (Case, AbstractExpression)), str(p)
            if isinstance(p, Case):
                n_case += 1
            else:
                n_expr += 1
                p = p.macro_expand()
            # either one plain expression, or only Cases
            assert n_expr <= 1
            assert n_case * n_expr == 0
            self._body.append(p)

    def __call__(self, *args):
        assert len(args) == len(self._variables), \
            "%s takes %d arguments" % (self._name, len(self._variables))
        return Reference(self, list(args))

    def getObjects(self, objType):
        found = []
        for p in self._body:
            for o in p.collect(objType):
                if all(o is not q for q in found):
                    found.append(o)
        for d in self._varDomain:
            for o in d.collect(objType):
                if all(o is not q for q in found):
                    found.append(o)
        return found

    def hasBoundedIntegerDomain(self):
        from .expression import isAffine
        return all(isAffine(d.lowerBound) and isAffine(d.upperBound)
                   for d in self._varDomain)

    def clone(self):
        f = Function(([v for v in self._variables],
                      [d.clone() for d in self._varDomain]),
                     self._typ, self._name, "const" if self._const else "")
        f.defn = [c.clone() for c in self._body]
        return f

    def __str__(self):
        if not self._body:
            return self._name
        var_str = ", ".join(str(v) for v in self._variables)
        dom_str = ', '.join(str(v) + str(d) for v, d in
                            zip(self._variables, self._varDomain))
        case_str = "{ " + "\n ".join(str(c) for c in self._body) + " }"
        return "Domain: " + dom_str + '\n' + self._name + "(" + var_str + \
            ") = " + case_str + '\n'


class Image(Function):
    """A pipeline input: a dense row-major array with the given dimensions
    (sandbox/constructs.py:1066-1090).  Dimension ``i`` spans
    ``[0, dims[i]-1]``."""

    def __init__(self, typ, name, dims):
        dims = [_lift(d) for d in dims]
        for d in dims:
            assert isinstance(d, AbstractExpression)
        self._dims = dims
        intervals = [Interval(UInt, 0, d - 1) for d in dims]
        variables = [Variable(UInt, "_" + name + str(i))
                     for i in range(len(dims))]
        Function.__init__(self, (variables, intervals), typ, name)

    @property
    def dimensions(self):
        return tuple(self._dims)

    def __str__(self):
        return str(self._name) + "(" + ", ".join(str(d) for d in self._dims) \
            + ")"


class Reduction(Function):
    """A function whose cells accumulate contributions from every point of a
    separate reduction domain (sandbox/constructs.py:1092-1215).  Cells start
    at ``default`` (zero of the element type unless set)."""

    def __init__(self, varDom, redDom, typ, name):
        Function.__init__(self, varDom, typ, name)
        assert len(redDom[0]) == len(redDom[1])
        for v, d in zip(redDom[0], redDom[1]):
            assert isinstance(v, Variable)
            assert isinstance(d, Interval)
            assert v.typ == d.typ
        self._redVariables = list(redDom[0])
        self._redDomain = list(redDom[1])
        self._default = Value(0, typ)

    @property
    def is_reduction(self):
        return True

    @property
    def default(self):
        return self._default

    @default.setter
    def default(self, expr):
        expr = _lift(expr)
        assert isinstance(expr, AbstractExpression)
        self._default = expr

    @property
    def reductionDomain(self):
        return self._redDomain

    @property
    def reductionVariables(self):
        return self._redVariables

    @property
    def defn(self):
        return self._body

    @defn.setter
    def defn(self, parts):
        assert self._body == []
        for p in parts:
            p = _lift(p)
            assert isinstance(p, (Case, Reduce)), str(p)
            self._body.append(p)

    def getObjects(self, objType):
        found = Function.getObjects(self, objType)
        extra = []
        for d in self._redDomain:
            extra += d.collect(objType)
        extra += self._default.collect(objType)
        for o in extra:
            if all(o is not q for q in found):
                found.append(o)
        return found

    def clone(self):
        r = Reduction(([v for v in self._variables],
                       [d.clone() for d in self._varDomain]),
                      ([v for v in self._redVariables],
                       [d.clone() for d in self._redDomain]),
                      self._typ, self._name)
        r.defn = [c.clone() for c in self._body]
        r.default = self._default.clone()
        return r

    def __str__(self):
        if not self._body:
            return self._name
        var_str = ", ".join(str(v) for v in self._variables)
        dom_str = ', '.join(str(v) + str(d) for v, d in
                            zip(self._variables, self._varDomain))
        red_str = ', '.join(str(v) + str(d) for v, d in
                            zip(self._redVariables, self._redDomain))
        case_str = "{ " + "\n ".join(str(c) for c in self._body) + " }"
        return "Domain: " + dom_str + '\n' + "Reduction Domain: " + \
            red_str + '\n' + self._name + "(" + var_str + ") = " + \
            case_str + '\n' + "Default: " + str(self._default)


# ---------------------------------------------------------------------------
# Stencils (sandbox/constructs.py:415-720)
# ---------------------------------------------------------------------------
def _inner_dims(lst):
    if isinstance(lst, list):
        return [len(x) if isinstance(x, list) else 0 for x in lst]
    return 0


def is_valid_kernel(kernel, num_dimensions):
    """True when ``kernel`` is a rectangular nested list with exactly
    ``num_dimensions`` levels; raises AssertionError otherwise."""
    def rec(k, n, chain):
        inner = _inner_dims(k)
        assert not inner or inner.count(inner[0]) == len(inner), (
            "kernel does not have equal dimensions.\nErroring dimensions: "
            "%s\nKernel: %s" % (inner, k))
        if isinstance(k, list):
            for sub in k:
                assert rec(sub, n - 1, [k] + chain)
            return True
        if n < 0:
            msg = "kernel has more dimensions than expected"
        elif n > 0:
            msg = "Kernel has less dimensions than expected"
        else:
            return True
        raise AssertionError("%s\nExpected Dimensions: %s\nIncorrect "
                             "Kernel: %s\n" % (msg, num_dimensions,
                                                " ->\n\t".join(map(str,
                                                                   chain))))
    return rec(kernel, num_dimensions, [])


def get_valid_kernel_sizes(kernel):
    sizes = []
    k = kernel
    while isinstance(k, list):
        if len(k) == 0:
            sizes.append(0)
            break
        sizes.append(len(k))
        k = k[0]
    return sizes


class Stencil(AbstractExpression):
    """Weighted neighbourhood sum of ``input_fn`` around the iteration
    variables.  ``origin`` defaults to ``(size-1)//2`` per dimension.
    ``macro_expand`` produces ``sum(input(v + i - origin) * w)`` with zero
    weights dropped and unit weights unmultiplied, in row-major kernel
    order (sandbox/constructs.py:544-687)."""

    def __init__(self, input_fn, iteration_vars, kernel, origin=None,
                 _origin=None):
        if origin is None:
            origin = _origin
        if not isinstance(input_fn, Function):
            raise TypeError("Expected %s to be of type Function" % input_fn)
        for v in iteration_vars:
            if not isinstance(v, Variable):
                raise TypeError("Expected %s to be of type Variable" % v)
        assert is_valid_kernel(kernel, len(iteration_vars))
        self._input_fn = input_fn
        self._iteration_vars = list(iteration_vars)
        self._kernel = kernel
        self._sizes = get_valid_kernel_sizes(kernel)
        self._origin = origin
        if self._origin is None:
            self._origin = [(s - 1) // 2 for s in self._sizes]

    @property
    def input_func(self):
        return self._input_fn

    @property
    def iter_vars(self):
        return self._iteration_vars

    @property
    def kernel(self):
        return self._kernel

    @property
    def sizes(self):
        return self._sizes

    @property
    def origin(self):
        return self._origin

    def _indexed_kernel(self):
        out = []

        def rec(prefix, dim, sub):
            for i in range(self._sizes[dim]):
                idx = self._iteration_vars[dim] + (i - self._origin[dim])
                if dim == len(self._sizes) - 1:
                    out.append((prefix + [idx], sub[i]))
                else:
                    rec(prefix + [idx], dim + 1, sub[i])
        rec([], 0, self._kernel)
        return out

    def macro_expand(self):
        total = 0
        for idx, w in self._indexed_kernel():
            total = total + Reference(self._input_fn, idx) * w
        return 1 * total

    def __str__(self):
        return ("Stencil object\n%s\n\tinput: %s\n\titeration vars: %s"
                "\n\tdimension sizes: %s\n\torigin: %s\n\tkernel: %s" % (
                    str(Stencil.macro_expand(self)), self._input_fn,
                    [str(v) for v in self._iteration_vars], self._sizes,
                    self._origin, self._kernel))


class TStencil(object):
    """Time-iterated stencil declaration (sandbox/constructs.py:689-720).
    Like the reference, it is a declaration only: it is not a ``Function``
    and pipelines do not accept it."""

    def __init__(self, var_domain, kernel, name, origin=None, timesteps=1):
        self.name = name
        self.var_domain = var_domain
        self.timesteps = int(timesteps)
        assert is_valid_kernel(kernel, len(var_domain))
        self.size = get_valid_kernel_sizes(kernel)
        self.kernel = kernel
        self.origin = origin
        if origin is None:
            self.origin = [int(math.floor(s / 2)) for s in self.size]

    def getObjects(self, objType):
        found = []
        for d in self.var_domain:
            found += d.collect(objType)
        return found
