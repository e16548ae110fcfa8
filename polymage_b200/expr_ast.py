"""Expression trees of the PolyMage language.

Operator overloading on expressions builds the tree, with the same small
algebraic shortcuts the reference applies while building
(sandbox/expr_ast.py:31-160): adding or subtracting literal 0 and multiplying
or dividing by literal 1 return the other operand, multiplying by literal 0
returns ``Value(0, Int)``, and ``0 - e`` is a unary minus.  Both ``/`` and
``//`` build a ``Div`` node, which has C semantics (truncating for integers).
Python ``int`` literals become ``Int`` values, ``float`` literals ``Float``
values and ``Fraction`` literals ``Rational`` values
(sandbox/expr_ast.py:193-203).

``str()`` of an expression prints the same text the reference prints (the
ported stencil macro-expansion tests compare these strings).
"""

from fractions import Fraction

from .expr_types import Int, Float, Rational


def _lift(v):
    return Value.numericToValue(v)


class AbstractExpression(object):
    """Base of every expression node."""

    # ---- arithmetic -----------------------------------------------------
    def __add__(self, other):
        other = _check(other)
        if isinstance(other, Value) and other.value == 0:
            return self
        return Add(self, other)

    def __radd__(self, other):
        other = _check(other)
        if isinstance(other, Value) and other.value == 0:
            return self
        return Add(other, self)

    def __sub__(self, other):
        other = _check(other)
        if isinstance(other, Value) and other.value == 0:
            return self
        return Sub(self, other)

    def __rsub__(self, other):
        other = _check(other)
        if isinstance(other, Value) and other.value == 0:
            return UnaryMinus(self)
        return Sub(other, self)

    def __mul__(self, other):
        other = _check(other)
        if isinstance(other, Value):
            if other.value == 1:
                return self
            if other.value == 0:
                return Value(0, Int)
        return Mul(self, other)

    def __rmul__(self, other):
        other = _check(other)
        if isinstance(other, Value):
            if other.value == 1:
                return self
            if other.value == 0:
                return Value(0, Int)
        return Mul(other, self)

    def __truediv__(self, other):
        other = _check(other)
        if isinstance(other, Value) and other.value == 1:
            return self
        return Div(self, other)

    def __rtruediv__(self, other):
        return Div(_check(other), self)

    __floordiv__ = __truediv__
    __rfloordiv__ = __rtruediv__

    def __mod__(self, other):
        return Mod(self, _check(other))

    def __rmod__(self, other):
        return Mod(_check(other), self)

    def __lshift__(self, other):
        other = _check(other)
        if isinstance(other, Value) and other.value == 0:
            return self
        return LShift(self, other)

    def __rlshift__(self, other):
        return LShift(_check(other), self)

    def __rshift__(self, other):
        other = _check(other)
        if isinstance(other, Value) and other.value == 0:
            return self
        return RShift(self, other)

    def __rrshift__(self, other):
        return RShift(_check(other), self)

    def __and__(self, other):
        return LAnd(self, _check(other))

    def __rand__(self, other):
        return LAnd(_check(other), self)

    def __or__(self, other):
        return LOr(self, _check(other))

    def __ror__(self, other):
        return LOr(_check(other), self)

    def __xor__(self, other):
        return Xor(self, _check(other))

    def __rxor__(self, other):
        return Xor(_check(other), self)

    def __neg__(self):
        return UnaryMinus(self)

    def __pos__(self):
        return UnaryPlus(self)

    # ---- tree utilities --------------------------------------------------
    def children(self):
        return []

    def collect(self, objType):
        """All distinct nodes of exactly type ``objType`` in this tree."""
        found = []
        seen = set()
        stack = [self]
        while stack:
            node = stack.pop()
            if type(node) is objType and id(node) not in seen:
                seen.add(id(node))
                found.append(node)
            stack.extend(node.children())
        return found

    def has(self, objType):
        return len(self.collect(objType)) > 0

    def macro_expand(self):
        return self

    __hash__ = object.__hash__


def _check(other):
    other = _lift(other)
    if not isinstance(other, AbstractExpression):
        raise TypeError("cannot combine an expression with %r" % (other,))
    return other


class Value(AbstractExpression):
    """A literal constant with an explicit type."""

    @classmethod
    def numericToValue(cls, v):
        if type(v) is int:
            return Value(v, Int)
        if type(v) is float:
            return Value(v, Float)
        if type(v) is Fraction:
            return Value(v, Rational)
        return v

    def __init__(self, value, typ):
        self._value = value
        self._typ = typ

    @property
    def value(self):
        return self._value

    @property
    def typ(self):
        return self._typ

    def clone(self):
        return Value(self._value, self._typ)

    def __eq__(self, other):
        if isinstance(other, Value):
            return self._value == other._value
        return self._value == other

    __hash__ = object.__hash__

    def __str__(self):
        return str(self._value)


class AbstractBinaryOpNode(AbstractExpression):
    def __init__(self, left, right, op=None):
        self._left = left
        self._right = right
        self._op = op

    @property
    def left(self):
        return self._left

    @property
    def right(self):
        return self._right

    @property
    def op(self):
        return self._op

    def children(self):
        return [self._left, self._right]

    def clone(self):
        cls = _BINOP_CLASS.get(self._op)
        if cls is None:
            return AbstractBinaryOpNode(self._left.clone(),
                                        self._right.clone(), self._op)
        return cls(self._left.clone(), self._right.clone())

    def macro_expand(self):
        self._left = self._left.macro_expand()
        self._right = self._right.macro_expand()
        return self

    def __str__(self):
        return "(" + str(self._left) + " " + self._op + " " + \
            str(self._right) + ")"


class Add(AbstractBinaryOpNode):
    def __init__(self, left, right):
        AbstractBinaryOpNode.__init__(self, left, right, '+')


class Sub(AbstractBinaryOpNode):
    def __init__(self, left, right):
        AbstractBinaryOpNode.__init__(self, left, right, '-')


class Mul(AbstractBinaryOpNode):
    def __init__(self, left, right):
        AbstractBinaryOpNode.__init__(self, left, right, '*')


class Div(AbstractBinaryOpNode):
    def __init__(self, left, right):
        AbstractBinaryOpNode.__init__(self, left, right, '/')


class Mod(AbstractBinaryOpNode):
    def __init__(self, left, right):
        AbstractBinaryOpNode.__init__(self, left, right, '%')


class LShift(AbstractBinaryOpNode):
    def __init__(self, left, right):
        AbstractBinaryOpNode.__init__(self, left, right, '<<')


class RShift(AbstractBinaryOpNode):
    def __init__(self, left, right):
        AbstractBinaryOpNode.__init__(self, left, right, '>>')


class LAnd(AbstractBinaryOpNode):
    """Bitwise and (the reference calls it LAnd and prints ``&``)."""
    def __init__(self, left, right):
        AbstractBinaryOpNode.__init__(self, left, right, '&')


class LOr(AbstractBinaryOpNode):
    def __init__(self, left, right):
        AbstractBinaryOpNode.__init__(self, left, right, '|')


class Xor(AbstractBinaryOpNode):
    def __init__(self, left, right):
        AbstractBinaryOpNode.__init__(self, left, right, '^')


_BINOP_CLASS = {'+': Add, '-': Sub, '*': Mul, '/': Div, '%': Mod,
                '<<': LShift, '>>': RShift, '&': LAnd, '|': LOr, '^': Xor}


def make_binop(op, left, right):
    """Build the node class for ``op`` without the building shortcuts."""
    return _BINOP_CLASS[op](left, right)


class AbstractUnaryOpNode(AbstractExpression):
    def __init__(self, child, op=None):
        self._child = child
        self._op = op

    @property
    def child(self):
        return self._child

    @property
    def op(self):
        return self._op

    def children(self):
        return [self._child]

    def clone(self):
        cls = UnaryMinus if self._op == '-' else UnaryPlus
        return cls(self._child.clone())

    def macro_expand(self):
        self._child = self._child.macro_expand()
        return self

    def __str__(self):
        return self._op + "(" + str(self._child) + ")"


class UnaryPlus(AbstractUnaryOpNode):
    def __init__(self, child):
        AbstractUnaryOpNode.__init__(self, child, '+')


class UnaryMinus(AbstractUnaryOpNode):
    def __init__(self, child):
        AbstractUnaryOpNode.__init__(self, child, '-')


class InbuiltFunction(AbstractExpression):
    """A call of a math builtin; subclasses live in ``constructs``."""
    c_name = None          # C/CUDA function name
    result = None          # result type tag (None: type of first argument)

    def __init__(self, *args):
        args = [_lift(a) for a in args]
        for a in args:
            if not isinstance(a, AbstractExpression):
                raise TypeError("builtin argument %r is not an expression"
                                % (a,))
        self._args = args

    @property
    def arguments(self):
        return self._args

    def children(self):
        return list(self._args)

    def getType(self):
        from .expression import getType
        if self.result is not None:
            return self.result
        return getType(self._args[0])

    def clone(self):
        return type(self)(*[a.clone() for a in self._args])

    def rebuild(self, args):
        return type(self)(*args)

    def __str__(self):
        return self.c_name + "(" + ", ".join(str(a) for a in self._args) + ")"
