"""Scalar types of the PolyMage language and their promotion rules.

The type classes and the promotion order follow the reference language
(sandbox/expr_types.py:25-104): a binary operation takes the "wider" of its
operand types, doubles first, then floats, then the integer types from the
widest down.  Each type also knows its C spelling (used by the CUDA code
generator), its numpy dtype (used by the host bindings and the oracle) and its
size in bytes (used by storage mapping and shared-memory planning).
"""

import numpy as np


class _ScalarType(object):
    """Base of all scalar type tags.  Types are used as classes, never
    instantiated, exactly as in the reference language."""
    _c_name = None
    _np = None
    _short = None

    @classmethod
    def c_type_name(cls):
        """numpy-style short name ('int32', 'float32', ...), as the reference's
        ``c_type_name`` returns (sandbox/expr_types.py:27-80)."""
        return cls._short

    @classmethod
    def c_decl(cls):
        """C/CUDA spelling of the type."""
        return cls._c_name

    @classmethod
    def np_dtype(cls):
        return np.dtype(cls._np) if cls._np is not None else None

    @classmethod
    def size(cls):
        return np.dtype(cls._np).itemsize

    @classmethod
    def is_float(cls):
        return cls in (Float, Double)

    @classmethod
    def is_integer(cls):
        return cls in (Char, UChar, Short, UShort, Int, UInt, Long, ULong)


class Void(_ScalarType):
    _c_name = 'void'
    _short = 'void'


class Float(_ScalarType):
    _c_name = 'float'
    _np = np.float32
    _short = 'float32'


class Double(_ScalarType):
    _c_name = 'double'
    _np = np.float64
    _short = 'float64'


class Int(_ScalarType):
    _c_name = 'int'
    _np = np.int32
    _short = 'int32'


class UInt(_ScalarType):
    _c_name = 'unsigned int'
    _np = np.uint32
    _short = 'uint32'


class Short(_ScalarType):
    _c_name = 'short'
    _np = np.int16
    _short = 'int16'


class UShort(_ScalarType):
    _c_name = 'unsigned short'
    _np = np.uint16
    _short = 'uint16'


class Char(_ScalarType):
    _c_name = 'signed char'
    _np = np.int8
    _short = 'int8'


class UChar(_ScalarType):
    _c_name = 'unsigned char'
    _np = np.uint8
    _short = 'uint8'


class Long(_ScalarType):
    _c_name = 'long long'
    _np = np.int64
    _short = 'int64'


class ULong(_ScalarType):
    _c_name = 'unsigned long long'
    _np = np.uint64
    _short = 'uint64'


class Rational(_ScalarType):
    """Exact fractions appearing in affine analysis (e.g. ``x/2``)."""
    _c_name = None
    _short = 'rational'


ALL_TYPES = (Float, Double, Int, UInt, Short, UShort, Char, UChar, Long, ULong)

# Widest first: the promotion order of sandbox/expr_types.py:83-104.
_PROMOTION = (Double, Float, ULong, Long, UInt, Int, UShort, Short, UChar)


def result_type(a, b):
    """Type of a binary operation between operands of types ``a`` and ``b``.

    Mirrors sandbox/expr_types.py:83-104, including its TypeError when no rule
    applies (e.g. Char with a non-Char operand other than the listed ones)."""
    for t in _PROMOTION:
        if a is t or b is t:
            return t
    if a is Char and b is Char:
        return Char
    raise TypeError((a, b))
