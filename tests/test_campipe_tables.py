"""The camera pipe's const tables (colour matrix, tone-curve LUT) computed
by the product's host code are bit-identical to the oracle's C restatement
(no GPU: the tables are tabulated on the host)."""

import ctypes

import numpy as np
import pytest

import oracle.campipe as OC
from polymage_b200.apps.campipe import build_campipe


@pytest.fixture(scope="module")
def lib():
    cp = build_campipe().build()
    return cp


def _call(cp, fname, params, reads, out):
    meta = cp.module.meta['const'][fname]
    fn = getattr(cp.lib, meta['symbol'])
    args = []
    types = []
    for p in cp.params:
        if p.name in ('C', 'R'):
            args.append(int(params[p.name]))
            types.append(ctypes.c_int)
        else:
            args.append(float(params[p.name]))
            types.append(ctypes.c_float)
    for r in meta['reads']:
        args.append(reads[r].ctypes.data)
        types.append(ctypes.c_void_p)
    args.append(out.ctypes.data)
    types.append(ctypes.c_void_p)
    fn.argtypes = types
    fn.restype = None
    fn(*args)


@pytest.mark.parametrize("kelvin,contrast,gamma", [
    (3700.0, 50.0, 2.0), (3200.0, 0.0, 1.0), (6500.0, 80.0, 2.4),
    (2500.0, 25.0, 1.8)])
def test_tables_bit_identical(lib, kelvin, contrast, gamma):
    prm = {'C': 2592, 'R': 1968, 'colour_temp': kelvin,
           'contrast': contrast, 'gamma': gamma}
    reads = {'matrix_3200': OC.MATRIX_3200, 'matrix_7000': OC.MATRIX_7000}
    mat = np.zeros((3, 4), np.int32)
    _call(lib, 'matrix', prm, reads, mat)
    lut = np.zeros(65536, np.uint8)
    _call(lib, 'curveLUT', prm, reads, lut)
    omat, olut = OC.tables(kelvin, contrast, gamma)
    assert np.array_equal(mat, omat)
    assert np.array_equal(lut, olut)
    # the LUT saturates outside [0, 1024): a 1024-entry table with
    # clamping is equivalent
    assert np.all(lut[:32768] == lut[32768])
    assert np.all(lut[32768 + 1024:] == lut[32768 + 1024])
