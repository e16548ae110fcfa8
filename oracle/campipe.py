"""ctypes wrapper of the C restatement of the camera pipeline
(oracle/campipe.c, built by `make -C oracle restatements`) -- test
infrastructure only.  Spec: sandbox/apps/python/img_proc/campipe/
polymage_campipe.py:13-304; matrices from campipe/init.py:26-40."""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libcampipe.so")

MATRIX_3200 = np.array([[1.6697, -0.2693, -0.4004, -42.4346],
                        [-0.3576, 1.0615, 1.5949, -37.1158],
                        [-0.2175, -1.8751, 6.9640, -26.6970]], np.float32)
MATRIX_7000 = np.array([[2.2997, -0.4478, 0.1706, -39.0923],
                        [-0.3826, 1.5906, -0.2080, -25.4311],
                        [-0.0888, -0.7344, 2.2832, -20.0826]], np.float32)

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise FileNotFoundError("%s not built (make -C oracle "
                                    "restatements)" % LIB)
        _lib = ctypes.CDLL(LIB)
        _lib.campipe.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                 ctypes.c_float, ctypes.c_float] + \
            [ctypes.c_void_p] * 4
        _lib.campipe_tables.argtypes = [ctypes.c_float] * 3 + \
            [ctypes.c_void_p] * 4
    return _lib


def campipe(img, colour_temp=3700.0, contrast=50.0, gamma=2.0,
            m3200=MATRIX_3200, m7000=MATRIX_7000):
    """img: int16 [R][C] -> uint8 [3][R-48][C-64]."""
    img = np.ascontiguousarray(img, dtype=np.int16)
    R, C = img.shape
    out = np.zeros((3, R - 48, C - 64), np.uint8)
    m3 = np.ascontiguousarray(m3200, np.float32)
    m7 = np.ascontiguousarray(m7000, np.float32)
    lib().campipe(R, C, colour_temp, contrast, gamma, img.ctypes.data,
                  m3.ctypes.data, m7.ctypes.data, out.ctypes.data)
    return out


def tables(colour_temp=3700.0, contrast=50.0, gamma=2.0, m3200=MATRIX_3200,
           m7000=MATRIX_7000):
    """(matrix int32 [3][4], curve LUT uint8 [65536] indexed v + 32768)."""
    mat = np.zeros((3, 4), np.int32)
    lut = np.zeros(65536, np.uint8)
    m3 = np.ascontiguousarray(m3200, np.float32)
    m7 = np.ascontiguousarray(m7000, np.float32)
    lib().campipe_tables(colour_temp, contrast, gamma, m3.ctypes.data,
                         m7.ctypes.data, mat.ctypes.data, lut.ctypes.data)
    return mat, lut


def make_input(R=1968, C=2592, seed=0):
    """Synthetic raw: int16 values U{0..1023} (a 10-bit GRBG Bayer)."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, 1024, (R, C), dtype=np.int16)
