"""ctypes wrappers around the reference's own generated C++, compiled from
the reference tree into oracle/_ref by oracle/Makefile -- test
infrastructure only (parity pinning and the CPU baseline).

* ``ref_harris``: ``void refHarris(int C, int R, float* img, float*& out)``
  (sandbox/ipp_bench/harris/harris_function.cpp:9-64): the apps/python
  Harris spec on float input; it mallocs and zero-fills its output.
* ``ref_unsharp``: ``pipeline_mask(int C, int R, float threshold,
  float weight, void* uint8 [R+4][C+4][3], void* float [R][C][3])``
  (sandbox/video_demo/unsharp_polymage.cpp:10-99): unsharp mask over the
  whole image (no Case), interleaved uint8 input scaled by 1/255.
* ``ref_laplacian``: ``pipeline_laplacian(int C, int R, float alpha,
  float beta, void* uint8 [R-92][C-92][3], void* uint8 [R-92][C-92][3])``
  (sandbox/video_demo/laplacian_polymage.cpp:10-1062): the local
  Laplacian filter of the video demo, frame padded internally.
"""

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_libs = {}


def available(name):
    return os.path.exists(os.path.join(REF_DIR, "libref_%s.so" % name))


def _lib(name):
    if name not in _libs:
        path = os.path.join(REF_DIR, "libref_%s.so" % name)
        if not os.path.exists(path):
            raise FileNotFoundError(
                "%s not built (run: make -C oracle)" % path)
        lib = ctypes.CDLL(path)
        if hasattr(lib, "pool_init"):
            lib.pool_init()
        _libs[name] = lib
    return _libs[name]


_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]


def ref_harris(img):
    """img: float32 [R+2][C+2] C-contiguous -> float32 [R+2][C+2]."""
    img = np.ascontiguousarray(img, dtype=np.float32)
    H, W = img.shape
    lib = _lib("harris")
    fn = lib._Z9refHarrisiiPfRS_
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                   ctypes.POINTER(ctypes.c_void_p)]
    fn.restype = None
    out = ctypes.c_void_p()
    fn(W - 2, H - 2, img.ctypes.data, ctypes.byref(out))
    res = np.ctypeslib.as_array(ctypes.cast(out, ctypes.POINTER(
        ctypes.c_float)), shape=(H, W)).copy()
    _libc.free(out)
    return res


def ref_unsharp(img_u8, threshold, weight, out=None):
    """img_u8: uint8 [R+4][C+4][3] -> float32 [R][C][3]."""
    img_u8 = np.ascontiguousarray(img_u8, dtype=np.uint8)
    H, W, _ = img_u8.shape
    R, C = H - 4, W - 4
    if out is None:
        out = np.zeros((R, C, 3), np.float32)
    lib = _lib("unsharp")
    fn = lib.pipeline_mask
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                   ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = None
    fn(C, R, float(threshold), float(weight), img_u8.ctypes.data,
       out.ctypes.data)
    return out


def ref_laplacian(frame_u8, alpha, beta, out=None):
    """frame_u8: uint8 [rows][cols][3] -> uint8 [rows][cols][3]."""
    frame_u8 = np.ascontiguousarray(frame_u8, dtype=np.uint8)
    H, W, _ = frame_u8.shape
    if out is None:
        out = np.zeros((H, W, 3), np.uint8)
    lib = _lib("laplacian")
    fn = lib.pipeline_laplacian
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                   ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = None
    fn(W + 92, H + 92, float(alpha), float(beta), frame_u8.ctypes.data,
       out.ctypes.data)
    return out


def planar_from_u8(img_u8):
    """The float planar [3][R+4][C+4] image pipeline_mask computes on."""
    return np.ascontiguousarray(np.moveaxis(
        img_u8.astype(np.float32) / np.float32(255.0), 2, 0))
