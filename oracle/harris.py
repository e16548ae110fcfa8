"""FP64 restatement of the reference's Harris spec
(sandbox/apps/python/img_proc/harris/polymage_harris.py:13-78) --
test infrastructure only.

``img`` is [R+2][C+2]; the output has the same shape and is defined on
[2, R-1] x [2, C-1] (``condRed``, :30-31); other points are left as the
caller's buffer had them (the reference writes only the Case domain).
"""

import numpy as np


def harris(img, out=None):
    """img: float array [R+2][C+2]; returns float64 [R+2][C+2] with the
    border (outside [2,R-1]x[2,C-1]) taken from ``out`` (zeros if None)."""
    img = np.asarray(img, dtype=np.float64)
    H, W = img.shape
    R, C = H - 2, W - 2
    res = np.zeros((H, W)) if out is None else np.array(out, np.float64)
    if R < 3 or C < 3:
        return res
    i = img
    # Iy, Ix on x in [1, R], y in [1, C]  (:33-42)
    def s(dx, dy):
        return i[1 + dx:R + 1 + dx, 1 + dy:C + 1 + dy]
    Iy = (s(-1, -1) * (-1.0 / 12) + s(-1, 1) * (1.0 / 12) +
          s(0, -1) * (-2.0 / 12) + s(0, 1) * (2.0 / 12) +
          s(1, -1) * (-1.0 / 12) + s(1, 1) * (1.0 / 12))
    Ix = (s(-1, -1) * (-1.0 / 12) + s(1, -1) * (1.0 / 12) +
          s(-1, 0) * (-2.0 / 12) + s(1, 0) * (2.0 / 12) +
          s(-1, 1) * (-1.0 / 12) + s(1, 1) * (1.0 / 12))
    # products (:44-51); index [k][l] <-> (x, y) = (k+1, l+1)
    Ixx, Iyy, Ixy = Ix * Ix, Iy * Iy, Ix * Iy

    def box(a):
        # 3x3 sums at x in [2, R-1], y in [2, C-1]  (:53-66)
        o = np.zeros((R - 2, C - 2))
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                o += a[1 + dx:R - 1 + dx, 1 + dy:C - 1 + dy]
        return o
    Sxx, Syy, Sxy = box(Ixx), box(Iyy), box(Ixy)
    det = Sxx * Syy - Sxy * Sxy               # (:68-69)
    trace = Sxx + Syy                         # (:71-72)
    res[2:R, 2:C] = det - 0.04 * trace * trace   # (:74-76)
    return res


def make_input(rows, cols, seed=0):
    """The synthetic workload: a rows x cols float32 image, U[0,1)."""
    rng = np.random.default_rng(seed)
    return rng.random((rows, cols), dtype=np.float32)
