"""FP64 restatement of the reference's unsharp-mask spec
(sandbox/apps/python/img_proc/unsharp_mask/polymage_unsharp_mask.py:16-77)
-- test infrastructure only.

Points a stage's ``Case`` does not cover read as 0 (the convention of this
backend; the reference leaves them uninitialized).  Consequences
(:44-74): blurx exists only for y in [1, C], so output columns whose blury
taps reach y = 0 or y > C (y = 2, C-1, C in domain coordinates) depend on
the convention; row R+1 and column C+1 of the domain are never written.
``defined_region`` gives the output box that does not depend on it.
"""

import numpy as np


def unsharp(img, threshold, weight, out=None):
    """img: [3][R+4][C+4]; returns float64 [3][R][C] (domain x in [2,R+1],
    y in [2,C+1] mapped to [0,R) x [0,C)); unwritten points keep ``out``."""
    img = np.asarray(img, dtype=np.float64)
    _, H, W = img.shape
    R, C = H - 4, W - 4
    res = np.zeros((3, R, C)) if out is None else np.array(out, np.float64)
    if R < 1 or C < 1:
        return res
    # blurx on x in [2, R], y in [1, C] (:50-55), domain y in [0, C+3]
    bx = np.zeros((3, R + 2, C + 4))     # index [c][x][y]
    xs = slice(2, R + 1)
    ys = slice(1, C + 1)

    def im(dx):
        return img[:, 2 + dx:R + 1 + dx, 1:C + 1]
    bx[:, xs, ys] = (im(-2) + im(-1) * 4.0 + im(0) * 6.0 + im(1) * 4.0 +
                     im(2)) * 0.0625
    # blury on x in [2, R], y in [2, C] (:57-62)
    by = np.zeros((3, R + 2, C + 2))

    def b(dy):
        return bx[:, 2:R + 1, 2 + dy:C + 1 + dy]
    by[:, 2:R + 1, 2:C + 1] = (b(-2) + b(-1) * 4.0 + b(0) * 6.0 +
                               b(1) * 4.0 + b(2)) * 0.0625
    src = img[:, 2:R + 1, 2:C + 1]
    blur = by[:, 2:R + 1, 2:C + 1]
    sharpen = src * (1 + weight) - blur * weight          # (:64-66)
    masked = np.where(np.abs(src - blur) < threshold, src, sharpen)  # (:68)
    res[:, 0:R - 1, 0:C - 1] = masked
    return res


def margin(img, threshold):
    """Distance of ``|img - blury|`` from ``threshold`` at written points
    (inf elsewhere): pixels with a tiny margin may legitimately take either
    arm of the select under float rounding."""
    img = np.asarray(img, dtype=np.float64)
    _, H, W = img.shape
    R, C = H - 4, W - 4
    # with weight 0 both arms equal img, so recover blury from a second
    # evaluation with weight 1: sharpen = 2*img - blur
    a = unsharp(img, -1.0, 1.0)      # threshold < 0: always the sharpen arm
    blur = 2.0 * img[:, 2:R + 1, 2:C + 1] - a[:, 0:R - 1, 0:C - 1]
    m = np.full((3, R, C), np.inf)
    m[:, 0:R - 1, 0:C - 1] = np.abs(np.abs(img[:, 2:R + 1, 2:C + 1] - blur)
                                    - threshold)
    return m


def defined_region(R, C):
    """(x0, x1, y0, y1) slices of the [3][R][C] output that do not depend on
    the uncomputed-point convention: domain x in [2, R], y in [3, C-2]."""
    return slice(0, R - 1), slice(1, C - 3)


def make_input(R, C, seed=0):
    """Synthetic workload: planar [3][R+4][C+4] float32, U[0,1) inside and
    a zero ghost zone of 2 pixels (as unsharp_mask/init.py:26-35 builds)."""
    rng = np.random.default_rng(seed)
    img = np.zeros((3, R + 4, C + 4), np.float32)
    img[:, 2:R + 2, 2:C + 2] = rng.random((3, R, C), dtype=np.float32)
    return img
