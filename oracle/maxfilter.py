"""Integer restatement of the reference's max filter spec
(sandbox/apps/python/img_proc/max_filter/polymage_maxfilter.py:14-103) --
test infrastructure only, in NumPy with C semantics (int32 stores of the
float image's values, truncating casts, double log / pow).

Readings of what the spec leaves ill-formed (the same as the DSL
statement's, polymage_b200/apps/max_filter.py): the first Reduce writes
vert_log at its reduction variables' point (x, rx, c, ry); reads of
vert_log outside its domain (y - t < 0) give 0; a data-dependent index
(final's slice, filter_height(dx) up to r + 1) is clamped into the
producer's domain, as the compiled code clamps every data-dependent
index; Reductions start at 0.
Parity unpinned: the reference holds no output of this app.
"""

import math

import numpy as np

RADIUS = 26


def maxfilter(img):
    """img: float32 [3][R][C] (values 0..255) -> int32 [R][C][3]."""
    img = np.asarray(img, np.float32)
    _, R, C = img.shape
    r = RADIUS
    slices = int(math.ceil(math.log(r, 2))) + 1

    def cl(k, i, j):
        return img[k, np.clip(i, 0, R - 1), np.clip(j, 0, C - 1)]

    # vert_log(x, y, c, t): Op.Max over rx in [r, C-R-3r-1], ry in
    # [1, slices-1] of max(img(x, rx), img(x, rx + clamp(2^(ry-1))))
    vl = np.zeros((R, C, 3, slices + 1), np.int64)
    xs = np.arange(R)[:, None]
    for ry in range(1, slices):
        step = min(max(int(math.pow(2, ry - 1)), 0), 2 * r)
        for rx in range(r, C - R - 3 * r - 1 + 1):
            for c in range(3):
                a = cl(c, xs[:, 0], rx)
                b = cl(c, xs[:, 0], rx + step)
                v = np.where(a > b, a, b).astype(np.int64)   # Max(a, b)
                vl[:, rx, c, ry] = np.maximum(vl[:, rx, c, ry], v)

    sfr = [int(math.log(2 * t + 1) / 0.693147) for t in range(slices + 1)]
    # vert(x, y, c, t)
    vert = np.zeros((R, C, 3, slices + 1), np.int64)
    ys = np.arange(C)
    for t in range(slices + 1):
        e = min(max(sfr[t], 0), slices)
        s2 = min(max(int(math.pow(2, e)), 0), 2 * r)
        y1 = ys - t
        y2 = ys + t + 1 - s2
        a = np.zeros((R, C, 3), np.int64)
        b = np.zeros((R, C, 3), np.int64)
        ok1 = (y1 >= 0) & (y1 <= C - 1)
        ok2 = (y2 >= 0) & (y2 <= C - 1)
        ve = vl[:, :, :, e]
        a[:, ok1, :] = ve[:, y1[ok1], :]
        b[:, ok2, :] = ve[:, y2[ok2], :]
        vert[..., t] = np.where(a > b, a, b)
    # filter_height(x) for x in [-r, 2r+1]: Sum over x in [0, r], dy in
    # [0, r+1] of (x^2 + dy^2 < (r + 0.25)^2)
    rr = (r + 0.25) * (r + 0.25)
    fh = {}
    for x in range(-r, 2 * r + 2):
        fh[x] = 0
    for x in range(0, r + 1):
        for dy in range(0, r + 2):
            if x * x + dy * dy < rr:
                fh[x] += 1
    # final(x, y, c): Op.Max over x in [r, R-2r-2], dx in [-r, 2r+1] of
    # vert(x+dx, y, c, clamp(fh(dx), 0, r+1))
    out = np.zeros((R, C, 3), np.int64)
    x0, x1 = r, R - 2 * r - 2
    if x1 >= x0:
        for dx in range(-r, 2 * r + 2):
            # the slice index is data dependent (filter_height) and reaches
            # r + 1 > slices: it is clamped into vert's domain [0, slices]
            # as every data-dependent index is
            t = min(min(max(fh[dx], 0), r + 1), slices)
            v = vert[x0 + dx:x1 + dx + 1, :, :, t]
            out[x0:x1 + 1] = np.maximum(out[x0:x1 + 1], v)
    return out.astype(np.int32)


def make_input(R, C, seed=0):
    rng = np.random.default_rng(seed)
    return rng.integers(0, 256, (3, R, C)).astype(np.float32)
