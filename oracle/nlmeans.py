"""FP64 restatement of the reference's non-local means spec
(sandbox/apps/python/img_proc/non_local_means/polymage_nlmeans.py:13-165)
-- test infrastructure only.

Conventions (the spec reads outside what it defines):
* channel 3 of the 3-channel image reads 0 (the reference's driver passes
  a 4-channel buffer whose channel 3 is zero: non_local_means/init.py:
  28-29);
* Reduction points outside a reduction's domain keep its default, 0;
  outside the interior the output is then min/max of 0/0 against 1 and 0,
  which the spec's selects make 1.0 (a NaN compares false);
* integer divisions truncate toward zero (``-search_area / 2``).
Parity unpinned: the reference holds no output of this app.
"""

import numpy as np

SIGMA = 0.12


def _tdiv(a, b):
    return int(a / b)


def nlmeans(img, patch_size=7, search_area=7):
    """img: float32 [3][R][C] -> float64 [3][R][C]."""
    img = np.asarray(img, np.float64)
    _, R, C = img.shape
    img4 = np.zeros((4, R, C))
    img4[:3] = img
    p, s = patch_size, search_area
    offs = range(_tdiv(-s, 2), s + 2)
    win = range(_tdiv(-p, 2), p + 2)
    xs = np.arange(R)[:, None]
    ys = np.arange(C)[None, :]

    def cl(i, j):
        return img4[:, np.clip(i, 0, R - 1), np.clip(j, 0, C - 1)]

    inv = -1.0 / (SIGMA * SIGMA * p * p)
    base = cl(xs, ys)
    nls = np.zeros((4, R, C))
    x0, x1 = _tdiv(s, 2), R - s - 2
    y0, y1 = _tdiv(s, 2), C - s - 2
    px0, px1 = _tdiv(p, 2), R - p - 2
    py0, py1 = _tdiv(p, 2), C - p - 2
    for dx in offs:
        for dy in offs:
            # d: sum over the 4 channels of the squared difference (:62-89)
            d = ((base - cl(xs + dx, ys + dy)) ** 2).sum(axis=0)
            # blur along y on [p/2, C-p-2], then along x on [p/2, R-p-2]
            bdy = np.zeros((R, C))
            if py1 >= py0:
                for pv in win:
                    bdy[:, py0:py1 + 1] += d[:, py0 + pv:py1 + 1 + pv]
            bd = np.zeros((R, C))
            if px1 >= px0:
                for pv in win:
                    bd[px0:px1 + 1, :] += bdy[px0 + pv:px1 + 1 + pv, :]
            w = np.exp(bd * inv)
            if x1 >= x0 and y1 >= y0:
                cwa = cl(xs + dx, ys + dy)
                cwa[3] = 1.0
                nls[:, x0:x1 + 1, y0:y1 + 1] += \
                    (w[None] * cwa)[:, x0:x1 + 1, y0:y1 + 1]
    with np.errstate(divide='ignore', invalid='ignore'):
        q = nls[:3] / nls[3:4]
    q = np.where(q < 1.0, q, 1.0)          # Min(q, 1.0): NaN gives 1.0
    return np.where(q > 0.0, q, 0.0)       # Max(., 0.0)


def make_input(R, C, seed=0):
    """A smooth image (a ramp and sinusoids per channel) with small noise,
    so that patches resemble each other and the weights are not all 0."""
    rng = np.random.default_rng(seed)
    x = np.arange(R)[:, None] / max(R, 1)
    y = np.arange(C)[None, :] / max(C, 1)
    img = np.empty((3, R, C), np.float32)
    for c in range(3):
        img[c] = 0.5 + 0.3 * np.sin(6.0 * x + 2.0 * c) * np.cos(5.0 * y) + \
            0.02 * rng.standard_normal((R, C))
    return img
