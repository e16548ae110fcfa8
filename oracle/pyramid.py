"""FP64 restatement of the reference's Laplacian pyramid blending spec
(sandbox/apps/python/img_proc/pyramid_blend/polymage_blending.py:13-196)
-- test infrastructure only.  ``L`` levels (the reference fixes L = 4).

Each function is an array over its domain box; index expressions use the
spec's integer arithmetic (truncating division on non-negative indices).
"""

import numpy as np


class Box(object):
    """A function's values over the box lo[d] .. lo[d] + shape[d] - 1."""

    def __init__(self, data, lo):
        self.data = data
        self.lo = tuple(lo)

    def at(self, *idx):
        return self.data[tuple(np.asarray(i) - l for i, l in
                               zip(idx, self.lo))]


def _grid(ranges):
    axes = [np.arange(a, b + 1) for a, b in ranges]
    return np.meshgrid(*axes, indexing='ij')


def pyramid_blend(img1, img2, mask, L=4):
    """img1, img2: [3][R][C]; mask: [R][C] -> float64 [3][Ro][Co] over the
    output domain [2^(L+1)-1, R - 2^(L+1) + 2] (per side)."""
    img1 = np.asarray(img1, np.float64)
    img2 = np.asarray(img2, np.float64)
    mask = np.asarray(mask, np.float64)
    _, R, C = img1.shape
    g1 = {0: Box(img1, (0, 0, 0))}
    g2 = {0: Box(img2, (0, 0, 0))}
    gm = {0: Box(mask, (0, 0))}

    def down(f, l, color):
        # :42-89
        dec, org = 1 << l, 1 << (l - 1)
        xr = (l, R // dec - 2)
        ycol = (l - 1, C // org - 2)
        ydec = (l, C // dec - 2)
        w = (1, 4, 6, 4, 1)
        if color:
            c, x, y = _grid([(0, 2), xr, ycol])
            dx = sum(wt * f.at(c, 2 * x + k, y)
                     for k, wt in zip(range(-2, 3), w)) * 0.0625
            dxb = Box(dx, (0, xr[0], ycol[0]))
            c, x, y = _grid([(0, 2), xr, ydec])
            dy = sum(wt * dxb.at(c, x, 2 * y + k)
                     for k, wt in zip(range(-2, 3), w)) * 0.0625
            return Box(dy, (0, xr[0], ydec[0]))
        x, y = _grid([xr, ycol])
        dx = sum(wt * f.at(2 * x + k, y)
                 for k, wt in zip(range(-2, 3), w)) * 0.0625
        dxb = Box(dx, (xr[0], ycol[0]))
        x, y = _grid([xr, ydec])
        dy = sum(wt * dxb.at(x, 2 * y + k)
                 for k, wt in zip(range(-2, 3), w)) * 0.0625
        return Box(dy, (xr[0], ydec[0]))

    for l in range(1, L):
        g1[l] = down(g1[l - 1], l, True)
        g2[l] = down(g2[l - 1], l, True)
        gm[l] = down(gm[l - 1], l, False)

    def rows_cols(l):
        rowr = ((1 << (L - l + 1)) - 1, R // (1 << l) - (1 << (L - l + 1)) + 2)
        colr = ((1 << (L - l + 1)) - 1, C // (1 << l) - (1 << (L - l + 1)) + 2)
        dec_colr = ((1 << (L - l)) - 1,
                    C // (1 << (l + 1)) - (1 << (L - l)) + 2)
        return rowr, colr, dec_colr

    def up(fd, f, l, sign):
        # :91-136 (sign -1) and :152-194 (sign +1)
        rowr, colr, dec_colr = rows_cols(l)
        c, x, y = _grid([(0, 2), rowr, dec_colr])
        even = (fd.at(c, x // 2 - 1, y) + 6 * fd.at(c, x // 2, y) +
                fd.at(c, x // 2 + 1, y)) * 0.125
        odd = (4 * fd.at(c, (x - 1) // 2, y) + 4 * fd.at(c, (x + 1) // 2, y)
               ) * 0.125
        upx = Box(np.where(x % 2 == 0, even, odd), (0, rowr[0], dec_colr[0]))
        c, x, y = _grid([(0, 2), rowr, colr])
        even = (upx.at(c, x, y // 2 - 1) + 6 * upx.at(c, x, y // 2) +
                upx.at(c, x, y // 2 + 1)) * 0.125
        odd = (4 * upx.at(c, x, (y - 1) // 2) + 4 * upx.at(c, x, (y + 1) // 2)
               ) * 0.125
        base = f.at(c, x, y)
        v = np.where(y % 2 == 0, base + sign * even, base + sign * odd)
        return Box(v, (0, rowr[0], colr[0]))

    lap1, lap2 = {}, {}
    for l in range(L - 1):
        lap1[l] = up(g1[l + 1], g1[l], l, -1)
        lap2[l] = up(g2[l + 1], g2[l], l, -1)
    lap1[L - 1] = g1[L - 1]
    lap2[L - 1] = g2[L - 1]
    res = {}
    for l in range(L):
        rowr, colr, _ = rows_cols(l)
        c, x, y = _grid([(0, 2), rowr, colr])
        m = gm[l].at(x, y)
        res[l] = Box(lap1[l].at(c, x, y) * m + lap2[l].at(c, x, y) * (1 - m),
                     (0, rowr[0], colr[0]))
    out = res[L - 1]
    for l in range(L - 2, -1, -1):
        out = up(out, res[l], l, +1)
    return out.data


def output_box(R, C, L=4):
    m = (1 << (L + 1)) - 1
    return (m, R - (1 << (L + 1)) + 2), (m, C - (1 << (L + 1)) + 2)


def make_inputs(R, C, seed=0):
    rng = np.random.default_rng(seed)
    img1 = rng.random((3, R, C), dtype=np.float32)
    img2 = rng.random((3, R, C), dtype=np.float32)
    mask = rng.random((R, C), dtype=np.float32)
    return img1, img2, mask


# ---------------------------------------------------------------------------
# Generalized spec: any number of levels on any image size, indices clamped
# to each level's domain (polymage_b200/apps/pyramid_blend.py,
# pyramid_blending_clamped).  The filters are the reference's
# (polymage_blending.py:42-194); only the boundary handling differs.

def _down_rows(g):
    """5-tap [1,4,6,4,1]/16 decimation by 2 along axis -2, clamped."""
    n = g.shape[-2]
    m = (n + 1) // 2
    x = np.arange(m)
    w = (1, 4, 6, 4, 1)
    out = 0.0
    for k in range(5):
        idx = np.clip(2 * x + k - 2, 0, n - 1)
        out = out + w[k] * np.take(g, idx, axis=-2)
    return out * 0.0625


def _down(g):
    return np.swapaxes(_down_rows(np.swapaxes(_down_rows(g), -1, -2)),
                       -1, -2)


def _up_rows(g, n):
    """Level-l+1 rows interpolated to ``n`` rows (even: [1,6,1]/8, odd:
    [4,4]/8), clamped."""
    m = g.shape[-2]
    x = np.arange(n)
    h = x // 2
    lo = np.clip(h - 1, 0, m - 1)
    hi = np.clip(h + 1, 0, m - 1)
    gh = np.take(g, h, axis=-2)
    even = (np.take(g, lo, axis=-2) + 6 * gh + np.take(g, hi, axis=-2)) * \
        0.125
    odd = (4 * gh + 4 * np.take(g, hi, axis=-2)) * 0.125
    sel = (x % 2 == 0).reshape((-1, 1))
    return np.where(sel, even, odd)


def _up(g, n_rows, n_cols):
    u = _up_rows(g, n_rows)
    return np.swapaxes(_up_rows(np.swapaxes(u, -1, -2), n_cols), -1, -2)


def pyramid_blend_clamped(img1, img2, mask, L=8):
    """img1, img2: [3][R][C]; mask: [R][C] -> float64 [3][R][C]."""
    g1 = [np.asarray(img1, np.float64)]
    g2 = [np.asarray(img2, np.float64)]
    gm = [np.asarray(mask, np.float64)]
    for _ in range(1, L):
        g1.append(_down(g1[-1]))
        g2.append(_down(g2[-1]))
        gm.append(_down(gm[-1]))

    def lap(g, l):
        if l == L - 1:
            return g[l]
        r, c = g[l].shape[-2:]
        return g[l] - _up(g[l + 1], r, c)
    res = [lap(g1, l) * gm[l] + lap(g2, l) * (1 - gm[l]) for l in range(L)]
    out = res[L - 1]
    for l in range(L - 2, -1, -1):
        r, c = res[l].shape[-2:]
        out = res[l] + _up(out, r, c)
    return out
