"""FP64 restatement of the reference's bilateral-grid spec
(sandbox/apps/python/img_proc/bilateral_grid/polymage_bilateral_grid.py:
16-130) -- test infrastructure only.

The z bin follows the C types of the reference's generated code: ``img *
10`` is a float product (float * int), truncated to int (:57-63, :93-97),
so every point falls into the bin the compiled code puts it in; the rest,
the fraction ``img * 10 - bin`` included, is evaluated in double.  Grid points that no
``Case`` covers read as 0 (blury at z = 12 and at the last row/column
block, which the reference leaves uninitialized); splats whose z bin falls outside the grid (inputs >=
1.4) are dropped.
"""

import numpy as np


def _blur(a, axis, interior):
    """Unnormalised [1,4,6,4,1] along ``axis`` on the interior (:65-91),
    0 outside; interior taps never wrap around the array."""
    out = np.zeros_like(a)
    acc = None
    for k, wt in zip(range(-2, 3), (1, 4, 6, 4, 1)):
        sh = np.roll(a, -k, axis=axis)
        acc = sh * wt if acc is None else acc + sh * wt
    out[interior] = acc[interior]
    return out


def bilateral(img):
    """img: float32 [rows][cols] -> float64 [1][rows][cols]."""
    img = np.asarray(img, dtype=np.float32)
    rows, cols = img.shape
    gx, gy = rows // 8 + 4, cols // 8 + 4
    grid = np.zeros((2, gx, gy, 14))
    x, y = np.meshgrid(np.arange(rows), np.arange(cols), indexing='ij')
    zv32 = img * np.float32(10)                 # float * int -> float
    zb = np.trunc(zv32).astype(np.int64)
    cx, cy, cz = 2 + x // 8, 2 + y // 8, 2 + zb
    ok = (cz >= 0) & (cz <= 13)
    np.add.at(grid[0], (cx[ok], cy[ok], cz[ok]), img[ok].astype(np.float64))
    np.add.at(grid[1], (cx[ok], cy[ok], cz[ok]), 1.0)
    # interior: x in [2, rows/8+1], y in [2, cols/8+1], z in [2, 11]
    interior = np.zeros(grid.shape, dtype=bool)
    interior[:, 2:rows // 8 + 2, 2:cols // 8 + 2, 2:12] = True
    blurz = _blur(grid, 3, interior)
    blurx = _blur(blurz, 1, interior)
    blury = _blur(blurx, 2, interior)
    zi = zb
    zf = img.astype(np.float64) * 10 - zi         # the fraction in FP64
    xf = (x % 8).astype(np.float32) / np.float32(8)
    yf = (y % 8).astype(np.float32) / np.float32(8)
    xf = xf.astype(np.float64)
    yf = yf.astype(np.float64)
    xi, yi = x // 8, y // 8

    def lerp(a, b, w):
        return a + w * (b - a)

    out = np.zeros((1, rows, cols))
    interp = []
    for c in (0, 1):
        def g(dx, dy, dz):
            zz = np.clip(2 + zi + dz, 0, 13)
            return blury[c, 2 + xi + dx, 2 + yi + dy, zz]
        z0 = lerp(lerp(g(0, 0, 0), g(1, 0, 0), xf),
                  lerp(g(0, 1, 0), g(1, 1, 0), xf), yf)
        z1 = lerp(lerp(g(0, 0, 1), g(1, 0, 1), xf),
                  lerp(g(0, 1, 1), g(1, 1, 1), xf), yf)
        interp.append(lerp(z0, z1, zf))
    i0, i1 = interp
    with np.errstate(divide='ignore', invalid='ignore'):
        out[0] = np.where(i1 > 0, i0 / np.where(i1 > 0, i1, 1.0),
                          img.astype(np.float64))
    return out


def make_input(rows, cols, seed=0):
    rng = np.random.default_rng(seed)
    return rng.random((rows, cols), dtype=np.float32)
