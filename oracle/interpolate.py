"""Pyramid interpolation, restated in NumPy FP64 -- test infrastructure
only.  Follows the reference app's spec
(sandbox/apps/python/img_proc/interpolate/polymage_interpolate.py:14-189):
premultiplied level 0 (:152-155), [1 2 1]/4 decimations with zero borders
(:39-85), upsampling by averaging rows (x+1)/2 and (x+2)/2 then columns,
``interpolated_l = D_l + (1 - alpha_l) * up`` (:87-149), and division by
the alpha channel (:163-169).  Parity unpinned: the reference tree holds
no generated code for this app; the restatement is checked against a
direct evaluation of the DSL definitions (tests/test_dsl_eval.py).
"""

import numpy as np


def _down_x(f, rd, co):
    """Dx over [0, rd+1] x [0, co+1]: interior rows 1..rd, cols 1..co."""
    out = np.zeros((f.shape[0], rd + 2, co + 2))
    x = np.arange(1, rd + 1)
    core = (f[:, 2 * x - 2, :] + f[:, 2 * x - 1, :] * 2.0 +
            f[:, 2 * x, :]) * 0.25
    out[:, 1:rd + 1, 1:co + 1] = core[:, :, 1:co + 1]
    return out


def _down_y(f, rd, cd):
    out = np.zeros((f.shape[0], rd + 2, cd + 2))
    y = np.arange(1, cd + 1)
    core = (f[:, :, 2 * y - 2] + f[:, :, 2 * y - 1] * 2.0 +
            f[:, :, 2 * y]) * 0.25
    out[:, 1:rd + 1, 1:cd + 1] = core[:, 1:rd + 1, :]
    return out


def interpolate(img, L=10):
    """img: float32 [4][R+2][C+2] -> float64 [3][R][C]."""
    img = np.asarray(img, np.float64)
    R, C = img.shape[1] - 2, img.shape[2] - 2
    ds = [img * img[3:4]]
    for l in range(1, L):
        rd, cd, co = R >> l, C >> l, C >> (l - 1)
        ds.append(_down_y(_down_x(ds[-1], rd, co), rd, cd))
    it = ds[L - 1]
    for l in range(L - 2, -1, -1):
        ro, co, cd = R >> l, C >> l, C >> (l + 1)
        ux = np.zeros((4, ro + 2, cd + 2))
        x = np.arange(1, ro + 1)
        ux[:, 1:ro + 1, 1:cd + 1] = ((it[:, (x + 1) // 2, :] +
                                      it[:, (x + 2) // 2, :]) / 2.0)[
            :, :, 1:cd + 1]
        y = np.arange(1, co + 1)
        upy = (ux[:, :, (y + 1) // 2] + ux[:, :, (y + 2) // 2]) / 2.0
        d = ds[l]
        out = np.zeros((4, ro + 2, co + 2))
        out[:, 1:ro + 1, 1:co + 1] = (
            d[:, 1:ro + 1, 1:co + 1] +
            (1.0 - d[3:4, 1:ro + 1, 1:co + 1]) * upy[:, 1:ro + 1, :])
        it = out
    return it[0:3, 1:R + 1, 1:C + 1] / it[3:4, 1:R + 1, 1:C + 1]


def make_input(R, C, seed=0):
    """RGBA in [0, 1) with alpha in [0.25, 1) (the division by alpha stays
    well conditioned), zero ghost border."""
    rng = np.random.default_rng(seed)
    img = np.zeros((4, R + 2, C + 2), np.float32)
    img[0:3, 1:R + 1, 1:C + 1] = rng.random((3, R, C), dtype=np.float32)
    img[3, 1:R + 1, 1:C + 1] = 0.25 + 0.75 * rng.random((R, C),
                                                        dtype=np.float32)
    return img
