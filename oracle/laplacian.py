"""Local Laplacian filter, restated in NumPy float32 with the operation
order of the reference's generated pipeline_laplacian
(sandbox/video_demo/laplacian_polymage.cpp:10-1062) -- test
infrastructure only.  It checks the DSL statement of the pipeline
(polymage_b200/apps/local_laplacian.py) against the reference's own
compiled code on the CPU; the GPU output is checked against that
compiled code (oracle/ref.py ref_laplacian) and the committed fixtures.

Stage order and index conventions follow the reference (line numbers of
laplacian_naive.cpp, the untiled copy of the same stages):
grey level and edge padding (:202-213 and :64-135 of the tiled file),
remap LUT (:202-205), gPyramid_L0 (:216-235), [1 3 3 1]/8 decimation
(:237-390), Laplacian levels with 0.25/0.75 upsampling (:395-700),
intensity blending (:515), collapse and colour output (:700-900).
"""

import numpy as np

F = np.float32


def _gray(frame):
    """Grey level of the frame padded by 31/61 pixels with edge values:
    (0.299 R + 0.587 G + 0.114 B) / 255 (double division)."""
    f = frame.astype(F)
    s = (F(0.299) * f[:, :, 2] + F(0.587) * f[:, :, 1]) + \
        F(0.114) * f[:, :, 0]
    g = (s.astype(np.float64) / 255.0).astype(F)
    return np.pad(g, ((31, 61), (31, 61)), mode='edge')


def _down(a, axis):
    """[1 3 3 1]/8 decimation along ``axis`` onto [1, n/2 - 2] (stored
    from index 1; index 0 unused)."""
    n = a.shape[axis]
    m = n // 2
    x = np.arange(1, m - 1)

    def t(o):
        return np.take(a, 2 * x + o, axis=axis)
    core = (((t(-1) + F(3.0) * t(0)) + F(3.0) * t(1)) + t(2)) * F(0.125)
    pad = [(0, 0)] * a.ndim
    pad[axis] = (1, 1)
    return np.pad(core, pad)


def _up(a, axis, lo, hi):
    """0.25 a(x/2 - 1 + 2(x%2)) + 0.75 a(x/2) for x in [lo, hi], placed at
    indices lo..hi of an array of length hi + 1 (zeros elsewhere)."""
    x = np.arange(lo, hi + 1)
    h = x // 2
    other = np.where(x % 2 == 0, h - 1, h + 1)
    v = F(0.25) * np.take(a, other, axis=axis) + \
        F(0.75) * np.take(a, h, axis=axis)
    pad = [(0, 0)] * a.ndim
    pad[axis] = (lo, 0)
    return np.pad(v, pad)


def _inner(n, l, J=5):
    if l == J - 1:
        return 1, n // 16 - 2
    return (1 << (5 - l)) - 1, (n >> l) - (1 << (6 - l)) + 2


def local_laplacian(frame, alpha=1.0 / 3.0, beta=1.0):
    """frame: uint8 [rows][cols][3] (B, G, R) -> uint8 [rows][cols][3]."""
    alpha, beta = F(alpha), F(beta)
    H, W, _ = frame.shape
    R, C = H + 92, W + 92
    img = _gray(frame)
    i = np.arange(-768, 768)
    fi = i.astype(F) / F(256.0)
    lut = (alpha * fi) * np.exp(((-fi) * fi) / F(2.0)).astype(F)
    v = np.clip((img * F(768.0)).astype(np.int64), 0, 768)
    k = np.arange(4).reshape(4, 1, 1)
    kt = (k * F(0.333333333333)).astype(F)
    idx = np.clip(v[None] - 256 * k + 768, 0, 1535)
    g0 = (beta * (img[None] - kt) + kt) + lut[idx]
    gP = [g0]
    inG = [img]
    for l in range(1, 5):
        gP.append(_down(_down(gP[-1], 1), 2))
        inG.append(_down(_down(inG[-1], 0), 1))
    lP = {4: gP[4]}
    for l in range(3, -1, -1):
        rlo, rhi = _inner(R, l)
        clo, chi = _inner(C, l)
        c1lo, c1hi = _inner(C, l + 1)
        ux = _up(gP[l + 1][:, :, :c1hi + 1], 1, rlo, rhi)
        u = np.zeros_like(gP[l][:, :rhi + 1, :chi + 1])
        up = _up(ux, 2, clo, chi)
        u[:, rlo:, clo:] = gP[l][:, rlo:rhi + 1, clo:chi + 1] - \
            up[:, rlo:, clo:]
        lP[l] = u
    outL = {}
    for l in range(5):
        rlo, rhi = _inner(R, l)
        clo, chi = _inner(C, l)
        g3 = inG[l][rlo:rhi + 1, clo:chi + 1] * F(3.0)
        li = np.clip(g3.astype(np.int64), 0, 2)
        lf = g3 - li.astype(F)
        xs = np.arange(rlo, rhi + 1)[:, None]
        ys = np.arange(clo, chi + 1)[None, :]
        a = lP[l][li, xs, ys]
        b = lP[l][li + 1, xs, ys]
        o = np.zeros((rhi + 1, chi + 1), F)
        o[rlo:, clo:] = (F(1.0) - lf) * a + lf * b
        outL[l] = o
    outG = outL[4]
    for l in range(3, -1, -1):
        rlo, rhi = _inner(R, l)
        clo, chi = _inner(C, l)
        c1lo, c1hi = _inner(C, l + 1)
        ux = _up(outG[:, :c1hi + 1], 0, rlo, rhi)
        up = _up(ux, 1, clo, chi)
        g = np.zeros((rhi + 1, chi + 1), F)
        g[rlo:, clo:] = outL[l][rlo:, clo:] + up[rlo:, clo:]
        outG = g
    res = outG[31:31 + H, 31:31 + W]
    gi = img[31:31 + H, 31:31 + W]
    col = frame.astype(F) / F(256.0) + F(0.01)
    val = (res[:, :, None] * col) / (gi[:, :, None] + F(0.01))
    val = np.minimum(np.maximum(val, F(0.0)), F(1.0))
    return (val * F(255.0)).astype(np.uint8)
