"""Builds with option 'prefetch' (a CTA loads its next tile's staged inputs
into a second copy of their shared-memory buffers while it computes the
current tile) against the oracles, with the single-image tolerances:
unsharp max |d| <= 1e-5 where the select margin exceeds 1e-6, Harris
max |d| / max |ref| <= 1e-5, camera pipe bit-exact, bilateral 1e-5,
8-level pyramid 2e-5.  Sizes include the benchmark sizes (persistent
launches, several tiles per CTA, so the copies alternate) and odd sizes;
a batch of uneven images checks the prefetch across image boundaries of
the tile queue."""

import numpy as np
import pytest

import oracle.bilateral as OB
import oracle.campipe as OC
import oracle.harris as OH
import oracle.pyramid as OP
import oracle.unsharp as OU
from polymage_b200.apps import catalog

pytestmark = pytest.mark.gpu

_cache = {}


def build(app, **over):
    key = (app, tuple(sorted(over.items())))
    if key not in _cache:
        b, kw = catalog._BUILDERS[app]
        kw = dict(kw)
        kw.update(over)
        kw['options'] = tuple(kw.get('options', ())) + ('prefetch',)
        _cache[key] = b(**kw).build()
    return _cache[key]


@pytest.mark.parametrize("tile", [(128, 128), (64, 128)])
@pytest.mark.parametrize("R,C", [(4096, 4096), (1037, 771), (67, 133)])
def test_unsharp_prefetch(tile, R, C):
    cp = build("unsharp", tile_sizes=tile)
    img = OU.make_input(R, C, seed=R)
    out = np.zeros((3, R, C), np.float32)
    cp.run_host({'R': R, 'C': C, 'threshold': 0.001, 'weight': 3.0},
                {'img': img}, {'mask': out})
    ref = OU.unsharp(img, 0.001, 3.0)
    xs, ys = OU.defined_region(R, C)
    ok = OU.margin(img, 0.001)[:, xs, ys] > 1e-6
    d = np.abs(out[:, xs, ys].astype(np.float64) - ref[:, xs, ys])
    assert d[ok].max() <= 1e-5


@pytest.mark.parametrize("n", [2048, 999])
def test_harris_prefetch(n):
    cp = build("harris")
    img = OH.make_input(n, n + 7, seed=n)
    out = np.zeros((n, n + 7), np.float32)
    cp.run_host({'R': n - 2, 'C': n + 5}, {'img': img}, {'harris': out})
    ref = OH.harris(img)
    assert np.abs(out - ref).max() / np.abs(ref).max() <= 1e-5


@pytest.mark.parametrize("R,C", [(1968, 2592), (131, 197)])
def test_campipe_prefetch(R, C):
    cp = build("campipe")
    img = OC.make_input(R, C, seed=R + C)
    out = np.zeros((3, R - 48, C - 64), np.uint8)
    cp.run_host({'C': C, 'R': R, 'colour_temp': 3700.0, 'contrast': 50.0,
                 'gamma': 2.0}, {'img': img, 'matrix_3200': OC.MATRIX_3200,
                                 'matrix_7000': OC.MATRIX_7000},
                {'process': out})
    assert np.array_equal(out, OC.campipe(img, 3700.0, 50.0, 2.0))


@pytest.mark.parametrize("rows,cols", [(1536, 2560), (200, 331)])
def test_bilateral_prefetch(rows, cols):
    cp = build("bilateral")
    img = OB.make_input(rows, cols, seed=rows + cols)
    out = np.zeros((1, rows, cols), np.float32)
    cp.run_host({'rows': rows, 'cols': cols}, {'input': img},
                {'filtered': out})
    assert np.abs(out.astype(np.float64) - OB.bilateral(img)).max() <= 1e-5


@pytest.mark.parametrize("R,C", [(2048, 2048), (301, 517)])
def test_pyramid8_prefetch(R, C):
    cp = build("pyramid8")
    img1, img2, mask = OP.make_inputs(R, C, seed=R)
    out = np.zeros((3, R, C), np.float32)
    cp.run_host({'R': R, 'C': C}, {'img1': img1, 'img2': img2,
                                   'mask': mask}, {'blend': out})
    ref = OP.pyramid_blend_clamped(img1, img2, mask, L=8)
    assert np.abs(out.astype(np.float64) - ref).max() <= 2e-5


def test_unsharp_prefetch_batch_uneven(cuda):
    """Twelve images of uneven sizes through one persistent launch: a CTA's
    next tile may belong to another image (another descriptor)."""
    import torch
    cp = build("unsharp", tile_sizes=(64, 128))
    rng = np.random.default_rng(5)
    prms, ins, outs, imgs = [], [], [], []
    for i in range(12):
        R, C = (int(v) for v in rng.integers(64, 1500, 2))
        img = OU.make_input(R, C, seed=100 + i)
        imgs.append(img)
        prms.append({'R': R, 'C': C, 'threshold': 0.001, 'weight': 3.0})
        ins.append({'img': torch.from_numpy(img).to(cuda)})
        outs.append({'mask': torch.zeros((3, R, C), dtype=torch.float32,
                                         device=cuda)})
    for graph in (False, True):
        for o in outs:
            o['mask'].zero_()
        cp.run_batch(prms, ins, outs, graph=graph)
        torch.cuda.synchronize()
        cp.check()
        for p, o, img in zip(prms, outs, imgs):
            R, C = p['R'], p['C']
            ref = OU.unsharp(img, 0.001, 3.0)
            xs, ys = OU.defined_region(R, C)
            ok = OU.margin(img, 0.001)[:, xs, ys] > 1e-6
            got = o['mask'].cpu().numpy()[:, xs, ys].astype(np.float64)
            assert np.abs(got - ref[:, xs, ys])[ok].max() <= 1e-5
