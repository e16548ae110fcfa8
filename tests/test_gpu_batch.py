"""Batched execution through pipeline_<name>_batch and _batch_graph.

Many images of different sizes, each with its own parameters, run through
each group in one launch; every image is checked against the oracle with
the tolerance of the single-image parity tests (bilateral 1e-5, unsharp
1e-5 where the select margin exceeds 1e-6, Harris 1e-5 relative, pyramid
2e-5, camera pipe bit-exact).  Batches whose groups have more tiles than
fit on the GPU at once run as a persistent grid draining a device-side tile
queue.  A repeated call with unchanged arguments relaunches the kernels
with the descriptors already on the device, and _batch_graph runs the
batch as a CUDA graph; both must recompute from the inputs' current
contents.
"""

import numpy as np
import pytest

import oracle.bilateral as OB
import oracle.campipe as OC
import oracle.harris as OH
import oracle.pyramid as OP
import oracle.unsharp as OU
from polymage_b200.apps import catalog
from polymage_b200.runtime import PipelineRuntimeError
from tests import pipelines

pytestmark = pytest.mark.gpu


def _zero(outs):
    for o in outs:
        for t in o.values():
            t.zero_()


def _bilateral_batch(cuda, sides, seed):
    import torch
    prms, ins, outs, imgs = [], [], [], []
    for i, (r, c) in enumerate(sides):
        img = OB.make_input(r, c, seed=seed * 1000 + i)
        imgs.append(img)
        prms.append({'rows': r, 'cols': c})
        ins.append({'input': torch.from_numpy(img).to(cuda)})
        outs.append({'filtered': torch.zeros((1, r, c), dtype=torch.float32,
                                             device=cuda)})
    return prms, ins, outs, imgs


def _check_bilateral(outs, imgs):
    for o, img in zip(outs, imgs):
        ref = OB.bilateral(img)
        err = np.abs(o['filtered'].cpu().numpy().astype(np.float64) -
                     ref).max()
        assert err <= 1e-5, err


def test_bilateral_batch_uneven_sizes(cuda):
    import torch
    cp = catalog.build("bilateral")
    rng = np.random.default_rng(1)
    sides = [(int(a), int(b)) for a, b in rng.integers(37, 900, (10, 2))]
    sides += [(37, 53), (1536, 2560)]
    prms, ins, outs, imgs = _bilateral_batch(cuda, sides, seed=1)
    cp.run_batch(prms, ins, outs)
    torch.cuda.synchronize()
    cp.check()
    _check_bilateral(outs, imgs)
    # unchanged arguments: kernels only; the grids are re-initialized
    _zero(outs)
    cp.run_batch(prms, ins, outs)
    torch.cuda.synchronize()
    cp.check()
    _check_bilateral(outs, imgs)


def test_bilateral_batch_graph_and_new_data(cuda):
    import torch
    cp = catalog.build("bilateral")
    sides = [(300, 500), (64, 64), (700, 333), (1024, 1280)]
    prms, ins, outs, imgs = _bilateral_batch(cuda, sides, seed=2)
    for _ in range(2):
        _zero(outs)
        cp.run_batch(prms, ins, outs, graph=True)
        torch.cuda.synchronize()
        cp.check()
        _check_bilateral(outs, imgs)
    # same pointers, new contents: the graph must read them
    for i, (r, c) in enumerate(sides):
        imgs[i] = OB.make_input(r, c, seed=77 + i)
        ins[i]['input'].copy_(torch.from_numpy(imgs[i]))
    _zero(outs)
    cp.run_batch(prms, ins, outs, graph=True)
    torch.cuda.synchronize()
    cp.check()
    _check_bilateral(outs, imgs)
    # a single-image call in between, then the batch again
    img = OB.make_input(211, 97, seed=5)
    out1 = torch.zeros((1, 211, 97), dtype=torch.float32, device=cuda)
    cp.run_dev({'rows': 211, 'cols': 97},
               {'input': torch.from_numpy(img).to(cuda)},
               {'filtered': out1})
    _zero(outs)
    cp.run_batch(prms, ins, outs, graph=True)
    torch.cuda.synchronize()
    cp.check()
    _check_bilateral(outs, imgs)
    assert np.abs(out1.cpu().numpy() - OB.bilateral(img)).max() <= 1e-5


def _unsharp_ok(img, thr, w, out):
    ref = OU.unsharp(img, thr, w)
    ok = OU.margin(img, thr) > 1e-6
    d = np.abs(out.astype(np.float64) - ref)
    assert d[ok].max() <= 1e-5, d[ok].max()


@pytest.mark.parametrize("graph", [False, True])
def test_unsharp_batch_per_image_params(cuda, graph):
    import torch
    cp = pipelines.unsharp()
    cases = [(1000, 1200, 0.001, 3.0), (37, 53, 0.01, 1.5),
             (1500, 900, 0.0, 2.0), (3, 3, 0.001, 3.0),
             (640, 480, 0.05, 0.5), (1024, 1024, 0.001, 3.0),
             (2048, 1536, 0.002, 4.0)]
    prms, ins, outs, imgs = [], [], [], []
    for i, (R, C, thr, w) in enumerate(cases):
        img = OU.make_input(R, C, seed=40 + i)
        imgs.append(img)
        prms.append({'R': R, 'C': C, 'threshold': thr, 'weight': w})
        ins.append({'img': torch.from_numpy(img).to(cuda)})
        outs.append({'mask': torch.zeros((3, R, C), dtype=torch.float32,
                                         device=cuda)})
    for rep in range(2):
        if rep == 1:      # same pointers, new contents
            for i, (R, C, _, _) in enumerate(cases):
                imgs[i] = OU.make_input(R, C, seed=90 + i)
                ins[i]['img'].copy_(torch.from_numpy(imgs[i]))
        _zero(outs)
        cp.run_batch(prms, ins, outs, graph=graph)
        torch.cuda.synchronize()
        cp.check()
        for (R, C, thr, w), img, o in zip(cases, imgs, outs):
            _unsharp_ok(img, thr, w, o['mask'].cpu().numpy())


def test_harris_batch(cuda):
    import torch
    cp = pipelines.harris()
    sides = [(5, 5), (130, 257), (2048, 2048), (515, 771), (1200, 64)]
    prms, ins, outs, imgs = [], [], [], []
    for i, (r, c) in enumerate(sides):
        img = OH.make_input(r, c, seed=i + 3)
        imgs.append(img)
        prms.append({'R': r - 2, 'C': c - 2})
        ins.append({'img': torch.from_numpy(img).to(cuda)})
        outs.append({'harris': torch.zeros((r, c), dtype=torch.float32,
                                           device=cuda)})
    for graph in (False, False, True):
        _zero(outs)
        cp.run_batch(prms, ins, outs, graph=graph)
        torch.cuda.synchronize()
        cp.check()
        for img, o in zip(imgs, outs):
            ref = OH.harris(img)
            scale = max(np.abs(ref).max(), 1e-30)
            err = np.abs(o['harris'].cpu().numpy() - ref).max() / scale
            assert err <= 1e-5, err


def test_pyramid_batch(cuda):
    import torch
    cp = catalog.build("pyramid")
    sides = [(96, 128), (157, 211), (300, 260), (1100, 900)]
    prms, ins, outs, refs = [], [], [], []
    for i, (R, C) in enumerate(sides):
        img1, img2, mask = OP.make_inputs(R, C, seed=i)
        refs.append(OP.pyramid_blend(img1, img2, mask))
        (x0, x1), (y0, y1) = OP.output_box(R, C)
        prms.append({'R': R, 'C': C})
        ins.append({'img1': torch.from_numpy(img1).to(cuda),
                    'img2': torch.from_numpy(img2).to(cuda),
                    'mask': torch.from_numpy(mask).to(cuda)})
        outs.append({'blend': torch.zeros((3, x1 - x0 + 1, y1 - y0 + 1),
                                          dtype=torch.float32, device=cuda)})
    for graph in (False, True, True):
        _zero(outs)
        cp.run_batch(prms, ins, outs, graph=graph)
        torch.cuda.synchronize()
        cp.check()
        for ref, o in zip(refs, outs):
            err = np.abs(o['blend'].cpu().numpy().astype(np.float64) -
                         ref).max()
            assert err <= 2e-5, err


def test_campipe_batch(cuda):
    """One const table per batch: images share the parameters.  The tables
    are computed from the colour matrices' contents, so the batch never
    replays and has no graph form."""
    import torch
    cp = catalog.build("campipe")
    R, C = 256, 384
    prm = {'C': C, 'R': R, 'colour_temp': 4500.0, 'contrast': 40.0,
           'gamma': 1.8}
    m3 = torch.from_numpy(OC.MATRIX_3200).to(cuda)
    m7 = torch.from_numpy(OC.MATRIX_7000).to(cuda)
    prms, ins, outs, imgs = [], [], [], []
    for i in range(3):
        img = OC.make_input(R, C, seed=20 + i)
        imgs.append(img)
        prms.append(dict(prm))
        ins.append({'img': torch.from_numpy(img).to(cuda),
                    'matrix_3200': m3, 'matrix_7000': m7})
        outs.append({'process': torch.zeros((3, R - 48, C - 64),
                                            dtype=torch.uint8, device=cuda)})
    for rep in range(2):
        _zero(outs)
        cp.run_batch(prms, ins, outs)
        torch.cuda.synchronize()
        cp.check()
        for img, o in zip(imgs, outs):
            ref = OC.campipe(img, 4500.0, 40.0, 1.8)
            assert np.array_equal(o['process'].cpu().numpy(), ref)
    with pytest.raises(PipelineRuntimeError):
        cp.run_batch(prms, ins, outs, graph=True)
    bad = [dict(prm) for _ in range(3)]
    bad[1]['gamma'] = 2.2
    with pytest.raises(PipelineRuntimeError):
        cp.run_batch(bad, ins, outs)
