"""Eight-level pyramid blending with clamped borders on the GPU against the
FP64 restatement of the same spec (oracle.pyramid.pyramid_blend_clamped).
Tolerance: max |gpu - ref| <= 2e-5 (inputs in [0, 1), FP32 through the
levels).  Sizes include sides below 2^7, where the coarsest levels are a
single row or column and every stencil tap is clamped."""

import numpy as np
import pytest

import oracle.pyramid as OP
from polymage_b200.apps import catalog

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cp():
    return catalog.build("pyramid8")


@pytest.mark.parametrize("R,C", [(37, 53), (256, 300), (513, 1025),
                                 (2048, 2048)])
def test_pyramid8_host_abi(cp, R, C):
    img1, img2, mask = OP.make_inputs(R, C, seed=R + C)
    out = np.zeros((3, R, C), np.float32)
    cp.run_host({'R': R, 'C': C}, {'img1': img1, 'img2': img2,
                                   'mask': mask}, {'blend': out})
    ref = OP.pyramid_blend_clamped(img1, img2, mask, L=8)
    err = np.abs(out.astype(np.float64) - ref).max()
    assert err <= 2e-5, err


def test_pyramid8_batch_graph(cp, cuda):
    import torch
    sides = [(37, 53), (130, 257), (700, 333), (1100, 900)]
    prms, ins, outs, refs = [], [], [], []
    for i, (R, C) in enumerate(sides):
        img1, img2, mask = OP.make_inputs(R, C, seed=50 + i)
        refs.append(OP.pyramid_blend_clamped(img1, img2, mask, L=8))
        prms.append({'R': R, 'C': C})
        ins.append({'img1': torch.from_numpy(img1).to(cuda),
                    'img2': torch.from_numpy(img2).to(cuda),
                    'mask': torch.from_numpy(mask).to(cuda)})
        outs.append({'blend': torch.zeros((3, R, C), dtype=torch.float32,
                                          device=cuda)})
    for graph in (False, True, True):
        for o in outs:
            o['blend'].zero_()
        cp.run_batch(prms, ins, outs, graph=graph)
        torch.cuda.synchronize()
        cp.check()
        for ref, o in zip(refs, outs):
            err = np.abs(o['blend'].cpu().numpy().astype(np.float64) -
                         ref).max()
            assert err <= 2e-5, err


@pytest.mark.parametrize("graph", [False, True])
def test_pyramid8_joins_the_callers_stream(cp, cuda, graph):
    """The groups run on several streams; the call's stream must follow
    all of them: a copy queued on that stream right after the call, with
    no device synchronization in between, sees the finished output."""
    import torch
    R, C = 1500, 1700
    img1, img2, mask = OP.make_inputs(R, C, seed=9)
    ref = OP.pyramid_blend_clamped(img1, img2, mask, L=8)
    ins = {'img1': torch.from_numpy(img1).to(cuda),
           'img2': torch.from_numpy(img2).to(cuda),
           'mask': torch.from_numpy(mask).to(cuda)}
    side = torch.cuda.Stream(cuda)
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        for _ in range(3):
            out = torch.zeros((3, R, C), dtype=torch.float32, device=cuda)
            cp.run_dev({'R': R, 'C': C}, ins, {'blend': out}, graph=graph)
            snap = out.clone()
        side.synchronize()
    cp.check()
    err = np.abs(snap.cpu().numpy().astype(np.float64) - ref).max()
    assert err <= 2e-5, err
