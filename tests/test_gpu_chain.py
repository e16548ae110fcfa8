"""GPU parity of chain builds (option ``chain``): runs of consecutive small
stencil groups execute as one launch whose phases are separated by grid
barriers.  Each build is checked against the same oracle and tolerance as
its per-group build (tests/test_gpu_widening.py, test_gpu_pyramid8.py,
test_gpu_laplacian.py), through the host-buffer ABI, the device entry and
its CUDA graph, and the per-group batch path the chain build keeps."""

import numpy as np
import pytest

import oracle.interpolate as OI
import oracle.multigrid as OM
import oracle.pyramid as OP
from polymage_b200.apps import catalog

pytestmark = pytest.mark.gpu

_built = {}


def _chain(name):
    if name not in _built:
        cp = catalog.variant(name, ('chain',)).build()
        assert cp.module.meta.get('chains'), "no chain formed"
        _built[name] = cp
    return _built[name]


def _f64_close(out, ref):
    err = np.abs(out - ref).max()
    assert err <= 1e-10 * max(1.0, np.abs(ref).max()), err


@pytest.mark.parametrize("name,n", [("vcycle", 31), ("vcycle", 20),
                                    ("wcycle", 31), ("wcycle", 13)])
def test_chain_multigrid(name, n):
    cp = _chain(name)
    kw = dict(catalog._BUILDERS[name][1])
    V, F = OM.make_input(n, L=kw['L'], seed=n)
    N = V.shape[0] - 2
    out = np.zeros((N + 2, N + 2), np.float64)
    cp.run_host({'n': n}, {'V_': V, 'F_': F}, {cp.outputs[0].name: out})
    ref = OM.v_cycle(V, F, n, L=kw['L'], nu1=kw['nu1'], nu2=kw['nu2'],
                     nuc=kw['nuc'], gamma=kw.get('gamma', 1))
    _f64_close(out, ref)


@pytest.mark.parametrize("R,C", [(37, 53), (513, 1025), (2048, 2048)])
def test_chain_pyramid8(R, C):
    cp = _chain("pyramid8")
    img1, img2, mask = OP.make_inputs(R, C, seed=R + C)
    out = np.zeros((3, R, C), np.float32)
    cp.run_host({'R': R, 'C': C}, {'img1': img1, 'img2': img2,
                                   'mask': mask}, {'blend': out})
    ref = OP.pyramid_blend_clamped(img1, img2, mask, L=8)
    assert np.abs(out.astype(np.float64) - ref).max() <= 2e-5


@pytest.mark.parametrize("R,C", [(211, 157), (2048, 2048)])
def test_chain_interpolate(R, C):
    cp = _chain("interpolate")
    img = OI.make_input(R, C, seed=R + C)
    out = np.zeros((3, R, C), np.float32)
    cp.run_host({'R': R, 'C': C}, {'img': img}, {'interpolate': out})
    assert np.abs(out.astype(np.float64) - OI.interpolate(img)).max() <= 1e-5


def test_chain_laplacian_matches_reference_fixtures():
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden",
                             "laplacian.npz"))
    cp = _chain("laplacian")
    for k in range(2):
        frame = z['frame%d' % k]
        H, W, _ = frame.shape
        out = np.zeros((H, W, 3), np.uint8)
        cp.run_host({'R': H + 92, 'C': W + 92, 'alpha': float(z['alpha']),
                     'beta': float(z['beta'])},
                    {'img_colour': np.ascontiguousarray(frame)},
                    {'laplacian': out})
        d = np.abs(out.astype(np.int16) - z['out%d' % k].astype(np.int16))
        assert d.max() <= 1 and (d > 0).mean() <= 1e-3


def test_chain_graph_replays_and_batch(cuda):
    """The device entry and its CUDA graph (replayed with new input
    contents) agree with the host entry; a batch of two images, which runs
    the per-group kernels, agrees with the oracle too."""
    import torch
    cp = _chain("pyramid8")
    R, C = 300, 420
    for seed in (5, 6):
        img1, img2, mask = OP.make_inputs(R, C, seed=seed)
        ref = OP.pyramid_blend_clamped(img1, img2, mask, L=8)
        d = {'img1': torch.from_numpy(img1).to(cuda),
             'img2': torch.from_numpy(img2).to(cuda),
             'mask': torch.from_numpy(mask).to(cuda)}
        for graph in (False, True, True):
            o = torch.zeros((3, R, C), dtype=torch.float32, device=cuda)
            cp.run_dev({'R': R, 'C': C}, d, {'blend': o}, graph=graph)
            torch.cuda.synchronize()
            cp.check()
            got = o.cpu().numpy().astype(np.float64)
            assert np.abs(got - ref).max() <= 2e-5
    sizes = [(R, C), (77, 130)]
    params, ins, bouts, refs = [], [], [], []
    for (r, c), s in zip(sizes, (8, 9)):
        img1, img2, mask = OP.make_inputs(r, c, seed=s)
        refs.append(OP.pyramid_blend_clamped(img1, img2, mask, L=8))
        params.append({'R': r, 'C': c})
        ins.append({'img1': torch.from_numpy(img1).to(cuda),
                    'img2': torch.from_numpy(img2).to(cuda),
                    'mask': torch.from_numpy(mask).to(cuda)})
        bouts.append({'blend': torch.zeros((3, r, c), dtype=torch.float32,
                                           device=cuda)})
    cp.run_batch(params, ins, bouts)
    torch.cuda.synchronize()
    cp.check()
    for o, ref in zip(bouts, refs):
        got = o['blend'].cpu().numpy().astype(np.float64)
        assert np.abs(got - ref).max() <= 2e-5
