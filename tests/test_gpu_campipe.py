"""Camera raw pipeline on the GPU, bit-exact against the C restatement
(integer pipeline: every output byte must match)."""

import numpy as np
import pytest

import oracle.campipe as OC
from polymage_b200.apps import catalog

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cp():
    return catalog.build("campipe")


@pytest.mark.parametrize("R,C", [(80, 120), (131, 197), (256, 384),
                                 (1968, 2592)])
def test_campipe_bit_exact_host_abi(cp, R, C):
    img = OC.make_input(R, C, seed=R + C)
    out = np.zeros((3, R - 48, C - 64), np.uint8)
    prm = {'C': C, 'R': R, 'colour_temp': 3700.0, 'contrast': 50.0,
           'gamma': 2.0}
    cp.run_host(prm, {'img': img, 'matrix_3200': OC.MATRIX_3200,
                      'matrix_7000': OC.MATRIX_7000}, {'process': out})
    ref = OC.campipe(img, 3700.0, 50.0, 2.0)
    assert np.array_equal(out, ref), int((out != ref).sum())


def test_campipe_device_abi_params_change(cp, cuda):
    import torch
    R, C = 300, 420
    img = OC.make_input(R, C, seed=7)
    t_img = torch.from_numpy(img).to(cuda)
    m3 = torch.from_numpy(OC.MATRIX_3200).to(cuda)
    m7 = torch.from_numpy(OC.MATRIX_7000).to(cuda)
    for kelvin, contrast, gamma in [(3700.0, 50.0, 2.0), (6000.0, 20.0, 1.6),
                                    (3700.0, 50.0, 2.0)]:
        out = torch.zeros((3, R - 48, C - 64), dtype=torch.uint8,
                          device=cuda)
        prm = {'C': C, 'R': R, 'colour_temp': kelvin, 'contrast': contrast,
               'gamma': gamma}
        cp.run_dev(prm, {'img': t_img, 'matrix_3200': m3,
                         'matrix_7000': m7}, {'process': out})
        torch.cuda.synchronize()
        cp.check()
        ref = OC.campipe(img, kelvin, contrast, gamma)
        assert np.array_equal(out.cpu().numpy(), ref)


def test_campipe_device_abi_host_matrices(cp, cuda):
    """The colour matrices feed only a const table, so the device entry
    takes them in host memory (no read-back per call); a matrix edited in
    place between calls is seen by the next call."""
    import torch
    R, C = 260, 388
    img = OC.make_input(R, C, seed=11)
    t_img = torch.from_numpy(img).to(cuda)
    m3 = torch.from_numpy(OC.MATRIX_3200.copy())
    m7 = torch.from_numpy(OC.MATRIX_7000.copy())
    prm = {'C': C, 'R': R, 'colour_temp': 4500.0, 'contrast': 50.0,
           'gamma': 2.0}
    for step in range(2):
        if step:
            m3[0, 0] += 0.25
        out = torch.zeros((3, R - 48, C - 64), dtype=torch.uint8,
                          device=cuda)
        cp.run_dev(prm, {'img': t_img, 'matrix_3200': m3,
                         'matrix_7000': m7}, {'process': out})
        torch.cuda.synchronize()
        cp.check()
        ref = OC.campipe(img, 4500.0, 50.0, 2.0, m3200=m3.numpy())
        assert np.array_equal(out.cpu().numpy(), ref)


def test_campipe_too_small_refused(cp):
    from polymage_b200.runtime import PipelineRuntimeError
    R, C = 40, 50          # no output domain; the raw is smaller than the
    img = np.zeros((R, C), np.int16)   # ghost zones
    out = np.zeros((1,), np.uint8)
    with pytest.raises((PipelineRuntimeError, ValueError)):
        cp.run_host({'C': C, 'R': R, 'colour_temp': 3700.0,
                     'contrast': 50.0, 'gamma': 2.0},
                    {'img': img, 'matrix_3200': OC.MATRIX_3200,
                     'matrix_7000': OC.MATRIX_7000}, {'process': out})


def test_campipe_matches_reference_spec_fixtures(cp):
    """Byte for byte against the reference's own camera_pipe spec
    evaluated with C semantics (tests/golden/campipe_spec.npz), at two
    parameter sets and an odd image width."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden",
                             "campipe_spec.npz"))
    for n in range(2):
        img = z['img%d' % n]
        R, C = img.shape
        kelvin, contrast, gamma = (float(v) for v in z['params%d' % n])
        out = np.zeros((3, R - 48, C - 64), np.uint8)
        cp.run_host({'C': C, 'R': R, 'colour_temp': kelvin,
                     'contrast': contrast, 'gamma': gamma},
                    {'img': img, 'matrix_3200': OC.MATRIX_3200,
                     'matrix_7000': OC.MATRIX_7000}, {'process': out})
        assert np.array_equal(out, z['out%d' % n])


@pytest.mark.parametrize("R,C", [(1968, 2592), (131, 197), (80, 120)])
def test_campipe_fused_into_one_group_bit_exact(R, C):
    """Option 'fuse_all': every non-const stage in one overlapped-tile
    kernel (one group instead of the greedy grouping's six)."""
    b, kw = catalog._BUILDERS["campipe"]
    kw = dict(kw)
    kw['options'] = tuple(kw['options']) + ('fuse_all',)
    cp = b(**kw).build()
    assert sum(1 for g in cp.module.meta['groups']
               if g['kind'] == 'stencil') == 1
    img = OC.make_input(R, C, seed=R * 3 + C)
    out = np.zeros((3, R - 48, C - 64), np.uint8)
    cp.run_host({'C': C, 'R': R, 'colour_temp': 3700.0, 'contrast': 50.0,
                 'gamma': 2.0}, {'img': img, 'matrix_3200': OC.MATRIX_3200,
                                 'matrix_7000': OC.MATRIX_7000},
                {'process': out})
    assert np.array_equal(out, OC.campipe(img, 3700.0, 50.0, 2.0))
