"""Laplacian pyramid blending on the GPU against the FP64 restatement.
Tolerance: max |gpu - ref| <= 2e-5 (inputs in [0, 1), FP32 through the
pyramid levels)."""

import numpy as np
import pytest

import oracle.pyramid as OP
from polymage_b200.apps import catalog

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cp():
    return catalog.build("pyramid")


@pytest.mark.parametrize("R,C", [(96, 128), (157, 211), (2108, 2108)])
def test_pyramid_host_abi(cp, R, C):
    img1, img2, mask = OP.make_inputs(R, C, seed=R)
    (x0, x1), (y0, y1) = OP.output_box(R, C)
    out = np.zeros((3, x1 - x0 + 1, y1 - y0 + 1), np.float32)
    cp.run_host({'R': R, 'C': C}, {'img1': img1, 'img2': img2,
                                   'mask': mask}, {'blend': out})
    ref = OP.pyramid_blend(img1, img2, mask)
    err = np.abs(out.astype(np.float64) - ref).max()
    assert err <= 2e-5, err


def test_pyramid_matches_reference_spec_fixtures(cp):
    """Against the reference's own pyramid_blending spec evaluated in FP64
    (tests/golden/pyramid_spec.npz), same tolerance."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden",
                             "pyramid_spec.npz"))
    for n in range(2):
        R, C = (int(v) for v in z['shape%d' % n])
        img1, img2, mask = OP.make_inputs(R, C, seed=R)
        ref = z['fp64%d' % n]
        out = np.zeros(ref.shape, np.float32)
        cp.run_host({'R': R, 'C': C}, {'img1': img1, 'img2': img2,
                                       'mask': mask}, {'blend': out})
        assert np.abs(out.astype(np.float64) - ref).max() <= 2e-5
