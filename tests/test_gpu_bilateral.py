"""Bilateral grid on the GPU against the FP64 restatement.

The grid is a float reduction accumulated with atomics, so its summation
order differs from the oracle's; filtered values are ratios of such sums.
Tolerance: max |gpu - ref| <= 1e-5 (outputs lie in [0, 1))."""

import numpy as np
import pytest

import oracle.bilateral as OB
from polymage_b200.apps import catalog

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cp():
    return catalog.build("bilateral")


@pytest.mark.parametrize("rows,cols", [(37, 53), (64, 64), (200, 331),
                                       (1536, 2560)])
def test_bilateral_host_abi(cp, rows, cols):
    img = OB.make_input(rows, cols, seed=rows + cols)
    out = np.zeros((1, rows, cols), np.float32)
    cp.run_host({'rows': rows, 'cols': cols}, {'input': img},
                {'filtered': out})
    ref = OB.bilateral(img)
    err = np.abs(out.astype(np.float64) - ref).max()
    assert err <= 1e-5, err


def test_bilateral_device_abi_repeatable(cp, cuda):
    import torch
    rows, cols = 300, 500
    img = OB.make_input(rows, cols, seed=3)
    t_in = torch.from_numpy(img).to(cuda)
    ref = OB.bilateral(img)
    for _ in range(3):        # the grid must be re-initialized every call
        out = torch.zeros((1, rows, cols), dtype=torch.float32, device=cuda)
        cp.run_dev({'rows': rows, 'cols': cols}, {'input': t_in},
                   {'filtered': out})
        torch.cuda.synchronize()
        cp.check()
        assert np.abs(out.cpu().numpy() - ref).max() <= 1e-5


def test_bilateral_matches_reference_spec_fixtures(cp):
    """Against the reference's own bilateral_grid spec evaluated in FP64
    (tests/golden/bilateral_spec.npz), same tolerance."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden",
                             "bilateral_spec.npz"))
    for n in range(2):
        img = z['img%d' % n]
        rows, cols = img.shape
        out = np.zeros((1, rows, cols), np.float32)
        cp.run_host({'rows': rows, 'cols': cols}, {'input': img},
                    {'filtered': out})
        assert np.abs(out.astype(np.float64) - z['fp64%d' % n]).max() \
            <= 1e-5
