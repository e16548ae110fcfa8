"""Non-local means on the GPU against its FP64 restatement
(oracle/nlmeans.py), built with option 'oob_zero' (the spec's reads of
image channel 3 read 0).  Inputs are smooth images with small noise, so
that many patch weights are far from 0.  Tolerance: max |gpu - ref| <=
1e-4 (float32 sums of up to 144 weighted terms; outputs in [0, 1])."""

import numpy as np
import pytest

import oracle.nlmeans as ONL
from polymage_b200.apps import catalog
from polymage_b200.apps.nlmeans import build_nlmeans

pytestmark = pytest.mark.gpu


# (48, 56, 9, 9): offsets and windows of 15, longer than the 12 the build
# was planned for, so the reductions split them over two tiles and combine
# with atomics
@pytest.mark.parametrize("R,C,p,s", [(64, 80, 3, 3), (61, 75, 7, 7),
                                     (48, 56, 9, 9), (256, 256, 7, 7)])
def test_nlmeans(R, C, p, s):
    cp = catalog.build("nlmeans")
    img = ONL.make_input(R, C, seed=R + C)
    out = np.zeros((3, R, C), np.float32)
    cp.run_host({'R': R, 'C': C, 'patch_size': p, 'search_area': s},
                {'img': img}, {'non_local_means': out})
    ref = ONL.nlmeans(img, p, s)
    assert np.abs(out.astype(np.float64) - ref).max() <= 1e-4
