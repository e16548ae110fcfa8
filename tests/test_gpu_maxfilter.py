"""Max filter (radius 26) on the GPU against its integer restatement
(oracle/maxfilter.py), built with option 'oob_zero' (the spec's reads of
vert_log outside its domain read 0).  Integer pipeline: bit-exact."""

import numpy as np
import pytest

import oracle.maxfilter as OMF
from polymage_b200.apps import catalog

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("R,C", [(100, 300), (131, 407), (1536, 2560)])
def test_maxfilter_bit_exact(R, C):
    cp = catalog.build("maxfilter")
    img = OMF.make_input(R, C, seed=R + C)
    out = np.zeros((R, C, 3), np.int32)
    cp.run_host({'R': R, 'C': C}, {'img': img}, {'final': out})
    ref = OMF.maxfilter(img)
    assert (ref > 0).any()
    assert np.array_equal(out, ref), int((out != ref).sum())
