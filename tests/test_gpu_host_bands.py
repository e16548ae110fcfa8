"""The reference ABI (host buffers) on pinned memory: a single-group
pipeline then runs in row bands with the input copy, the kernel and the
output copy of different bands overlapping.  Results must equal the
oracle's as in the single-call parity tests (unsharp: max |gpu - ref| <=
1e-5 where the select margin exceeds 1e-6), and output points the pipeline
does not write must keep the caller's values."""

import numpy as np
import pytest

import oracle.unsharp as OU
from tests import pipelines

pytestmark = pytest.mark.gpu


def _pinned(shape, dtype, fill=0.0):
    import torch
    t = torch.empty(shape, dtype=dtype, pin_memory=True)
    t.fill_(fill)
    return t


@pytest.mark.parametrize("R,C", [(1000, 1500), (1531, 877), (4096, 4096)])
def test_unsharp_pinned_host_buffers(R, C, cuda):
    import torch
    cp = pipelines.unsharp()
    img = OU.make_input(R, C, seed=R ^ C)
    t_in = _pinned(img.shape, torch.float32)
    t_in.numpy()[...] = img
    t_out = _pinned((3, R, C), torch.float32, fill=7.5)
    out = t_out.numpy()
    for rep in range(2):
        if rep:
            out[...] = 7.5
        cp.run_host({'R': R, 'C': C, 'threshold': 0.001, 'weight': 3.0},
                    {'img': t_in.numpy()}, {'mask': out})
        ref = OU.unsharp(img, 0.001, 3.0, out=np.full((3, R, C), 7.5))
        ok = OU.margin(img, 0.001) > 1e-6
        d = np.abs(out.astype(np.float64) - ref)
        assert d[ok].max() <= 1e-5, d[ok].max()
        # the last domain row and column are never written
        assert np.all(out[:, R - 1, :] == 7.5) and np.all(out[:, :, C - 1] == 7.5)
