"""Parity of the CUDA pipelines with the CPU oracle, through the C ABI.

Tolerances (float pipelines, FP32 on the GPU vs the FP64 restatement):
  * Harris: max|gpu - ref| / max|ref| <= 1e-5 (elementwise relative error is
    meaningless where det - k*trace^2 cancels), border points exactly 0.
  * Unsharp: max|gpu - ref| <= 1e-5 at every written point whose select
    margin | |img - blur| - threshold | exceeds 1e-6; unwritten points keep
    the caller's values.
"""

import numpy as np
import pytest

import oracle.harris as OH
import oracle.unsharp as OU
from tests import pipelines

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rows,cols", [(5, 5), (37, 53), (64, 64),
                                       (130, 257), (2048, 2048)])
def test_harris_host_abi(rows, cols):
    cp = pipelines.harris()
    img = OH.make_input(rows, cols, seed=rows * 7 + cols)
    out = np.zeros((rows, cols), np.float32)
    cp.run_host({'R': rows - 2, 'C': cols - 2}, {'img': img}, {'harris': out})
    ref = OH.harris(img)
    scale = max(np.abs(ref).max(), 1e-30)
    err = np.abs(out.astype(np.float64) - ref).max() / scale
    assert err <= 1e-5, err
    inner = np.zeros_like(out, dtype=bool)
    inner[2:rows - 1, 2:cols - 1] = True
    assert np.all(out[~inner] == 0)


def test_harris_untouched_border_kept():
    cp = pipelines.harris()
    rows, cols = 40, 60
    img = OH.make_input(rows, cols, seed=3)
    out = np.full((rows, cols), 7.5, np.float32)
    cp.run_host({'R': rows - 2, 'C': cols - 2}, {'img': img}, {'harris': out})
    ref = OH.harris(img, out=np.full((rows, cols), 7.5))
    assert np.all(out[0, :] == 7.5) and np.all(out[:, -2:] == 7.5)
    scale = np.abs(ref[2:rows - 1, 2:cols - 1]).max()
    assert np.abs(out - ref).max() / scale <= 1e-5


def test_harris_device_abi(cuda):
    import torch
    cp = pipelines.harris()
    rows, cols = 515, 771
    img = OH.make_input(rows, cols, seed=11)
    t_in = torch.from_numpy(img).to(cuda)
    t_out = torch.zeros((rows, cols), dtype=torch.float32, device=cuda)
    cp.run_dev({'R': rows - 2, 'C': cols - 2}, {'img': t_in},
               {'harris': t_out})
    torch.cuda.synchronize()
    cp.check()
    ref = OH.harris(img)
    err = np.abs(t_out.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err <= 1e-5


def _unsharp_check(R, C, thr, w, out, img):
    ref = OU.unsharp(img, thr, w)
    m = OU.margin(img, thr)
    ok = m > 1e-6
    d = np.abs(out.astype(np.float64) - ref)
    assert d[ok].max() <= 1e-5, d[ok].max()
    return ref


@pytest.mark.parametrize("R,C", [(3, 3), (37, 53), (100, 300), (257, 130),
                                 (4096, 4096)])
def test_unsharp_host_abi(R, C):
    cp = pipelines.unsharp()
    img = OU.make_input(R, C, seed=R + C)
    out = np.zeros((3, R, C), np.float32)
    cp.run_host({'R': R, 'C': C, 'threshold': 0.001, 'weight': 3.0},
                {'img': img}, {'mask': out})
    _unsharp_check(R, C, 0.001, 3.0, out, img)
    # row R-1 and column C-1 of the output are never written
    assert np.all(out[:, R - 1, :] == 0) and np.all(out[:, :, C - 1] == 0)


def test_unsharp_device_abi_and_graph(cuda):
    import torch
    cp = pipelines.unsharp()
    R, C = 300, 517
    img = OU.make_input(R, C, seed=5)
    prm = {'R': R, 'C': C, 'threshold': 0.01, 'weight': 4.0}
    t_in = torch.from_numpy(img).to(cuda)
    for graph in (False, True, True):
        t_out = torch.zeros((3, R, C), dtype=torch.float32, device=cuda)
        cp.run_dev(prm, {'img': t_in}, {'mask': t_out}, graph=graph)
        torch.cuda.synchronize()
        cp.check()
        _unsharp_check(R, C, 0.01, 4.0, t_out.cpu().numpy(), img)


def test_unsharp_no_tma_path(cuda, monkeypatch):
    """Odd row pitch: the input is not 16-byte aligned per row, so the
    kernel stages it with cooperative loads instead of TMA."""
    cp = pipelines.unsharp()
    R, C = 61, 95          # C+4 = 99 floats per row: not a multiple of 4
    img = OU.make_input(R, C, seed=9)
    out = np.zeros((3, R, C), np.float32)
    cp.run_host({'R': R, 'C': C, 'threshold': 0.001, 'weight': 3.0},
                {'img': img}, {'mask': out})
    _unsharp_check(R, C, 0.001, 3.0, out, img)


def test_bad_parameters_refused():
    from polymage_b200.runtime import PipelineRuntimeError
    cp = pipelines.harris()
    img = np.zeros((10, 10), np.float32)
    out = np.zeros((10, 10), np.float32)
    # R, C larger than the buffers' spec allows is caught by shape checks;
    # negative sizes are refused by the library's validation
    with pytest.raises((PipelineRuntimeError, ValueError)):
        cp.run_host({'R': -5, 'C': 8}, {'img': img[:0].reshape(0)},
                    {'harris': out[:0].reshape(0)})
