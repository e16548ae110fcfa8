"""The cost model's CUDA kernels: forward outputs and MSE gradients against
the FP64 CPU reference (oracle/mlp.py), and training on the GPU."""

import numpy as np
import pytest

import oracle.mlp as OM
from polymage_b200 import costmodel

pytestmark = pytest.mark.gpu


def _dev(a, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(cuda)


def test_forward_and_gradients_match_fp64(cuda):
    import torch
    L = costmodel.lib()
    D, H, B = 20, 128, 37
    rng = np.random.default_rng(0)
    n = L.pm_mlp_param_count(D, H)
    p = rng.normal(0, 0.15, n).astype(np.float32)
    X = rng.normal(0, 1, (B, D)).astype(np.float32)
    y = rng.normal(0, 1, B).astype(np.float32)
    pd, xd, yd = _dev(p, cuda), _dev(X, cuda), _dev(y, cuda)
    acts = torch.zeros(L.pm_mlp_act_count(B, H), device=cuda)
    work = torch.zeros(L.pm_mlp_work_count(B, H), device=cuda)
    grads = torch.zeros(n, device=cuda)
    loss = torch.zeros(1, device=cuda)
    out = torch.zeros(B, device=cuda)
    s = torch.cuda.current_stream().cuda_stream
    assert L.pm_mlp_forward(pd.data_ptr(), D, H, xd.data_ptr(), B,
                            acts.data_ptr(), out.data_ptr(), s) == 0
    assert L.pm_mlp_backward(pd.data_ptr(), D, H, xd.data_ptr(),
                             yd.data_ptr(), B, acts.data_ptr(),
                             work.data_ptr(), grads.data_ptr(),
                             loss.data_ptr(), s) == 0
    torch.cuda.synchronize()
    ref_out, _ = OM.forward(p, X, D, H)
    ref_loss, ref_g = OM.loss_and_grad(p, X, y, D, H)
    o = out.cpu().numpy()
    assert np.abs(o - ref_out).max() <= 1e-4 * max(1.0, np.abs(ref_out).max())
    assert abs(float(loss.item()) - ref_loss) <= 1e-4 * max(1.0, ref_loss)
    g = grads.cpu().numpy()
    rel = np.abs(g - ref_g).max() / np.abs(ref_g).max()
    assert rel <= 1e-4, rel


def test_training_on_gpu_fits_a_nonlinear_target(cuda):
    rng = np.random.default_rng(1)
    X = rng.normal(0, 1, (256, len(costmodel.FEATURES))).astype(np.float32)
    y = (np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2] -
         0.3 * np.abs(X[:, 3])).astype(np.float32)
    m = costmodel.CostModel(seed=0)
    losses = m.fit(X, y, epochs=800, lr=2e-3)
    assert losses[-1] < 0.1 * losses[0]
    pred = m.predict(X)
    assert np.corrcoef(pred, y)[0, 1] > 0.95
