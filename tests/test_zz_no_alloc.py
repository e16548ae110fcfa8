"""pm_mlp_forward_static (activations in a fixed array of the cost-model
library, no allocation) against pm_mlp_forward (caller-provided activation
buffer), through the C ABI.

Both run the same kernels in the same order, so the outputs agree to
max |static - buffered| <= 1e-6 * max(1, max |buffered|); the static
entry's output is also checked directly against the FP64 forward pass of
oracle/mlp.py at the cost-model tests' tolerance (1e-4 relative to the
largest output).  Requests beyond
the array's 196,864 floats (B * (6H + 1)) return 1 and leave the output
untouched.
"""

import ctypes

import numpy as np
import pytest

from polymage_b200 import costmodel

pytestmark = pytest.mark.gpu

STATIC_FLOATS = 196864


def _static_entry(L):
    f = L.pm_mlp_forward_static
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def test_static_forward_matches_buffered_forward(cuda):
    import torch
    L = costmodel.lib()
    fwd_static = _static_entry(L)
    D, H, B = 20, 128, 200
    assert B * (6 * H + 1) <= STATIC_FLOATS
    rng = np.random.default_rng(5)
    n = L.pm_mlp_param_count(D, H)
    p = torch.from_numpy(rng.normal(0, 0.15, n).astype(np.float32)).to(cuda)
    X = torch.from_numpy(rng.normal(0, 1, (B, D)).astype(np.float32)).to(cuda)
    s = torch.cuda.current_stream().cuda_stream
    acts = torch.zeros(L.pm_mlp_act_count(B, H), device=cuda)
    ref = torch.zeros(B, device=cuda)
    assert L.pm_mlp_forward(p.data_ptr(), D, H, X.data_ptr(), B,
                            acts.data_ptr(), ref.data_ptr(), s) == 0
    torch.cuda.synchronize()
    r = ref.cpu().numpy()
    tol = 1e-6 * max(1.0, float(np.abs(r).max()))
    import oracle.mlp as OM
    exact, _ = OM.forward(p.cpu().numpy(), X.cpu().numpy(), D, H)
    for _ in range(2):                       # two calls in a row
        out = torch.full((B,), -7.0, device=cuda)
        assert fwd_static(p.data_ptr(), D, H, X.data_ptr(), B,
                          out.data_ptr(), s) == 0
        torch.cuda.synchronize()
        o = out.cpu().numpy()
        assert np.abs(o - r).max() <= tol
        assert np.abs(o - exact).max() <= 1e-4 * max(1.0,
                                                      np.abs(exact).max())


def test_static_forward_rejects_oversized_request(cuda):
    import torch
    L = costmodel.lib()
    fwd_static = _static_entry(L)
    D, H = 20, 128
    B = STATIC_FLOATS // (6 * H + 1) + 1          # one row too many
    n = L.pm_mlp_param_count(D, H)
    p = torch.zeros(n, device=cuda)
    X = torch.zeros((B, D), device=cuda)
    out = torch.full((B,), -7.0, device=cuda)
    s = torch.cuda.current_stream().cuda_stream
    assert fwd_static(p.data_ptr(), D, H, X.data_ptr(), B, out.data_ptr(),
                      s) == 1
    torch.cuda.synchronize()
    assert bool((out == -7.0).all())
