"""FP64 reference of the cost model's network (forward pass and MSE
gradients), with the same flat parameter layout as
polymage_b200/csrc/mlp.cu -- test infrastructure only: the GPU kernels'
outputs and gradients are checked against it."""

import numpy as np


def layout(D, H):
    sizes = [("W1", H * D), ("b1", H), ("W2", H * H), ("b2", H),
             ("W3", H * H), ("b3", H), ("W4", H), ("b4", 1)]
    out = {}
    o = 0
    for name, n in sizes:
        out[name] = (o, n)
        o += n
    return out, o


def unpack(p, D, H):
    lay, _ = layout(D, H)
    g = dict((k, p[o:o + n]) for k, (o, n) in lay.items())
    return (g["W1"].reshape(H, D), g["b1"], g["W2"].reshape(H, H), g["b2"],
            g["W3"].reshape(H, H), g["b3"], g["W4"].reshape(1, H), g["b4"])


def forward(p, X, D, H):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(np.asarray(p, np.float64), D, H)
    X = np.asarray(X, np.float64)
    Z1 = X @ W1.T + b1
    A1 = np.maximum(Z1, 0)
    Z2 = A1 @ W2.T + b2
    A2 = np.maximum(Z2, 0)
    Z3 = A2 @ W3.T + b3
    A3 = np.maximum(Z3, 0)
    out = (A3 @ W4.T + b4)[:, 0]
    return out, (X, Z1, A1, Z2, A2, Z3, A3)


def loss_and_grad(p, X, y, D, H):
    """(mean squared error, gradient in the flat layout)."""
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(np.asarray(p, np.float64), D, H)
    out, (X, Z1, A1, Z2, A2, Z3, A3) = forward(p, X, D, H)
    B = X.shape[0]
    d = out - np.asarray(y, np.float64)
    loss = float(np.mean(d * d))
    dout = (2.0 * d / B)[:, None]
    gW4 = dout.T @ A3
    gb4 = dout.sum(0)
    dZ3 = (dout @ W4) * (Z3 > 0)
    gW3 = dZ3.T @ A2
    gb3 = dZ3.sum(0)
    dZ2 = (dZ3 @ W3) * (Z2 > 0)
    gW2 = dZ2.T @ A1
    gb2 = dZ2.sum(0)
    dZ1 = (dZ2 @ W2) * (Z1 > 0)
    gW1 = dZ1.T @ X
    gb1 = dZ1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(),
                        gb3, gW4.ravel(), gb4])
    return loss, g
