"""ORACLE / TEST INFRASTRUCTURE ONLY -- numpy restatement of the preconditioner
network of simple-cpsd_b200/csrc/mlp.cuh, used to check the GPU forward and
backward kernels (gradient check).

y = W4 h3 + b4, h_k = tanh(W_k h_{k-1} + b_k), h_0 = x (4 -> 64 -> 64 -> 64 -> 1).
The forward uses BF16-rounded weights (round to nearest even) and FP32
biases, exactly like the GPU inference path; gradients are taken with
respect to the FP32 master parameters through that rounding
(straight-through), with the MSE loss mean((y - t)^2).  Arithmetic is float64
here, so the GPU's FP32 results must agree to FP32 rounding.
"""
from __future__ import annotations

import numpy as np

NIN, NH = 4, 64
W1 = 0
B1 = W1 + NH * NIN
W2 = B1 + NH
B2 = W2 + NH * NH
W3 = B2 + NH
B3 = W3 + NH * NH
W4 = B3 + NH
B4 = W4 + NH
NPARAMS = B4 + 1


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even) and back to float32."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray):
    q = bf16(p).astype(np.float64)
    p = p.astype(np.float64)
    return (q[W1:B1].reshape(NH, NIN), p[B1:W2], q[W2:B2].reshape(NH, NH), p[B2:W3],
            q[W3:B3].reshape(NH, NH), p[B3:W4], q[W4:B4], p[B4])


def forward(p: np.ndarray, X: np.ndarray):
    w1, b1, w2, b2, w3, b3, w4, b4 = unpack(p)
    X = X.astype(np.float64)
    h1 = np.tanh(X @ w1.T + b1)
    h2 = np.tanh(h1 @ w2.T + b2)
    h3 = np.tanh(h2 @ w3.T + b3)
    y = h3 @ w4 + b4
    return y, (X, h1, h2, h3)


def loss_and_grad(p: np.ndarray, X: np.ndarray, T: np.ndarray):
    w1, b1, w2, b2, w3, b3, w4, b4 = unpack(p)
    y, (x, h1, h2, h3) = forward(p, X)
    n = X.shape[0]
    r = y - T.astype(np.float64)
    loss = float(np.mean(r * r))
    dy = 2.0 * r / n
    g = np.zeros(NPARAMS)
    g[W4:B4] = dy @ h3
    g[B4] = dy.sum()
    d3 = np.outer(dy, w4) * (1 - h3 * h3)
    g[W3:B3] = (d3.T @ h2).reshape(-1)
    g[B3:W4] = d3.sum(0)
    d2 = (d3 @ w3) * (1 - h2 * h2)
    g[W2:B2] = (d2.T @ h1).reshape(-1)
    g[B2:W3] = d2.sum(0)
    d1 = (d2 @ w2) * (1 - h1 * h1)
    g[W1:B1] = (d1.T @ x).reshape(-1)
    g[B1:W2] = d1.sum(0)
    return loss, g
