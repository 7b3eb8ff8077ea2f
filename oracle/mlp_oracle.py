"""CPU oracle of the learned warm-start network (blockpowerflow_b200/learned.py, csrc/mlp.cu).

TEST INFRASTRUCTURE ONLY (tests/): the forward pass, loss and gradients of the 3-layer MLP in
numpy float64, with the device's BF16 roundings emulated at the same points (operands of every
product, round-to-nearest-even) and FP32 where the device keeps FP32, so that the device's
gradients can be checked term by term.  The network has no counterpart in the reference.

  u = b / ||b||, z1 = W1 u + b1, a1 = lrelu(z1), z2 = W2 a1 + b2, a2 = lrelu(z2),
  y = W3 a2 + b3, loss = (1/p) sum_j ||y_j - t_j||^2 / ||t_j||^2, t_j = x_j / (s ||b_j||).
"""
import numpy as np

LEAK = 0.25


def bf16(x):
    """Round to bfloat16 (nearest, ties to even) and return as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def lrelu(z):
    return np.where(z > 0, z, LEAK * z)


def forward_backward(params, B, X, scale):
    """params: dict of float32 arrays W1 (H x np), b1 (H), W2, b2, W3 (np x H), b3 (np);
    B, X: n x p float64.  Returns (loss, grads dict with the same keys)."""
    W1, b1, W2, b2, W3, b3 = (params[k].astype(np.float64) for k in ("W1", "b1", "W2", "b2", "W3", "b3"))
    H, npad = W1.shape
    n, p = B.shape
    bn = f32(np.linalg.norm(B, axis=0))
    U = np.zeros((p, npad))
    U[:, :n] = bf16(f32(B / bn).T)
    W1b, W2b, W3b = bf16(W1), bf16(W2), bf16(W3)
    Z1 = f32(f32(U @ W1b.T) + b1.reshape(-1))
    A1 = bf16(lrelu(Z1))
    Z2 = f32(f32(A1 @ W2b.T) + b2.reshape(-1))
    A2 = bf16(lrelu(Z2))
    Yp = f32(A2 @ W3b.T)                                   # p x np, without b3
    y = Yp[:, :n] + b3.reshape(-1)[:n]
    T = (X / (scale * bn)).T                               # p x n
    tn = f32(np.sum(T * T, axis=1))
    w = 1.0 / (p * tn)
    D = y - T
    loss = float(np.sum(w[:, None] * D * D))
    G = np.zeros((p, npad))
    G[:, :n] = f32(2.0 * w[:, None] * D)
    Gb = bf16(G)
    g = {}
    g["b3"] = G.sum(axis=0)
    g["W3"] = Gb.T @ A2
    dA2 = f32(Gb @ W3b)
    dZ2 = f32(dA2 * np.where(Z2 > 0, 1.0, LEAK))
    g["b2"] = dZ2.sum(axis=0)
    dZ2b = bf16(dZ2)
    g["W2"] = dZ2b.T @ A1
    dA1 = f32(dZ2b @ W2b)
    dZ1 = f32(dA1 * np.where(Z1 > 0, 1.0, LEAK))
    g["b1"] = dZ1.sum(axis=0)
    g["W1"] = bf16(dZ1).T @ U
    return loss, g


def forward(params, B, scale):
    """Warm starts x0 = s ||b|| (W3 a2 + b3) (n x p)."""
    W1, b1, W2, b2, W3, b3 = (params[k].astype(np.float64) for k in ("W1", "b1", "W2", "b2", "W3", "b3"))
    n, p = B.shape
    npad = W1.shape[1]
    bn = f32(np.linalg.norm(B, axis=0))
    U = np.zeros((p, npad))
    U[:, :n] = bf16(f32(B / bn).T)
    A1 = bf16(lrelu(f32(f32(U @ bf16(W1).T) + b1.reshape(-1))))
    A2 = bf16(lrelu(f32(f32(A1 @ bf16(W2).T) + b2.reshape(-1))))
    y = f32(A2 @ bf16(W3).T)[:, :n] + b3.reshape(-1)[:n]
    return (scale * bn * y.T)
