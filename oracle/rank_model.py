"""CPU oracle for the learned rank model's root network (TEST INFRASTRUCTURE).

The learned-start query has no counterpart in the reference; its oracle is a
float64 restatement of the root network 1 -> 32 -> 32 -> 1 (ReLU, mean squared
error on rank / n), used to check the gradients the GPU training kernels
compute.  Parameter order: w1[32], b1[32], w2[32][32] (out, in), b2[32],
w3[32], b3.
"""
import numpy as np

H = 32


def unpack(flat):
    flat = np.asarray(flat, dtype=np.float64)
    w1, b1 = flat[:H], flat[H:2 * H]
    w2 = flat[2 * H:2 * H + H * H].reshape(H, H)
    b2 = flat[2 * H + H * H:3 * H + H * H]
    w3 = flat[3 * H + H * H:4 * H + H * H]
    b3 = flat[4 * H + H * H]
    return w1, b1, w2, b2, w3, b3


def forward(flat, x):
    w1, b1, w2, b2, w3, b3 = unpack(flat)
    z1 = np.outer(x, w1) + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ w2.T + b2
    h2 = np.maximum(z2, 0)
    return h2 @ w3 + b3, (z1, h1, z2, h2)


def loss_and_grad(flat, x, y):
    """Mean squared error and its gradient, float64."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    w1, b1, w2, b2, w3, b3 = unpack(flat)
    out, (z1, h1, z2, h2) = forward(flat, x)
    m = len(x)
    diff = out - y
    loss = float(np.mean(diff ** 2))
    dout = 2 * diff / m
    g_w3 = h2.T @ dout
    g_b3 = dout.sum()
    dz2 = np.outer(dout, w3) * (z2 > 0)
    g_w2 = dz2.T @ h1
    g_b2 = dz2.sum(0)
    dz1 = (dz2 @ w2) * (z1 > 0)
    g_w1 = dz1.T @ x
    g_b1 = dz1.sum(0)
    grad = np.concatenate([g_w1, g_b1, g_w2.reshape(-1), g_b2, g_w3, [g_b3]])
    return loss, grad
