"""CPU restatement of the surrogate network's forward and backward passes
(numpy, float64 arithmetic on bf16-rounded operands) -- test infrastructure
only; the product network is pofd_affine_b200/csrc/surrogate.cu.

Rounding points follow the product: inputs, weights, activations and the
back-propagated pre-activation gradients are rounded to bfloat16
(round-to-nearest-even); products accumulate in float64 here (FP32 on the
tensor cores), so agreement is to FP32/bf16 accuracy, not bitwise.
"""
import numpy as np

IN_PAD = 16


def bf16(a):
    """Round float32 values to the nearest bfloat16 (ties to even)."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def unpack(params, H):
    W1 = params[0].reshape(H, IN_PAD)
    W2 = params[2].reshape(H, H)
    W3 = params[4].reshape(H, H)
    return W1, params[1], W2, params[3], W3, params[5], params[6], params[7][0]


def standardise(theta, idx, mu, W):
    """Network inputs x = W (theta[idx] - mu) in float32 (the product's
    k_pack_inputs), W the 16 x 16 input transform."""
    x = np.zeros((theta.shape[0], IN_PAD), np.float32)
    d = np.zeros((theta.shape[0], IN_PAD), np.float32)
    for k, p in enumerate(idx):
        d[:, k] = theta[:, p].astype(np.float32) - np.float32(mu[k])
    x[:, :] = d @ np.asarray(W, np.float32).T
    return x


def forward(params, H, x):
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(params, H)
    xb = bf16(x)
    z1 = xb @ bf16(W1).T + b1
    h1 = bf16(silu(z1))
    z2 = h1 @ bf16(W2).T + b2
    h2 = bf16(silu(z2))
    z3 = h2 @ bf16(W3).T + b3
    h3 = bf16(silu(z3))
    y = h3 @ w4.astype(np.float64) + b4
    return y, (xb, z1, h1, z2, h2, z3, h3)


def gradients(params, H, x, t):
    """Mean-square-loss gradients of the 8 tensors."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(params, H)
    y, (xb, z1, h1, z2, h2, z3, h3) = forward(params, H, x)
    M = x.shape[0]
    dy = 2.0 * (y - t) / M
    dz3 = bf16(dy[:, None] * w4[None, :] * dsilu(z3))
    g3 = dz3.T @ h2
    dz2 = bf16((dz3 @ bf16(W3)) * dsilu(z2))
    g2 = dz2.T @ h1
    dz1 = bf16((dz2 @ bf16(W2)) * dsilu(z1))
    g1 = dz1.T @ xb
    loss = float(np.mean((y - t) ** 2))
    return [g1.ravel(), dz1.sum(0), g2.ravel(), dz2.sum(0), g3.ravel(),
            dz3.sum(0), (dy[:, None] * h3).sum(0), np.array([dy.sum()])], loss
