"""TEST INFRASTRUCTURE ONLY: CPU FP64 restatement of the warm-start MLP
(pbf_b200/csrc/pbf_mlp.h layout) -- forward pass and backpropagation of
loss = mean (y - target / scale)^2 -- used to check the tensor-core kernels.

The weights are taken at their BF16 values (what the kernels multiply with);
everything else is exact FP64, so differences to the kernels come from their
BF16 activations and FP32 accumulation only.
"""
import numpy as np

W1, W2, W3, W4 = 0, 64 * 16, 64 * 16 + 64 * 64, 64 * 16 + 2 * 64 * 64
B1, B2, B3, B4, FMEAN, FISTD, OSCALE = 0, 64, 128, 192, 193, 209, 225
C = np.sqrt(2.0 / np.pi)
A = 0.044715


def bf16_round(x):
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(C * (z + A * z ** 3)))


def gelu_grad(z):
    t = np.tanh(C * (z + A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C * (1.0 + 3.0 * A * z * z)


def unpack(w32, b32):
    w = bf16_round(w32)
    return (w[W1:W2].reshape(64, 16), w[W2:W3].reshape(64, 64), w[W3:W4].reshape(64, 64), w[W4:],
            np.asarray(b32, np.float64))


def forward(w32, b32, feat):
    """Returns (lambda0, cache) for raw features [n, 12]."""
    w1, w2, w3, w4, b = unpack(w32, b32)
    x = np.zeros((feat.shape[0], 16))
    x[:, :12] = (np.asarray(feat, np.float64) - b[FMEAN:FMEAN + 12]) * b[FISTD:FISTD + 12]
    z1 = x @ w1.T + b[B1:B1 + 64]
    h1 = gelu(z1)
    z2 = h1 @ w2.T + b[B2:B2 + 64]
    h2 = gelu(z2)
    z3 = h2 @ w3.T + b[B3:B3 + 64]
    h3 = gelu(z3)
    y = h3 @ w4 + b[B4]
    return y * b[OSCALE], (x, z1, h1, z2, h2, z3, h3, y)


def gradients(w32, b32, feat, target):
    """(grad weights [9280], grad biases [226] with zeros for the constants, loss)."""
    w1, w2, w3, w4, b = unpack(w32, b32)
    _, (x, z1, h1, z2, h2, z3, h3, y) = forward(w32, b32, feat)
    n = feat.shape[0]
    r = y - np.asarray(target, np.float64) / b[OSCALE]
    loss = np.mean(r * r)
    dy = 2.0 * r / n
    gw = np.zeros(9280)
    gb = np.zeros(226)
    gw[W4:] = h3.T @ dy
    gb[B4] = dy.sum()
    dz3 = np.outer(dy, w4) * gelu_grad(z3)
    gw[W3:W4] = (dz3.T @ h2).ravel()
    gb[B3:B3 + 64] = dz3.sum(0)
    dz2 = (dz3 @ w3) * gelu_grad(z2)
    gw[W2:W3] = (dz2.T @ h1).ravel()
    gb[B2:B2 + 64] = dz2.sum(0)
    dz1 = (dz2 @ w2) * gelu_grad(z1)
    gw[W1:W2] = (dz1.T @ x).ravel()
    gb[B1:B1 + 64] = dz1.sum(0)
    return gw, gb, loss
