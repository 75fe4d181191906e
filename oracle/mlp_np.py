"""CPU restatement (numpy, FP64) of the learned cost model's network.

TEST INFRASTRUCTURE ONLY: the checker of pastix_b200/csrc/pgpu_mlp.cu's
forward, backward and Adam kernels; nothing in the shipped package imports
it.  Same packing as the CUDA side: W1[H][F], b1[H], W2[H][H], b2[H], W3[H],
b3; a1 = relu(W1 x + b1), a2 = relu(W2 a1 + b2), y = W3 . a2 + b3; loss =
mean squared error.  Pinned by a finite-difference check in
tests/test_costmodel.py (there is no reference implementation: the
reference's cost models, common/models.c, are polynomials, not networks).
"""
import numpy as np


def unpack(p, F, H):
    o = 0
    W1 = p[o:o + H * F].reshape(H, F); o += H * F
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def count(F, H):
    return H * F + H + H * H + H + H + 1


def forward(p, X, F, H):
    W1, b1, W2, b2, W3, b3 = unpack(p, F, H)
    a1 = np.maximum(X @ W1.T + b1, 0.0)
    a2 = np.maximum(a1 @ W2.T + b2, 0.0)
    return a2 @ W3 + b3, a1, a2


def loss_and_grad(p, X, t, F, H):
    n = X.shape[0]
    W1, b1, W2, b2, W3, b3 = unpack(p, F, H)
    y, a1, a2 = forward(p, X, F, H)
    loss = np.mean((y - t) ** 2)
    dy = 2.0 * (y - t) / n
    d2 = np.outer(dy, W3) * (a2 > 0)
    d1 = (d2 @ W2) * (a1 > 0)
    g = np.concatenate([(d1.T @ X).ravel(), d1.sum(0), (d2.T @ a1).ravel(), d2.sum(0), a2.T @ dy, [dy.sum()]])
    return loss, g


def adam_step(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    bc1, bc2 = 1 - b1 ** step, 1 - b2 ** step
    return p - lr * (m / bc1) / (np.sqrt(v / bc2) + eps), m, v
