"""CPU ORACLE — test infrastructure only.

float64 numpy forward and backward pass of the learned-guess network
(x -> SiLU(W1 x + b1) -> SiLU(W2 . + b2) -> W3 . + b3) and of its weighted mean
squared error, to check the CUDA training kernels' gradients.
"""

import numpy as np


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, X):
    W1, b1, W2, b2, W3, b3 = params
    Z1 = X @ W1.T + b1
    A1 = silu(Z1)
    Z2 = A1 @ W2.T + b2
    A2 = silu(Z2)
    Y = A2 @ W3.T + b3
    return Y, (Z1, A1, Z2, A2)


def loss_and_grads(params, X, T, w=None):
    W1, b1, W2, b2, W3, b3 = params
    Y, (Z1, A1, Z2, A2) = forward(params, X)
    B, N = Y.shape
    wi = np.ones(B) if w is None else w
    D = Y - T
    loss = float(np.sum(wi[:, None] * D * D) / (B * N))
    dY = 2.0 * wi[:, None] * D / (B * N)
    gW3 = dY.T @ A2
    gb3 = dY.sum(0)
    dZ2 = (dY @ W3) * silu_grad(Z2)
    gW2 = dZ2.T @ A1
    gb2 = dZ2.sum(0)
    dZ1 = (dZ2 @ W2) * silu_grad(Z1)
    gW1 = dZ1.T @ X
    gb1 = dZ1.sum(0)
    return loss, [gW1, gb1, gW2, gb2, gW3, gb3]
