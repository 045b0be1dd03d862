"""FP64 CPU oracle of the MADE proposal network (test infrastructure only).

Forward and backward of the network the CUDA kernels train (made.cu): h1 = relu(W1 x +
b1), h2 = relu(W2 h1 + b2), z = W3 h2 + b3 with masked weights, mean binary cross
entropy against soft targets, and the autoregressive log-likelihood.  Used to check the
GPU gradients (the weights are the same BF16 values the kernels read).
"""
import numpy as np


def forward(x, wb, b):
    """x [B, n]; wb = masked weights [W1, W2, W3]; returns (h1, h2, z) in float64."""
    h1 = np.maximum(x @ wb[0].T + b[0], 0.0)
    h2 = np.maximum(h1 @ wb[1].T + b[1], 0.0)
    z = h2 @ wb[2].T + b[2]
    return h1, h2, z


def loss_and_grads(x, target, wb, b, masks):
    """Mean-over-batch BCE(sigmoid(z), target) summed over outputs, and its gradients."""
    B = len(x)
    h1, h2, z = forward(x, wb, b)
    s = 1.0 / (1.0 + np.exp(-z))
    loss = float(np.sum(np.logaddexp(0.0, z) - target * z)) / B
    dz = (s - target) / B
    gw3 = (dz.T @ h2) * masks[2]
    gb3 = dz.sum(0)
    dh2 = (dz @ wb[2]) * (h2 > 0)
    gw2 = (dh2.T @ h1) * masks[1]
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ wb[1]) * (h1 > 0)
    gw1 = (dh1.T @ x) * masks[0]
    gb1 = dh1.sum(0)
    return loss, [gw1, gb1, gw2, gb2, gw3, gb3]


def log_q(x, wb, b):
    _, _, z = forward(x, wb, b)
    return np.sum(np.where(x > 0.5, -np.logaddexp(0.0, -z), -np.logaddexp(0.0, z)), axis=1)
