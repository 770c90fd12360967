"""Float64 numpy reference of the pool-sizing perceptron (test checker).

The same network as the CUDA kernels of edp_learned.cu: y = W3 relu(W2
relu(W1 x + b1) + b2) + b3 with weights rounded to BF16, and the loss
sum(mask (y - t)^2) * scale with its gradient by backpropagation.
"""

import numpy as np


def bf16(a):
    """Round float values to the nearest BF16 (ties to even), as float64."""
    a = np.asarray(a, dtype=np.float32)
    bits = a.view(np.uint32).astype(np.uint64)
    rounded = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(w, x, round_activations=False):
    """Layer values (h1, h2, y); with round_activations the inputs of layers
    1 and 2 are rounded to BF16, as the tensor-core inference does."""
    x = np.asarray(x, dtype=np.float64)
    x1 = bf16(x) if round_activations else x
    h1 = np.maximum(x1 @ bf16(w["W1"]).T + w["b1"], 0.0)
    h1r = bf16(h1) if round_activations else h1
    h2 = np.maximum(h1r @ bf16(w["W2"]).T + w["b2"], 0.0)
    y = h2 @ bf16(w["W3"]).T + w["b3"]
    return h1, h2, y


def loss_and_gradient(w, x, t, mask, scale):
    """(sum of squared masked errors, {name: gradient of loss * scale})."""
    x = np.asarray(x, dtype=np.float64)
    h1, h2, y = forward(w, x)
    e = (y - t) * mask
    dy = 2.0 * e * scale
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    dh2 = (dy @ bf16(w["W3"])) * (h2 > 0)
    g["W2"], g["b2"] = dh2.T @ h1, dh2.sum(0)
    dh1 = (dh2 @ bf16(w["W2"])) * (h1 > 0)
    g["W1"], g["b1"] = dh1.T @ x, dh1.sum(0)
    return float((e * e).sum()), g
