"""Float64 restatement of the surrogate network (TEST INFRASTRUCTURE ONLY).

The surrogate has no counterpart in the reference: this file is the CPU
checker for the library's tensor-core forward and backward kernels
(nanoxgen_b200/csrc/surrogate.cu).  It evaluates the same augmented network

    x  = [(features - offset) * scale, 1, 0 x 7]                 (16)
    h1 = relu(W1a x);  h2 = relu(W2a [h1, 1, 0 x 15]);  h3 = relu(W3a [h2, 1, 0 x 15])
    y  = (W4a [h3, 1, 0 x 15])[:2];  outputs = y * output_scale + output_offset

in float64.  With ``emulate=True`` every value the device stores in BF16
(weights, inputs, activations, the back-propagated dZ) is rounded to BF16
first, so the remaining difference is the device's FP32 accumulation.
Loss: mean over samples of the squared error of the normalised outputs.
"""
from __future__ import annotations

import numpy as np

P1, P2 = 0, 64 * 16
P3 = P2 + 64 * 80
P4 = P3 + 64 * 80
PARAMETERS = P4 + 16 * 80


def bf16(a) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), as float64."""
    u = np.asarray(a, np.float32).astype(np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def split(params):
    p = np.asarray(params, np.float64)
    return (p[P1:P2].reshape(64, 16), p[P2:P3].reshape(64, 80), p[P3:P4].reshape(64, 80),
            p[P4:PARAMETERS].reshape(16, 80))


def _augment(h):
    n = h.shape[0]
    return np.concatenate([h, np.ones((n, 1)), np.zeros((n, 15))], 1)


def network_input(features, input_offset, input_scale):
    """The 16-column input rows, normalised in float32 as the device does."""
    f = np.asarray(features, np.float32)
    x = (f - np.asarray(input_offset, np.float32)) * np.asarray(input_scale, np.float32)
    n = x.shape[0]
    return np.concatenate([x.astype(np.float64), np.ones((n, 1)), np.zeros((n, 7))], 1)


def forward(params, features, header, emulate=True):
    """(outputs (n, 2), cache) for raw features (n, 8)."""
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    W1, W2, W3, W4 = (r(w) for w in split(params))
    X = r(network_input(features, header["input_offset"], header["input_scale"]))
    h1 = r(np.maximum(X @ W1.T, 0.0))
    H1 = _augment(h1)
    h2 = r(np.maximum(H1 @ W2.T, 0.0))
    H2 = _augment(h2)
    h3 = r(np.maximum(H2 @ W3.T, 0.0))
    H3 = _augment(h3)
    y = (H3 @ W4.T)[:, :2]
    out = y * np.asarray(header["output_scale"], np.float64) + np.asarray(header["output_offset"], np.float64)
    return out, dict(X=X, H1=H1, H2=H2, H3=H3, y=y, W=(W1, W2, W3, W4))


def loss_and_gradients(params, features, targets, header, emulate=True):
    """(mean loss, gradient over all parameters in the device layout)."""
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    _, c = forward(params, features, header, emulate)
    W1, W2, W3, W4 = c["W"]
    n = c["y"].shape[0]
    tt = np.asarray(targets, np.float32)
    t = ((tt - np.asarray(header["output_offset"], np.float32)) / np.asarray(header["output_scale"], np.float32))
    t = t.astype(np.float64)
    diff = c["y"] - t
    loss = float((diff ** 2).sum(1).mean())
    dZ4 = np.zeros((n, 16))
    dZ4[:, :2] = r(2.0 * diff / n)
    dW4 = dZ4.T @ c["H3"]
    dZ3 = r((dZ4 @ W4)[:, :64] * (c["H3"][:, :64] > 0))
    dW3 = dZ3.T @ c["H2"]
    dZ2 = r((dZ3 @ W3)[:, :64] * (c["H2"][:, :64] > 0))
    dW2 = dZ2.T @ c["H1"]
    dZ1 = r((dZ2 @ W2)[:, :64] * (c["H1"][:, :64] > 0))
    dW1 = dZ1.T @ c["X"]
    return loss, np.concatenate([dW1.ravel(), dW2.ravel(), dW3.ravel(), dW4.ravel()])


def used_mask() -> np.ndarray:
    """Parameters that exist in the network (weights and biases)."""
    m = np.zeros(PARAMETERS, bool)
    m[P1:P2] = (np.arange(16)[None, :] <= 8).repeat(64, 0).ravel()
    cols = np.arange(80)[None, :] <= 64
    m[P2:P3] = cols.repeat(64, 0).ravel()
    m[P3:P4] = cols.repeat(64, 0).ravel()
    w4 = np.zeros((16, 80), bool)
    w4[:2] = cols
    m[P4:] = w4.ravel()
    return m
