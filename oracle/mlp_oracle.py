"""CPU oracle of the warm-start network (test infrastructure only).

The reference has no learned component, so nothing here restates reference
code; this file states the network's mathematics in numpy so that the CUDA
kernels (features, forward, backward, Adam) can be checked against it:

- ``features``: the 81 per-cell features by brute-force nearest neighbours,
  in float32 arithmetic like the kernel's;
- ``forward`` / ``backward``: the 96 -> 128 -> 128 -> 128 -> 3 GELU network and
  its exact gradient in float64, optionally rounding weights, inputs and
  activations to bf16 where the kernels do;
- ``adam``: one bias-corrected Adam step.

The gradient is pinned by central finite differences (tests/test_oracle_mlp.py).
Only tests and the benchmark's checker import this module.
"""

from __future__ import annotations

import math

import numpy as np

NEIGHBOURS = 16
FEATURES = 5 * NEIGHBOURS + 1
INPUT = 96
HIDDEN = 128
OUTPUTS = 3
OUTPUT_PAD = 8
POSITION_SCALE = 5.0
LENGTH_SCALE = 3.0

# Flat layout shared with the kernels.
W_SHAPES = [(HIDDEN, INPUT), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (OUTPUT_PAD, HIDDEN)]
B_SIZES = [HIDDEN, HIDDEN, HIDDEN, OUTPUT_PAD]
W_OFFSETS = np.cumsum([0] + [a * b for a, b in W_SHAPES]).tolist()
WEIGHTS = W_OFFSETS[-1]
B_OFFSETS = (WEIGHTS + np.cumsum([0] + B_SIZES)).tolist()
PARAMETERS = B_OFFSETS[-1]


def bf16_round(x) -> np.ndarray:
    """float32 values rounded to the nearest bf16 (ties to even), as float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = rounded.astype(np.uint32).view(np.float32)
    nan = np.isnan(a)
    out = out.copy()
    out[nan] = a[nan]
    return out


def bf16_bits(x) -> np.ndarray:
    return (bf16_round(x).view(np.uint32) >> 16).astype(np.uint16)


def from_bf16_bits(bits) -> np.ndarray:
    return (np.asarray(bits, dtype=np.uint32) << 16).view(np.float32)


def unpack(params):
    """Weights (list of 2-D arrays) and biases (list of 1-D arrays) of a flat vector."""
    p = np.asarray(params)
    ws = [p[W_OFFSETS[i]:W_OFFSETS[i + 1]].reshape(W_SHAPES[i]) for i in range(4)]
    bs = [p[B_OFFSETS[i]:B_OFFSETS[i + 1]] for i in range(4)]
    return ws, bs


def init(seed: int = 0) -> np.ndarray:
    """He-uniform weights (fan-in) and zero biases; output rows 3..7 zero."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMETERS, dtype=np.float32)
    for i, (o, k) in enumerate(W_SHAPES):
        limit = math.sqrt(6.0 / k) if i < 3 else math.sqrt(1.0 / k)
        w = rng.uniform(-limit, limit, size=(o, k)).astype(np.float32)
        if i == 0:
            w[:, FEATURES:] = 0.0
        if i == 3:
            w[OUTPUTS:] = 0.0
        p[W_OFFSETS[i]:W_OFFSETS[i + 1]] = w.ravel()
    return p


_ERF = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _ERF(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _ERF(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def forward(params, x, round_like_kernels: bool = False):
    """Outputs (n x 3) and the cache for ``backward``.  With
    ``round_like_kernels`` the weights, the inputs and each hidden activation
    are rounded to bf16 as the kernels round them; sums stay float64."""
    ws, bs = unpack(np.asarray(params, dtype=np.float64))
    r = (lambda a: bf16_round(a).astype(np.float64)) if round_like_kernels else (lambda a: np.asarray(a, np.float64))
    ws = [r(w) for w in ws]
    h = r(x)
    cache = {"h": [h], "z": [], "ws": ws}
    for layer in range(3):
        z = h @ ws[layer].T + bs[layer]
        h = r(gelu(z))
        cache["z"].append(z)
        cache["h"].append(h)
    y = h @ ws[3].T + bs[3]
    return y[:, :OUTPUTS], cache


def backward(cache, output_grad) -> np.ndarray:
    """Gradient of the parameters (flat float64) for d loss / d outputs."""
    ws = cache["ws"]
    g = np.zeros(PARAMETERS, dtype=np.float64)
    dy = np.zeros((output_grad.shape[0], OUTPUT_PAD))
    dy[:, :OUTPUTS] = output_grad
    g[W_OFFSETS[3]:W_OFFSETS[4]] = (dy.T @ cache["h"][3]).ravel()
    g[B_OFFSETS[3]:B_OFFSETS[4]] = dy.sum(axis=0)
    dh = dy @ ws[3]
    for layer in (2, 1, 0):
        dz = dh * gelu_grad(cache["z"][layer])
        g[W_OFFSETS[layer]:W_OFFSETS[layer + 1]] = (dz.T @ cache["h"][layer]).ravel()
        g[B_OFFSETS[layer]:B_OFFSETS[layer + 1]] = dz.sum(axis=0)
        dh = dz @ ws[layer]
    return g


def mse(outputs, targets):
    """Mean squared error over the batch and the three outputs, and its gradient."""
    diff = outputs - targets
    return float(np.mean(diff * diff)), 2.0 * diff / diff.size


def adam(params, grads, m, v, step, lr=1e-3, beta1=0.9, beta2=0.999, epsilon=1e-8):
    m = beta1 * m + (1 - beta1) * grads
    v = beta2 * v + (1 - beta2) * grads * grads
    mhat = m / (1 - beta1 ** step)
    vhat = v / (1 - beta2 ** step)
    return params - lr * mhat / (np.sqrt(vhat) + epsilon), m, v


def features(position_x, position_y, direction_x, direction_y, lengths) -> np.ndarray:
    """The network's input (n x 96, float32) by brute-force nearest centres,
    ties broken by slot, in float32 arithmetic."""
    px = np.asarray(position_x, np.float32)
    py = np.asarray(position_y, np.float32)
    dx_ = np.asarray(direction_x, np.float32)
    dy_ = np.asarray(direction_y, np.float32)
    ln = np.asarray(lengths, np.float32)
    n = px.shape[0]
    norm = np.sqrt(dx_ * dx_ + dy_ * dy_)
    safe = norm > 0
    ax = np.where(safe, dx_ / np.where(safe, norm, 1), np.float32(1)).astype(np.float32)
    ay = np.where(safe, dy_ / np.where(safe, norm, 1), np.float32(0)).astype(np.float32)
    out = np.zeros((n, INPUT), np.float32)
    slots = np.arange(n)
    ps, ls = np.float32(POSITION_SCALE), np.float32(LENGTH_SCALE)
    for s in range(n):
        ddx = (px - px[s]).astype(np.float32)
        ddy = (py - py[s]).astype(np.float32)
        d2 = (ddx * ddx + ddy * ddy).astype(np.float32)
        d2[s] = np.inf
        order = np.lexsort((slots, d2))[:NEIGHBOURS]
        for q, o in enumerate(order):
            if not np.isfinite(d2[o]):
                continue
            out[s, 5 * q + 0] = (ddx[o] * ax[s] + ddy[o] * ay[s]) / ps
            out[s, 5 * q + 1] = (ddy[o] * ax[s] - ddx[o] * ay[s]) / ps
            c = ax[s] * ax[o] + ay[s] * ay[o]
            sn = ax[s] * ay[o] - ay[s] * ax[o]
            if c < 0:
                c, sn = -c, -sn
            out[s, 5 * q + 2] = c
            out[s, 5 * q + 3] = sn
            out[s, 5 * q + 4] = ln[o] / ls
        out[s, FEATURES - 1] = ln[s] / ls
    return out
