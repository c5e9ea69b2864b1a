"""NumPy restatement of the early-termination network -- TEST INFRASTRUCTURE ONLY.

The network has no reference counterpart; this restatement is its oracle. It follows the CUDA
kernels of ``hnsw_engine_b200/csrc/mlp.cu``: 12 -> 64 -> 64 -> 1 with ReLU, forward pass with
BF16-rounded weights (round to nearest even) and float32 biases, mean squared error, gradients by
the chain rule with respect to the (rounded) weights, and Adam with bias correction. The tests check
the CUDA gradients against :func:`gradients` and :func:`gradients` against finite differences.

Parameter vector layout (float32): W1[64][12], b1[64], W2[64][64], b2[64], W3[64], b3[1].
"""

from __future__ import annotations

import numpy as np
from numpy.typing import NDArray

F, H = 12, 64
SIZES = (("W1", H * F), ("b1", H), ("W2", H * H), ("b2", H), ("W3", H), ("b3", 1))
NPARAM = sum(n for _, n in SIZES)


def unpack(p: NDArray) -> dict[str, NDArray]:
    out, o = {}, 0
    for name, n in SIZES:
        out[name] = p[o : o + n]
        o += n
    out["W1"] = out["W1"].reshape(H, F)
    out["W2"] = out["W2"].reshape(H, H)
    return out


def bf16_round(x: NDArray) -> NDArray[np.float32]:
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def forward(p: NDArray, X: NDArray, *, round_weights: bool = True, dtype=np.float32):
    w = unpack(np.asarray(p, dtype=np.float32 if round_weights else dtype))
    rnd = bf16_round if round_weights else (lambda a: a)
    W1, W2, W3 = (rnd(w[k]).astype(dtype) for k in ("W1", "W2", "W3"))
    b1, b2, b3 = (w[k].astype(dtype) for k in ("b1", "b2", "b3"))
    X = X.astype(dtype)
    z1 = X @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    out = h2 @ W3 + b3[0]
    return out, (X, h1, h2, W2, W3)


def loss(p: NDArray, X: NDArray, y: NDArray, **kw) -> float:
    out, _ = forward(p, X, **kw)
    return float(np.mean((out - y) ** 2))


def gradients(p: NDArray, X: NDArray, y: NDArray, *, round_weights: bool = True,
              dtype=np.float32) -> NDArray:
    """d(mean squared error)/d(parameters), in the parameter vector layout."""
    out, (Xc, h1, h2, W2, W3) = forward(p, X, round_weights=round_weights, dtype=dtype)
    B = X.shape[0]
    dO = 2.0 * (out - y.astype(dtype)) / B
    dh2 = (dO[:, None] * W3[None, :]) * (h2 > 0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    g = {
        "W1": dh1.T @ Xc, "b1": dh1.sum(0), "W2": dh2.T @ h1, "b2": dh2.sum(0),
        "W3": h2.T @ dO, "b3": np.array([dO.sum()]),
    }
    return np.concatenate([np.asarray(g[name], dtype=np.float64).ravel() for name, _ in SIZES])


def adam_step(p, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1, c2 = 1 - b1**step, 1 - b2**step
    return p - lr * (m / c1) / (np.sqrt(v / c2) + eps), m, v


def init_params(seed: int = 0) -> NDArray[np.float32]:
    """He-style initialisation (the same as the package's initialiser)."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, n in SIZES:
        if name == "W1":
            parts.append(rng.standard_normal(n) * np.sqrt(2.0 / F))
        elif name == "W2":
            parts.append(rng.standard_normal(n) * np.sqrt(2.0 / H))
        elif name == "W3":
            parts.append(rng.standard_normal(n) * np.sqrt(1.0 / H))
        else:
            parts.append(np.zeros(n))
    return np.concatenate(parts).astype(np.float32)
