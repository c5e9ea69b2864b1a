"""Seeded synthetic workloads with the shapes and value ranges of the reference's benchmark data.

The reference benchmarks on ANN-Benchmarks files (SIFT-128, Fashion-MNIST-784, GloVe-100,
``docs/DATASETS.md``) that are not available offline. These generators stand in for them with the
same dimensions, dtypes and value ranges. Every generator is a pure function of its seed, so a
graph built once by the reference's host build can be re-attached to vectors regenerated anywhere.

* :func:`mixture` -- SIFT-like integer descriptors in ``[0, 255]``: a 100-component Gaussian
  mixture whose centres (uniform in ``[0, 128]``) are shared by data and queries, sigma 20 per
  coordinate, rounded and clipped. Data uses seed 0, queries seed 1, training queries seed 2.
  (The reference's ``synthetic.clustered`` draws centres per seed and cannot express "queries from
  the same mixture", ``src/hnsw_engine/synthetic.py:29-42``.)
* :func:`student_t_unit` -- GloVe-like angular data: Student-t (nu = 3) coordinates, each row
  L2-normalised in float64.
* :func:`image_like` -- Fashion-MNIST-like 28 x 28 uint8-valued images: 70 % zeros, non-zeros
  uniform in 1..255, smoothed with a 3 x 3 box filter and rounded.
"""

from __future__ import annotations

import numpy as np
from numpy.typing import NDArray

MIXTURE_COMPONENTS = 100
MIXTURE_SIGMA = 20.0
MIXTURE_CENTRE_SEED = 0

# Seeds of the standard workloads.
DATA_SEED = 0
QUERY_SEED = 1
TRAIN_SEED = 2
T_DATA_SEED = 3
T_QUERY_SEED = 4
T_TRAIN_SEED = 5
IMAGE_DATA_SEED = 7
IMAGE_QUERY_SEED = 8


def mixture_centres(dim: int = 128) -> NDArray[np.float64]:
    """The shared mixture centres: ``default_rng(0).uniform(0, 128, (100, dim))``."""
    return np.random.default_rng(MIXTURE_CENTRE_SEED).uniform(0.0, 128.0, (MIXTURE_COMPONENTS, dim))


def mixture(n: int, seed: int, dim: int = 128, chunk: int = 1 << 18) -> NDArray[np.float32]:
    """``n`` integer-valued float32 rows in [0, 255] drawn from the shared Gaussian mixture.

    ``labels = rng.integers(0, 100, n)`` first, then the normal draws row-major, computed in
    float64 and cast to float32. Generated in chunks (same stream as one call) to bound memory.
    """
    centres = mixture_centres(dim)
    rng = np.random.default_rng(seed)
    labels = rng.integers(0, MIXTURE_COMPONENTS, n)
    out = np.empty((n, dim), dtype=np.float32)
    for start in range(0, n, chunk):
        stop = min(n, start + chunk)
        noise = rng.standard_normal((stop - start, dim))
        block = np.rint(centres[labels[start:stop]] + MIXTURE_SIGMA * noise)
        out[start:stop] = np.clip(block, 0.0, 255.0)
    return out


def student_t_unit(n: int, seed: int, dim: int = 100, chunk: int = 1 << 18) -> NDArray[np.float32]:
    """``n`` rows of Student-t (nu = 3) coordinates, L2-normalised in float64, cast to float32."""
    rng = np.random.default_rng(seed)
    out = np.empty((n, dim), dtype=np.float32)
    for start in range(0, n, chunk):
        stop = min(n, start + chunk)
        block = rng.standard_t(3.0, (stop - start, dim))
        block /= np.linalg.norm(block, axis=1)[:, None]
        out[start:stop] = block
    return out


def image_like(n: int, seed: int, side: int = 28, chunk: int = 1 << 15) -> NDArray[np.float32]:
    """``n`` flattened ``side x side`` images with uint8 values, as float32 rows.

    Per pixel: zero with probability 0.7, else uniform in 1..255; then a 3 x 3 box filter (zero
    padding, divided by 9) and ``rint``.
    """
    rng = np.random.default_rng(seed)
    out = np.empty((n, side * side), dtype=np.float32)
    for start in range(0, n, chunk):
        stop = min(n, start + chunk)
        m = stop - start
        zero = rng.random((m, side, side)) < 0.7
        values = rng.integers(1, 256, (m, side, side)).astype(np.float64)
        img = np.where(zero, 0.0, values)
        padded = np.pad(img, ((0, 0), (1, 1), (1, 1)))
        acc = np.zeros_like(img)
        for dy in range(3):
            for dx in range(3):
                acc += padded[:, dy : dy + side, dx : dx + side]
        out[start:stop] = np.rint(acc / 9.0).reshape(m, side * side)
    return out


def per_query_ef(nq: int, seed: int = 11, low: int = 32, high: int = 512) -> NDArray[np.int32]:
    """Per-query efSearch drawn uniformly from the integers ``low..high`` (inclusive)."""
    return np.random.default_rng(seed).integers(low, high + 1, nq).astype(np.int32)


def bernoulli_mask(n: int, p: float, seed: int = 12) -> NDArray[np.bool_]:
    """Filter mask with each id allowed independently with probability ``p``."""
    return np.random.default_rng(seed).random(n) < p


def prefix_mask(n: int, p: float) -> NDArray[np.bool_]:
    """Position-correlated filter mask: ids below ``p * n`` are allowed."""
    return np.arange(n) < int(p * n)
