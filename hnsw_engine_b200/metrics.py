"""Recall measure: the reference's tie-aware recall@k (``src/hnsw_engine/bench/metrics.py:13-51``).

A returned id counts when it is a valid id (not ``-1``), not a repeat within the row, and its exact
distance is at most the exact k-th neighbour distance plus ``1e-9 * max(1, |kth|)``: equally close
points are interchangeable, which matters on integer data where exact ties are common.
``recall_ids`` is the plain overlap with the oracle's top-k ids.
"""

from __future__ import annotations

import numpy as np
from numpy.typing import NDArray

RELATIVE_TIE_TOLERANCE = 1e-9


def per_query_hits(found_ids: NDArray[np.int64], found_exact: NDArray[np.float64],
                   true_dist: NDArray[np.float64], k: int) -> NDArray[np.int64]:
    """Tie-aware hits per query (0..k), vectorised."""
    f = np.asarray(found_ids)[:, :k]
    d = np.asarray(found_exact)[:, :k]
    kth = np.asarray(true_dist)[:, k - 1 : k]
    thr = kth + RELATIVE_TIE_TOLERANCE * np.maximum(1.0, np.abs(kth))
    order = np.argsort(f, axis=1, kind="stable")
    fs = np.take_along_axis(f, order, axis=1)
    first = np.ones_like(fs, dtype=bool)
    first[:, 1:] = fs[:, 1:] != fs[:, :-1]
    unique = np.empty_like(first)
    np.put_along_axis(unique, order, first, axis=1)
    ok = (f >= 0) & unique & (d <= thr)
    return ok.sum(axis=1)


def recall_at_k(found_ids: NDArray[np.int64], found_exact: NDArray[np.float64],
                true_ids: NDArray[np.int64], true_dist: NDArray[np.float64], k: int) -> dict[str, float]:
    hits = per_query_hits(found_ids, found_exact, true_dist, k)
    f = np.asarray(found_ids)[:, :k]
    t = np.asarray(true_ids)[:, :k]
    id_hits = [len(set(a[a >= 0].tolist()) & set(b.tolist())) for a, b in zip(f, t, strict=True)]
    return {"recall": float(hits.mean() / k), "recall_ids": float(np.mean(id_hits) / k)}
