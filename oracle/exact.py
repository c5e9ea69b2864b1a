"""Exact brute-force k-NN oracle, restated in NumPy -- TEST INFRASTRUCTURE ONLY.

Follows ``src/hnsw_engine/oracle.py`` (anamankev/hnsw-engine):

* ``exact_search`` <- ``oracle.py:35-126``: float32 distance filter (|q|^2 + |x|^2 - 2 q.x for L2,
  -q.x for ip, 1 - q.x for cosine on float64-normalised rows cast to float32), keep every point
  within ``2 * e`` of the k-th approximate distance, where ``e`` is the float32 error bound of
  ``oracle.py:169-178``; re-score survivors in float64 from the original input (cosine
  re-normalised) and order by (distance, id).
* ``exact_distances`` <- ``oracle.py:129-150`` (float64 distances of given ids, -1 -> +inf).

Pinned against the reference's outputs in ``tests/golden/exact.npz``. Used by the tests and by the
CPU baseline only.
"""

from __future__ import annotations

import numpy as np
from numpy.typing import NDArray

U_F32 = 2.0**-24
SAFETY = 4.0


def error_bound(metric: str, dim: int, qn: NDArray[np.float64], xmax: float) -> NDArray[np.float64]:
    s = SAFETY * U_F32
    if metric == "l2":
        return s * (dim + 4) * (qn + xmax) ** 2
    if metric == "ip":
        return s * (dim + 4) * qn * xmax
    return np.full(qn.shape, s * (dim + 8))


def _f32_rows(x: NDArray, metric: str, norms: NDArray[np.float64]) -> NDArray[np.float32]:
    if metric == "cosine":
        return np.ascontiguousarray(np.asarray(x, np.float64) / norms[:, None], dtype=np.float32)
    return np.ascontiguousarray(x, dtype=np.float32)


def exact_rows(metric: str, x: NDArray, q: NDArray, ids: NDArray[np.int64]) -> NDArray[np.float64]:
    rows = np.asarray(x[ids], dtype=np.float64)
    q64 = np.asarray(q, dtype=np.float64)
    if metric == "l2":
        diff = rows - q64
        return np.einsum("ij,ij->i", diff, diff)
    if metric == "ip":
        return -(rows @ q64)
    rows = rows / np.linalg.norm(rows, axis=1)[:, None]
    return 1.0 - rows @ (q64 / np.linalg.norm(q64))


def exact_search(data: NDArray, queries: NDArray, k: int, metric: str = "l2",
                 query_block: int = 256, data_block: int = 65536
                 ) -> tuple[NDArray[np.int64], NDArray[np.float64]]:
    x = np.asarray(data)
    q = np.asarray(queries)
    n, dim = x.shape
    xn = np.linalg.norm(np.asarray(x, np.float64), axis=1)
    qn = np.linalg.norm(np.asarray(q, np.float64), axis=1) if q.shape[0] else np.zeros(0)
    margins = 2.0 * error_bound(metric, dim, qn, float(xn.max()))
    x32_all = _f32_rows(x, metric, xn)
    xsq = np.einsum("ij,ij->i", x32_all, x32_all) if metric == "l2" else None
    out_ids = np.empty((q.shape[0], k), np.int64)
    out_d = np.empty((q.shape[0], k), np.float64)
    for qs in range(0, q.shape[0], query_block):
        qe = min(q.shape[0], qs + query_block)
        q32 = _f32_rows(q[qs:qe], metric, qn[qs:qe])
        qsq = np.einsum("ij,ij->i", q32, q32) if metric == "l2" else None
        m = margins[qs:qe]
        pool_i: list[list[NDArray[np.int64]]] = [[] for _ in range(qe - qs)]
        pool_d: list[list[NDArray[np.float32]]] = [[] for _ in range(qe - qs)]
        for ds in range(0, n, data_block):
            de = min(n, ds + data_block)
            dots = q32 @ x32_all[ds:de].T
            if metric == "l2":
                approx = qsq[:, None] + xsq[None, ds:de] - 2.0 * dots
            elif metric == "ip":
                approx = -dots
            else:
                approx = 1.0 - dots
            kk = min(k, de - ds)
            kth = np.partition(approx, kk - 1, axis=1)[:, kk - 1] if kk < de - ds else approx.max(axis=1)
            keep = approx <= (kth + m)[:, None]
            for row in range(qe - qs):
                cols = np.flatnonzero(keep[row])
                pool_i[row].append(cols.astype(np.int64) + ds)
                pool_d[row].append(approx[row, cols])
        for row in range(qe - qs):
            ci = np.concatenate(pool_i[row])
            ca = np.concatenate(pool_d[row])
            if ci.size > k:
                kth_g = np.partition(ca, k - 1)[k - 1]
                ci = ci[ca <= kth_g + m[row]]
            ex = exact_rows(metric, x, q[qs + row], ci)
            order = np.lexsort((ci, ex))[:k]
            out_ids[qs + row] = ci[order]
            out_d[qs + row] = ex[order]
    return out_ids, out_d


def exact_distances(data: NDArray, queries: NDArray, ids: NDArray, metric: str = "l2") -> NDArray[np.float64]:
    x = np.asarray(data)
    q = np.asarray(queries)
    idx = np.asarray(ids, dtype=np.int64)
    out = np.full(idx.shape, np.inf)
    for row in range(q.shape[0]):
        ok = idx[row] >= 0
        if ok.any():
            out[row, ok] = exact_rows(metric, x, q[row], idx[row, ok])
    return out
