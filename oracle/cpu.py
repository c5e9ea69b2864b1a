"""ctypes binding of the C oracle (``hnsw_oracle.c``) -- TEST INFRASTRUCTURE ONLY.

Only the tests, the smoke check and the benchmark's CPU-baseline leg use this module. It builds
``libhnsw_oracle.so`` with the Makefile beside it when the library is missing.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path
from typing import Any

import numpy as np
from numpy.typing import NDArray

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libhnsw_oracle.so"
METRIC_CODES = {"l2": 0, "ip": 1, "cosine": 2}

_lib: ctypes.CDLL | None = None


def build() -> Path:
    """Compile the oracle library (idempotent)."""
    src = HERE / "hnsw_oracle.c"
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        p = ctypes.c_void_p
        i32, i64 = ctypes.c_int32, ctypes.c_int64
        _lib.oracle_search_batch.argtypes = [
            p, i32, i64, i32, i32, p, i32, p, i32, i64, p, i32, p, p, i32, p, p, i64, i32, p, p,
            p, p, i32,
        ]
        _lib.oracle_search_batch.restype = ctypes.c_int
        _lib.oracle_rerank_batch.argtypes = [p, i64, i32, p, i64, i32, p, i32, i32, p, p, i32]
        _lib.oracle_rerank_batch.restype = ctypes.c_int
        _lib.oracle_max_threads.restype = ctypes.c_int
    return _lib


def _ptr(a: NDArray[Any] | None) -> int | None:
    return None if a is None else a.ctypes.data


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def search_batch(
    arrays: dict[str, NDArray[Any]],
    entry_point: int,
    max_level: int,
    queries: NDArray[Any],
    k: int,
    ef: int | NDArray[np.integer],
    metric: str,
    *,
    allowed: NDArray[np.bool_] | None = None,
    codes: NDArray[np.uint8] | None = None,
    threads: int = 1,
) -> tuple[NDArray[np.int64], NDArray[np.float64], NDArray[np.int64]]:
    """``_search_batch`` over the native arrays; returns ``(ids, dists, counters)``.

    ``queries`` are float32 prepared queries, or float64 code-space queries when ``codes`` is
    given (then distances are taken to the uint8 codes). ``ef`` is a scalar or one value per query
    (layer 0 uses ``max(ef, k)``). ``counters`` is ``(nq, 2)``: distance computations and hops.
    """
    vectors = np.ascontiguousarray(arrays["vectors"], dtype=np.float32)
    n, dim = vectors.shape
    nq = queries.shape[0]
    if codes is not None:
        q = np.ascontiguousarray(queries, dtype=np.float64)
        rows: NDArray[Any] = np.ascontiguousarray(codes, dtype=np.uint8)
    else:
        q = np.ascontiguousarray(queries, dtype=np.float32)
        rows = vectors
    efs = np.ascontiguousarray(np.broadcast_to(np.asarray(ef, dtype=np.int32), (nq,)))
    links0 = np.ascontiguousarray(arrays["links0"], dtype=np.int32)
    links_up = np.ascontiguousarray(arrays["links_up"], dtype=np.int32)
    if links_up.ndim != 2 or links_up.shape[0] == 0:
        links_up = np.zeros((1, links0.shape[1] // 2 + 1), dtype=np.int32)
    count0 = np.ascontiguousarray(arrays["count0"], dtype=np.int32)
    count_up = np.ascontiguousarray(arrays["count_up"], dtype=np.int32)
    if count_up.size == 0:
        count_up = np.zeros(1, dtype=np.int32)
    upper = np.ascontiguousarray(arrays["upper_offset"], dtype=np.int64)
    mask = None if allowed is None else np.ascontiguousarray(allowed, dtype=np.uint8)
    ids = np.empty((nq, k), dtype=np.int64)
    dists = np.empty((nq, k), dtype=np.float64)
    counters = np.empty((nq, 2), dtype=np.int64)
    rc = lib().oracle_search_batch(
        _ptr(q), int(codes is not None), nq, dim, k, _ptr(efs), METRIC_CODES[metric], _ptr(rows),
        int(codes is not None), n, _ptr(links0), links0.shape[1], _ptr(count0), _ptr(links_up),
        links_up.shape[1], _ptr(count_up), _ptr(upper), int(entry_point), int(max_level),
        _ptr(mask), _ptr(ids), _ptr(dists), _ptr(counters), int(threads),
    )
    if rc != 0:
        raise MemoryError("oracle search ran out of memory")
    return ids, dists, counters


def rerank_batch(
    vectors: NDArray[np.float32],
    queries: NDArray[np.float32],
    candidates: NDArray[np.int64],
    k: int,
    metric: str,
    *,
    threads: int = 1,
) -> tuple[NDArray[np.int64], NDArray[np.float64]]:
    """``_rerank_batch``: exact float64 distances to the candidates, best ``k`` by (d, id)."""
    vec = np.ascontiguousarray(vectors, dtype=np.float32)
    q = np.ascontiguousarray(queries, dtype=np.float32)
    cand = np.ascontiguousarray(candidates, dtype=np.int64)
    nq = q.shape[0]
    ids = np.empty((nq, k), dtype=np.int64)
    dists = np.empty((nq, k), dtype=np.float64)
    rc = lib().oracle_rerank_batch(
        _ptr(q), nq, q.shape[1], _ptr(vec), vec.shape[0], METRIC_CODES[metric], _ptr(cand),
        cand.shape[1], k, _ptr(ids), _ptr(dists), int(threads),
    )
    if rc != 0:
        raise MemoryError("oracle rerank ran out of memory")
    return ids, dists


def default_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)))
