"""The distance arithmetic chosen from the upload's host statistics (``mode_from_stats``) equals the
host rules of ``choose_mode`` on every kind of batch, without a GPU: the statistics come from the
library's host pass (``hnsw_b200_upload_queries`` with no device destination), the graph facts from
a stand-in object."""

from __future__ import annotations

import ctypes
import types

import numpy as np
import pytest


@pytest.fixture(scope="module")
def lib():
    from hnsw_engine_b200 import _lib, build

    build.build()
    return _lib.load()


def _stats(lib, q: np.ndarray):
    from hnsw_engine_b200._lib import ValueStats, check

    st = ValueStats()
    check(lib.hnsw_b200_upload_queries(q.ctypes.data, None, q.size, 4, ctypes.byref(st), None, None))
    return st


def _graph(metric: str, dim: int, byte_rows: bool, integer: bool, hi: float):
    from hnsw_engine_b200.engine import DeviceGraph

    g = types.SimpleNamespace(metric=metric, dim=dim, vector_bytes=b"rows" if byte_rows else None,
                              _integer=integer, _lo=np.zeros(dim), _hi=np.full(dim, hi))
    g.exact_f32_ok = types.MethodType(DeviceGraph.exact_f32_ok, g)
    g.choose_mode = types.MethodType(DeviceGraph.choose_mode, g)
    g.mode_from_stats = types.MethodType(DeviceGraph.mode_from_stats, g)
    return g


@pytest.mark.parametrize("metric", ["l2", "ip", "cosine"])
@pytest.mark.parametrize("byte_rows,integer,hi", [(True, True, 255.0), (False, True, 1000.0),
                                                  (False, True, 4e5), (False, False, 1.0)])
def test_mode_from_stats_equals_the_host_rules(lib, metric, byte_rows, integer, hi) -> None:
    rng = np.random.default_rng(5)
    dim = 16
    g = _graph(metric, dim, byte_rows, integer, hi)
    batches = {
        "bytes": rng.integers(0, 256, (50, dim)),
        "wide integers": rng.integers(-3000, 3000, (50, dim)),
        "huge integers": rng.integers(0, 10**6, (50, dim)),
        "fractions": rng.standard_normal((50, dim)),
        "half": rng.integers(0, 256, (50, dim)) + 0.5,
        "empty": np.zeros((0, dim)),
    }
    for name, b in batches.items():
        q = np.ascontiguousarray(b, dtype=np.float32)
        want = g.choose_mode(q, False) if q.size else 0  # choose_mode_device: float64 when empty
        assert g.mode_from_stats(_stats(lib, q), q) == want, name
