"""The host pass of the query upload (``hnsw_b200_upload_queries`` with no device destination, so
no GPU work): the statistics that choose the distance arithmetic equal NumPy's, for every split of
the batch over host threads. The copy itself is checked on the GPU through ``batch_search``."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest


@pytest.fixture(scope="module")
def lib():
    from hnsw_engine_b200 import _lib, build

    build.build()
    return _lib.load()


def _scan(lib, x: np.ndarray, threads: int):
    from hnsw_engine_b200._lib import ValueStats, check

    x = np.ascontiguousarray(x, dtype=np.float32)
    st = ValueStats()
    check(lib.hnsw_b200_upload_queries(x.ctypes.data, None, x.size, threads, ctypes.byref(st), None,
                                       None))
    return st


def _cases():
    rng = np.random.default_rng(4)
    n = 3 * 65536 + 7
    yield "integers", rng.integers(0, 256, n).astype(np.float32)
    yield "negative integers", rng.integers(-300, 300, n).astype(np.float32)
    yield "gaussian", rng.standard_normal(n).astype(np.float32)
    big = rng.integers(0, 256, n).astype(np.float32)
    big[n // 2] = 1e30  # every float32 beyond 2^23 is an integer
    yield "huge", big
    half = rng.integers(0, 256, n).astype(np.float32)
    half[-1] = 8388607.5  # the largest non-integer float32, in the last part
    yield "largest fraction", half
    neg0 = np.zeros(1000, np.float32)
    neg0[5] = -0.0
    yield "signed zeros", neg0
    yield "one value", np.array([3.25], np.float32)
    yield "empty", np.zeros(0, np.float32)
    for bad in (np.nan, np.inf, -np.inf):
        v = rng.integers(0, 256, n).astype(np.float32)
        v[2 * 65536 + 3] = bad
        yield f"{bad}", v


@pytest.mark.parametrize("threads", [1, 3, 16])
def test_upload_statistics_match_numpy(lib, threads: int) -> None:
    for name, x in _cases():
        st = _scan(lib, x, threads)
        finite = bool(np.isfinite(x).all())
        assert st.finite == int(finite), name
        if finite:
            assert st.integer == int(np.array_equal(x, np.rint(x))), name
            if x.size:
                assert (st.min, st.max) == (float(x.min()), float(x.max())), name
            else:
                assert (st.min, st.max) == (0.0, 0.0)


def test_upload_rejects_null_arguments(lib) -> None:
    from hnsw_engine_b200._lib import ValueStats

    st = ValueStats()
    assert lib.hnsw_b200_upload_queries(None, None, 4, 1, ctypes.byref(st), None, None) == -1
    assert lib.hnsw_b200_upload_queries(None, None, 0, 1, None, None, None) == -1
    assert lib.hnsw_b200_upload_queries(None, None, 0, 1, ctypes.byref(st), None, None) == 0
    # a misaligned staging buffer is refused before any copy
    buf = (ctypes.c_float * 8)()
    assert lib.hnsw_b200_upload_queries(None, None, 0, 1, ctypes.byref(st),
                                        ctypes.addressof(buf) + 4, None) == -1


def test_concurrent_callers_each_get_their_own_statistics(lib) -> None:
    """The host pool runs one batch at a time: callers on several threads (ctypes releases the
    GIL) each get the statistics of their own batch."""
    import threading

    rng = np.random.default_rng(9)
    batches = [rng.integers(0, 256, 300_000).astype(np.float32) for _ in range(6)]
    batches[2] = batches[2] + 0.5  # not integer
    batches[4][77] = np.inf        # not finite
    want = [(bool(np.isfinite(b).all()), bool(np.array_equal(b, np.rint(b)))) for b in batches]
    got: list = [None] * len(batches)

    def run(i: int) -> None:
        for _ in range(20):
            st = _scan(lib, batches[i], 8)
            got[i] = (bool(st.finite), bool(st.integer) if st.finite else want[i][1])

    threads = [threading.Thread(target=run, args=(i,)) for i in range(len(batches))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert got == want
