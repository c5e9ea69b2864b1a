"""Host-side search API without a GPU: argument rules and error messages of the reference's
``HNSWIndex`` (src/hnsw_engine/index.py:244-312, _validation.py:16-66, metrics.py:42-68), and the
all-false filter that returns padding without searching (index.py:289-291)."""

from __future__ import annotations

import numpy as np
import pytest

from hnsw_engine_b200.index import HNSWIndex
from hnsw_engine_b200.validation import as_matrix, check_int, check_k, prepare


def _index(n: int = 10, dim: int = 4, metric: str = "l2", ef_search: int = 50) -> HNSWIndex:
    """An index that reports n nodes but holds no device graph: only host checks can run."""
    idx = HNSWIndex(dim, metric=metric, ef_search=ef_search)
    idx._size = n
    return idx


def test_ef_defaults_and_is_raised_to_k() -> None:
    idx = _index(ef_search=7)
    assert idx._check_search_args(5, None) == (5, 7)
    assert idx._check_search_args(9, None) == (9, 9)
    assert idx._check_search_args(3, 2) == (3, 3)
    k, ef = idx._check_search_args(4, np.array([1, 8, 4]))
    assert k == 4 and ef.tolist() == [4, 8, 4]


@pytest.mark.parametrize("k,ef,exc,msg", [
    (0, None, ValueError, "k must be >= 1, got 0"),
    (11, None, ValueError, r"k=11 exceeds the number of indexed vectors \(10\)"),
    (True, None, TypeError, "k must be an integer, got bool"),
    (2.0, None, TypeError, "k must be an integer, got float"),
    (2, 0, ValueError, "ef must be >= 1, got 0"),
    (2, np.array([3, 0]), ValueError, "ef must be >= 1, got 0"),
    (2, np.array([[3]]), TypeError, "ef must be an integer or a 1-D integer array"),
])
def test_search_argument_errors(k, ef, exc, msg) -> None:
    with pytest.raises(exc, match=msg):
        _index()._check_search_args(k, ef)


def test_empty_index_refuses_to_search() -> None:
    with pytest.raises(ValueError, match="cannot search an empty index"):
        _index(n=0).batch_search(np.zeros((1, 4), np.float32))


def test_filter_checks() -> None:
    idx = _index()
    with pytest.raises(TypeError, match="filter must be a boolean array, got dtype int64"):
        idx._check_filter(np.ones(10, dtype=np.int64))
    with pytest.raises(ValueError, match=r"filter must have one entry per indexed vector \(10\)"):
        idx._check_filter(np.ones(9, dtype=bool))


def test_all_false_filter_pads_without_a_device() -> None:
    idx = _index()
    ids, d = idx.batch_search(np.zeros((3, 4), np.float32), k=2, filter=np.zeros(10, bool))
    assert ids.dtype == np.int64 and ids.shape == (3, 2) and (ids == -1).all()
    assert d.dtype == np.float64 and np.isinf(d).all()
    ids, d = idx.search(np.zeros(4, np.float32), k=2, filter=np.zeros(10, bool))
    assert ids.tolist() == [-1, -1] and np.isinf(d).all()


@pytest.mark.parametrize("queries,msg", [
    (np.zeros((2, 3)), "vectors has dimension 3, expected 4"),
    (np.zeros(4), r"vectors must be a 2-D array, got shape \(4,\)"),
    (np.array([[1, 2, 3, np.nan]]), "vectors contains NaN or infinite values"),
    (np.array([["a", "b", "c", "d"]]), "vectors must contain real numbers"),
])
def test_query_validation_messages(queries, msg) -> None:
    # batch_search names its queries "vectors" (index.py:239-240, 289), search names it "query"
    with pytest.raises(ValueError, match=msg):
        _index().batch_search(queries, k=1, filter=np.zeros(10, bool))


def test_single_query_validation_messages() -> None:
    with pytest.raises(ValueError, match="query has dimension 3, expected 4"):
        _index().search(np.zeros(3), k=1, filter=np.zeros(10, bool))
    with pytest.raises(ValueError, match=r"query must be a 1-D array, got shape \(1, 4\)"):
        _index().search(np.zeros((1, 4)), k=1, filter=np.zeros(10, bool))


def test_validation_helpers() -> None:
    assert check_int(np.int64(3), "x", minimum=1) == 3
    assert check_k(10, 10) == 10
    assert as_matrix([[1, 2]], "m", dim=2).shape == (1, 2)


def test_prepare_follows_the_reference() -> None:
    x = np.array([[3.0, 4.0], [1.0, 0.0]])
    np.testing.assert_array_equal(prepare(x, "l2"), x.astype(np.float32))
    got = prepare(x, "cosine")
    assert got.dtype == np.float32
    np.testing.assert_array_equal(got, (x / np.linalg.norm(x, axis=1)[:, None]).astype(np.float32))
    with pytest.raises(ValueError):
        prepare(np.array([[0.0, 0.0]]), "cosine")


def test_add_is_left_to_the_reference_build() -> None:
    with pytest.raises(NotImplementedError):
        _index().add(np.zeros((1, 4), np.float32))


@pytest.mark.parametrize("metric", ["l2", "cosine", "ip"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.int16, np.uint8])
def test_prepare_into_a_staging_buffer_matches(metric, dtype) -> None:
    # batch_search writes prepared queries straight into page-locked memory: same values
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((33, 8)) * 50 + 60).astype(dtype)
    out = np.empty((33, 8), np.float32)
    got = prepare(x, metric, out=out, checked_finite=True)
    assert got is out
    np.testing.assert_array_equal(out, prepare(x, metric))


def test_prepare_into_a_buffer_still_reports_overflow() -> None:
    out = np.empty((1, 2), np.float32)
    with pytest.raises(ValueError, match="overflow float32"):
        prepare(np.array([[1e39, 0.0]]), "l2", out=out, checked_finite=True)
    with pytest.raises(ValueError, match="overflow float32"):
        prepare(np.array([[np.inf, 0.0]], np.float32), "l2")
