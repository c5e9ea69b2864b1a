"""Parity of the tensor-core exact k-NN with the reference's ``oracle.exact_search``.

Ids must be bit-exact, and distances equal, on every known-answer case the reference tests
(``tests/golden/exact.npz``, produced by the reference), and on image-like uint8 data and float
data against the NumPy oracle. Float distances agree to 1e-12 (summation order differs from
NumPy's in the last bits on non-integer data).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def assert_same_neighbors(ids_a, dist_a, ids_b, dist_b, atol=1e-9):
    """Distances equal position by position; ids strictly inside the k-th distance identical.

    Rows tied (within ``atol``) at a distance may order differently when the last bits of two
    float64 sums differ (the criterion of the reference's ``tests/helpers.py:38-57``).
    """
    np.testing.assert_allclose(dist_a, dist_b, rtol=0, atol=atol)
    for row in range(ids_a.shape[0]):
        boundary = max(dist_a[row, -1], dist_b[row, -1]) - atol
        inside_a = set(ids_a[row][dist_a[row] < boundary].tolist())
        inside_b = set(ids_b[row][dist_b[row] < boundary].tolist())
        assert inside_a == inside_b, row
        for d in np.unique(np.round(dist_a[row], 9)):
            ta = set(ids_a[row][np.abs(dist_a[row] - d) <= atol].tolist())
            tb = set(ids_b[row][np.abs(dist_b[row] - d) <= atol].tolist())
            if d < boundary:
                assert ta == tb, (row, d)


def test_known_answers_match_reference() -> None:
    from hnsw_engine_b200.exact_knn import exact_search
    from hnsw_engine_b200.graphs import workload_vectors

    z = load_golden("exact")
    for name in z["names"]:
        name = str(name)
        data = z.get(f"{name}_data")
        if data is None:
            data = workload_vectors("mix10k")
        metric = str(z[f"{name}_metric"])
        ids, dists = exact_search(data, z[f"{name}_queries"], int(z[f"{name}_k"]), metric)
        if name.startswith("float") or metric == "cosine":
            assert_same_neighbors(ids, dists, z[f"{name}_ids"], z[f"{name}_dists"], atol=1e-12)
        else:
            np.testing.assert_array_equal(ids, z[f"{name}_ids"], err_msg=name)
            np.testing.assert_array_equal(dists, z[f"{name}_dists"], err_msg=name)


@pytest.mark.parametrize("metric", ["l2", "ip"])
def test_image_like_uint8_matches_oracle(metric: str) -> None:
    from hnsw_engine_b200 import synthetic
    from hnsw_engine_b200.exact_knn import exact_search
    from oracle import exact

    data = synthetic.image_like(6000, seed=7)
    queries = synthetic.image_like(64, seed=8)
    ids, dists, st = exact_search(data, queries, 100, metric, return_stats=True)
    o_ids, o_d = exact.exact_search(data, queries, 100, metric)
    np.testing.assert_array_equal(ids, o_ids)
    np.testing.assert_array_equal(dists, o_d)
    assert st.candidates >= 64 * 100
    u8 = exact_search(data.astype(np.uint8), queries.astype(np.uint8), 100, metric)
    np.testing.assert_array_equal(u8[0], o_ids)


@pytest.mark.parametrize("metric", ["l2", "ip"])
def test_byte_rows_of_any_width_match_oracle(metric: str) -> None:
    """The integer filter (byte rows) at widths around its 128-byte K chunks, values at both ends
    of [0, 255] and inner products beyond 2^24 (dim 1000): ids and distances bit-exact, and the
    measured error (float copies of 2^24 or more only) within the bound."""
    from hnsw_engine_b200.exact_knn import exact_search
    from oracle import exact

    rng = np.random.default_rng(21)
    for dim in (1, 127, 129, 1000):
        data = rng.integers(0, 256, (3000, dim)).astype(np.float32)
        data[:50] = 255.0
        data[50:100] = 0.0
        queries = rng.integers(0, 256, (40, dim)).astype(np.float32)
        queries[0] = 255.0
        queries[1] = 0.0
        ids, dists, st = exact_search(data, queries, 20, metric, return_stats=True)
        o_ids, o_d = exact.exact_search(data, queries, 20, metric)
        np.testing.assert_array_equal(ids, o_ids, err_msg=f"dim {dim}")
        np.testing.assert_array_equal(dists, o_d, err_msg=f"dim {dim}")
        assert 0.0 <= st.filter_max_error <= st.filter_error_bound
        u8 = exact_search(data.astype(np.uint8), queries.astype(np.uint8), 20, metric)
        np.testing.assert_array_equal(u8[0], o_ids)
        np.testing.assert_array_equal(u8[1], o_d)


def test_integer_rows_outside_bytes_and_cosine_bytes_match_oracle() -> None:
    """Signed integer rows (not bytes: the BF16 filter, one term) and byte rows under cosine (also
    the BF16 filter) against the oracle."""
    from hnsw_engine_b200.exact_knn import exact_search
    from oracle import exact

    rng = np.random.default_rng(22)
    data = rng.integers(-128, 128, (5000, 64)).astype(np.float32)
    queries = rng.integers(-128, 128, (30, 64)).astype(np.float32)
    for metric in ("l2", "ip"):
        ids, dists, st = exact_search(data, queries, 15, metric, return_stats=True)
        o_ids, o_d = exact.exact_search(data, queries, 15, metric)
        np.testing.assert_array_equal(ids, o_ids, err_msg=metric)
        np.testing.assert_array_equal(dists, o_d, err_msg=metric)
        assert st.filter_error_bound > 0.0  # signed values: the BF16 filter with its margins
    b = rng.integers(0, 256, (5000, 64)).astype(np.uint8)
    qb = rng.integers(0, 256, (30, 64)).astype(np.uint8)
    ids, dists = exact_search(b, qb, 15, "cosine")
    o_ids, o_d = exact.exact_search(b, qb, 15, "cosine")
    assert_same_neighbors(ids, dists, o_ids, o_d, atol=1e-12)


@pytest.mark.parametrize("metric", ["l2", "ip", "cosine"])
def test_float_data_matches_oracle(metric: str) -> None:
    from hnsw_engine_b200.exact_knn import exact_search
    from oracle import exact

    rng = np.random.default_rng(3)
    data = rng.standard_t(3.0, (20000, 100)).astype(np.float32)
    queries = rng.standard_t(3.0, (50, 100)).astype(np.float32)
    ids, dists, st = exact_search(data, queries, 10, metric, return_stats=True)
    o_ids, o_d = exact.exact_search(data, queries, 10, metric)
    assert_same_neighbors(ids, dists, o_ids, o_d, atol=1e-9 if metric != "cosine" else 1e-12)
    assert st.filter_error_bound > 0.0  # not bytes: the BF16 filter with its margins
    assert 0.0 <= st.filter_max_error <= st.filter_error_bound


def test_mixture_1m_shape_subset_matches_oracle() -> None:
    """The 1M x 128 workload's generator at 100K rows, k = 100 (integer data: bit-exact)."""
    from hnsw_engine_b200 import synthetic
    from hnsw_engine_b200.exact_knn import exact_search
    from oracle import exact

    data = synthetic.mixture(100_000, seed=0)
    queries = synthetic.mixture(200, seed=1)
    ids, dists = exact_search(data, queries, 100, "l2")
    o_ids, o_d = exact.exact_search(data, queries, 100, "l2")
    np.testing.assert_array_equal(ids, o_ids)
    np.testing.assert_array_equal(dists, o_d)


def _sample_rows(nq: int, count: int) -> np.ndarray:
    """Query rows spread over the whole batch (both 8192-query chunks of a 10K batch)."""
    return np.unique(np.linspace(0, nq - 1, count).round().astype(np.int64))


def test_full_mixture_config_1m_x_128_k100_matches_oracle() -> None:
    """The 1M x 128 mixture with its 10K queries at k = 100, searched in full on the GPU; a spread
    sample of 256 queries against the CPU restatement of oracle.exact_search over all 1M rows.
    Byte rows at d = 128 (distances below 2^24): the filter values are exact, error and bound 0."""
    from hnsw_engine_b200 import synthetic
    from hnsw_engine_b200.exact_knn import exact_search
    from oracle import exact

    data = synthetic.mixture(1_000_000, seed=synthetic.DATA_SEED)
    queries = synthetic.mixture(10_000, seed=synthetic.QUERY_SEED)
    ids, dists, st = exact_search(data, queries, 100, "l2", return_stats=True)
    rows = _sample_rows(10_000, 256)
    o_ids, o_d = exact.exact_search(data, queries[rows], 100, "l2")
    np.testing.assert_array_equal(ids[rows], o_ids)
    np.testing.assert_array_equal(dists[rows], o_d)
    assert st.filter_max_error == 0.0
    assert st.filter_error_bound == 0.0


def test_full_image_config_60k_x_784_k100_matches_oracle() -> None:
    """The 60K x 784 image-like uint8 set with its 10K queries at k = 100 on the GPU; a spread
    sample of 256 queries against the CPU oracle, ids and distances bit-exact. Byte rows take the
    integer filter: its distances are exact, and only float copies of 2^24 or more may round, within
    the bound."""
    from hnsw_engine_b200 import synthetic
    from hnsw_engine_b200.exact_knn import exact_search
    from oracle import exact

    data = synthetic.image_like(60_000, seed=synthetic.IMAGE_DATA_SEED).astype(np.uint8)
    queries = synthetic.image_like(10_000, seed=synthetic.IMAGE_QUERY_SEED).astype(np.uint8)
    ids, dists, st = exact_search(data, queries, 100, "l2", return_stats=True)
    rows = _sample_rows(10_000, 256)
    o_ids, o_d = exact.exact_search(data, queries[rows], 100, "l2")
    np.testing.assert_array_equal(ids[rows], o_ids)
    np.testing.assert_array_equal(dists[rows], o_d)
    assert 0.0 <= st.filter_max_error <= st.filter_error_bound


def test_candidate_overflow_is_retried_with_longer_lists() -> None:
    """50,000 identical rows all tie at every query's k-th distance: far more rows fall within the
    margin than the first candidate lists hold. The call re-runs with longer lists and returns the
    exact answer (ties to the lower id) instead of failing."""
    from hnsw_engine_b200.exact_knn import exact_search
    from oracle import exact

    rng = np.random.default_rng(11)
    data = rng.integers(0, 256, (100_000, 32)).astype(np.float32)
    data[10_000:60_000] = 7.0  # one row repeated 50,000 times
    queries = np.full((40, 32), 7.0, np.float32) + rng.integers(0, 2, (40, 32)).astype(np.float32)
    ids, dists, st = exact_search(data, queries, 10, "l2", return_stats=True)
    o_ids, o_d = exact.exact_search(data, queries, 10, "l2")
    np.testing.assert_array_equal(ids, o_ids)
    np.testing.assert_array_equal(dists, o_d)
    assert st.candidates >= 40 * 50_000
