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


@pytest.mark.parametrize("metric", ["l2", "ip", "cosine"])
def test_float_data_matches_oracle(metric: str) -> None:
    from hnsw_engine_b200.exact_knn import exact_search
    from oracle import exact

    rng = np.random.default_rng(3)
    data = rng.standard_t(3.0, (20000, 100)).astype(np.float32)
    queries = rng.standard_t(3.0, (50, 100)).astype(np.float32)
    ids, dists = exact_search(data, queries, 10, metric)
    o_ids, o_d = exact.exact_search(data, queries, 10, metric)
    assert_same_neighbors(ids, dists, o_ids, o_d, atol=1e-9 if metric != "cosine" else 1e-12)


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
