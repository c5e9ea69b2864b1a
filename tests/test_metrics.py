"""The recall judge against the reference's own recall cases (``tests/test_bench.py:23-49`` of the
reference, on ``src/hnsw_engine/bench/metrics.py:13-51``): tied alternatives count, missing and
repeated ids do not, and only the first k columns are read. CPU only."""

from __future__ import annotations

import numpy as np
import pytest

from hnsw_engine_b200.metrics import per_query_hits, recall_at_k


def test_a_tied_alternative_counts_for_recall_but_not_for_id_recall() -> None:
    # id 9 sits at the exact distance of the third true neighbour (3.0)
    out = recall_at_k(np.array([[0, 1, 9]]), np.array([[1.0, 2.0, 3.0]]),
                      np.array([[0, 1, 2]]), np.array([[1.0, 2.0, 3.0]]), k=3)
    assert out == {"recall": 1.0, "recall_ids": pytest.approx(2 / 3)}


def test_missing_and_repeated_ids_score_nothing() -> None:
    true_ids = np.array([[0, 1, 2], [0, 1, 2]])
    true_dist = np.array([[1.0, 2.0, 3.0], [1.0, 2.0, 3.0]])
    found = np.array([[0, 0, 0], [0, -1, 7]])
    found_dist = np.array([[1.0, 1.0, 1.0], [1.0, np.inf, 5.0]])
    out = recall_at_k(found, found_dist, true_ids, true_dist, k=3)
    assert out["recall"] == pytest.approx(1 / 3)
    assert out["recall_ids"] == pytest.approx(1 / 3)
    np.testing.assert_array_equal(per_query_hits(found, found_dist, true_dist, 3), [1, 1])


def test_only_the_first_k_columns_are_read() -> None:
    out = recall_at_k(np.array([[0, 5, 1, 2]]), np.array([[1.0, 9.0, 2.0, 3.0]]),
                      np.array([[0, 1, 2, 3]]), np.array([[1.0, 2.0, 3.0, 4.0]]), k=2)
    assert out["recall"] == 0.5


def test_the_tie_tolerance_is_relative_above_one_and_absolute_below() -> None:
    # threshold = kth + 1e-9 * max(1, |kth|)
    kth_big, kth_small = 1e6, 0.25
    found = np.array([[0], [0]])
    inside = np.array([[kth_big + 0.9e-3], [kth_small + 0.9e-9]])
    outside = np.array([[kth_big + 1.1e-3], [kth_small + 1.1e-9]])
    true_d = np.array([[kth_big], [kth_small]])
    np.testing.assert_array_equal(per_query_hits(found, inside, true_d, 1), [1, 1])
    np.testing.assert_array_equal(per_query_hits(found, outside, true_d, 1), [0, 0])
