"""The CPU oracle reproduces the reference's golden outputs bit for bit (no GPU needed).

Pins ``oracle/hnsw_oracle.c`` (search, filtered search, code-space search, re-rank; results AND
per-call work counters) and ``oracle/exact.py`` (brute-force k-NN) against outputs the reference
produced (``tests/golden/make_golden.py``).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import QUANT_CASES, SEARCH_CASES, case_arrays, iter_search_runs, load_golden
from hnsw_engine_b200.validation import prepare
from oracle import cpu, exact


@pytest.mark.parametrize("name", SEARCH_CASES)
def test_oracle_search_matches_reference(name: str) -> None:
    case = load_golden(f"search_{name}")
    arrays, ep, ml = case_arrays(case, name)
    metric = str(case["metric"])
    k = int(case["k"])
    queries = prepare(case["queries"], metric)
    for mi, mask, ef in iter_search_runs(case):
        ids, dists, ctr = cpu.search_batch(arrays, ep, ml, queries, k, ef, metric,
                                           allowed=mask, threads=4)
        np.testing.assert_array_equal(ids, case[f"ids_m{mi}_ef{ef}"])
        np.testing.assert_array_equal(dists, case[f"dists_m{mi}_ef{ef}"])
        np.testing.assert_array_equal(ctr.sum(axis=0), case[f"ctr_m{mi}_ef{ef}"])


def test_oracle_per_query_ef_matches_grouped_reference() -> None:
    case = load_golden("search_mix10k")
    arrays, ep, ml = case_arrays(case, "mix10k")
    ids, dists, ctr = cpu.search_batch(arrays, ep, ml, case["queries"], int(case["k"]),
                                       case["pq_ef"], "l2", threads=4)
    np.testing.assert_array_equal(ids, case["pq_ids"])
    np.testing.assert_array_equal(dists, case["pq_dists"])
    np.testing.assert_array_equal(ctr.sum(axis=0), case["pq_ctr"])


@pytest.mark.parametrize("name", QUANT_CASES)
def test_oracle_code_search_and_rerank_match_reference(name: str) -> None:
    from hnsw_engine_b200.quantization import ScalarQuantizer

    case = load_golden(f"quant_{name}")
    arrays, ep, ml = case_arrays(case, f"mix10k" if name == "mix10k" else name)
    metric = str(case["metric"])
    k, ef = int(case["k"]), int(case["ef"])
    quant = ScalarQuantizer.fit(arrays["vectors"])
    np.testing.assert_array_equal(quant.offset, case["offset"])
    assert quant.step == float(case["step"])
    codes = quant.encode(arrays["vectors"])
    if "codes" in case:
        np.testing.assert_array_equal(codes, case["codes"])
    prepared = prepare(case["queries"], metric)
    code_q = quant.transform_queries(prepared, metric)
    n = arrays["vectors"].shape[0]
    for r in case["reranks"]:
        r = int(r)
        fetch = min(max(r, k), n)
        ids, dists, _ = cpu.search_batch(arrays, ep, ml, code_q, fetch, max(ef, fetch), metric,
                                         codes=codes, threads=4)
        if r == 0:
            np.testing.assert_array_equal(ids, case[f"ids_r{r}"])
            np.testing.assert_array_equal(quant.to_distance(dists, prepared, metric), case[f"dists_r{r}"])
        else:
            rid, rd = cpu.rerank_batch(arrays["vectors"], prepared, ids, k, metric, threads=4)
            np.testing.assert_array_equal(rid, case[f"ids_r{r}"])
            np.testing.assert_array_equal(rd, case[f"dists_r{r}"])


def test_exact_oracle_matches_reference_known_answers() -> None:
    z = load_golden("exact")
    from hnsw_engine_b200.graphs import workload_vectors

    for name in z["names"]:
        name = str(name)
        data = z.get(f"{name}_data")
        if data is None:
            data = workload_vectors("mix10k")
        ids, dists = exact.exact_search(data, z[f"{name}_queries"], int(z[f"{name}_k"]),
                                        str(z[f"{name}_metric"]))
        np.testing.assert_array_equal(ids, z[f"{name}_ids"], err_msg=name)
        np.testing.assert_array_equal(dists, z[f"{name}_dists"], err_msg=name)


def test_oracle_epoch_and_threads_do_not_change_results() -> None:
    case = load_golden("search_int_l2")
    arrays, ep, ml = case_arrays(case, "int_l2")
    a = cpu.search_batch(arrays, ep, ml, case["queries"], 10, 50, "l2", threads=1)
    b = cpu.search_batch(arrays, ep, ml, case["queries"], 10, 50, "l2", threads=8)
    for x, y in zip(a, b, strict=True):
        np.testing.assert_array_equal(x, y)


def test_port_does_the_reference_work_query_by_query() -> None:
    """The CPU restatement timed as the reference arm and the CPU baseline does exactly the
    reference's work: per query, the same distance computations and hops as the reference's own
    counters (one ``HNSWIndex.search`` per query at ef = 192, the plain operating point of the 1M
    benchmark), and the same results. Equal work is what makes its speed stand for the reference's."""
    from conftest import mix10k_arrays
    from oracle import cpu

    case = load_golden("search_mix10k_counters")
    arrays, ep, ml = mix10k_arrays()
    ids, dists, ctr = cpu.search_batch(arrays, ep, ml, case["queries"], 10, int(case["ef"]), "l2",
                                       threads=4)
    np.testing.assert_array_equal(ctr, case["counters"])
    np.testing.assert_array_equal(ids, case["ids"])
    np.testing.assert_array_equal(dists, case["dists"])
