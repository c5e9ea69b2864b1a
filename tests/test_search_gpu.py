"""Parity of the CUDA search with the reference: bit-exact ids, distances and work counters.

Every case runs through the C ABI (``libhnsw_b200.so`` via :class:`DeviceGraph` or the
:class:`HNSWIndex` facade) and is compared with the reference's golden outputs, and on the larger
graphs with the CPU oracle on the same inputs.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import QUANT_CASES, SEARCH_CASES, case_arrays, iter_search_runs, load_golden

pytestmark = pytest.mark.gpu


def _index(arrays, ep, ml, metric, M, locality=None):
    from hnsw_engine_b200 import HNSWIndex

    return HNSWIndex.from_arrays(arrays, ep, ml, dim=arrays["vectors"].shape[1], metric=metric, M=M,
                                 locality=locality)


@pytest.mark.parametrize("locality", [False, True], ids=["reference_order", "cell_order"])
@pytest.mark.parametrize("name", SEARCH_CASES)
def test_search_matches_reference_bit_for_bit(name: str, locality: bool) -> None:
    """Both device node orders: the reference's, and the cell order (internal ids for memory,
    original ids for results and for ties between equal distances)."""
    case = load_golden(f"search_{name}")
    arrays, ep, ml = case_arrays(case, name)
    metric = str(case["metric"])
    M = (arrays["links0"].shape[1] - 1) // 2
    index = _index(arrays, ep, ml, metric, M, locality)
    k = int(case["k"])
    for mi, mask, ef in iter_search_runs(case):
        index.reset_counters()
        ids, dists = index.batch_search(case["queries"], k=k, ef=ef, filter=mask)
        np.testing.assert_array_equal(ids, case[f"ids_m{mi}_ef{ef}"], err_msg=f"{name} m{mi} ef{ef}")
        np.testing.assert_array_equal(dists, case[f"dists_m{mi}_ef{ef}"])
        st = index.stats()
        np.testing.assert_array_equal([st.distance_computations, st.hops], case[f"ctr_m{mi}_ef{ef}"])


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_every_arithmetic_mode_agrees_on_integer_data(mode: int) -> None:
    """Float64-sequential, exact float32 and byte (dp4a) kernels give identical results."""
    case = load_golden("search_mix10k")
    arrays, ep, ml = case_arrays(case, "mix10k")
    index = _index(arrays, ep, ml, "l2", 16)
    g = index.device_graph
    q = case["queries"]
    for ef in (16, 128):
        ids, dists, ctr = g.search(q, 10, ef, dist_mode=mode)
        np.testing.assert_array_equal(ids.cpu().numpy(), case[f"ids_m0_ef{ef}"])
        np.testing.assert_array_equal(dists.cpu().numpy(), case[f"dists_m0_ef{ef}"])
        np.testing.assert_array_equal(ctr.sum(0).cpu().numpy(), case[f"ctr_m0_ef{ef}"])


def test_device_mode_choice_equals_host_choice() -> None:
    """The arithmetic chosen from device-resident queries is the one the host rules choose."""
    import torch

    case = load_golden("search_mix10k")
    arrays, ep, ml = case_arrays(case, "mix10k")
    g = _index(arrays, ep, ml, "l2", 16).device_graph
    q = case["queries"].astype(np.float32)
    batches = [q, q + 0.5, q * 3.0, q - 40.0, q * 40.0, q[:0]]
    for b in batches:
        for codes in (False, True):
            if codes and g.codes is None:
                g.attach_codes(np.asarray(arrays["vectors"], dtype=np.uint8))
            dev = torch.from_numpy(np.ascontiguousarray(b, dtype=np.float64 if codes else np.float32)).cuda()
            host = g.choose_mode(b, codes) if b.size else g.choose_mode_device(dev, codes)
            assert g.choose_mode_device(dev, codes) == host
            if not codes:  # and from the statistics of the upload's host pass
                src = np.ascontiguousarray(b, dtype=np.float32)
                dst = torch.empty(src.shape, dtype=torch.float32, device="cuda")
                st = g.upload_queries(src, dst)
                assert g.mode_from_stats(st, src) == host
                assert torch.equal(dst.cpu(), torch.from_numpy(src))


def test_per_query_ef_matches_grouped_reference_calls() -> None:
    case = load_golden("search_mix10k")
    arrays, ep, ml = case_arrays(case, "mix10k")
    index = _index(arrays, ep, ml, "l2", 16)
    index.reset_counters()
    ids, dists = index.batch_search(case["queries"], k=10, ef=case["pq_ef"])
    np.testing.assert_array_equal(ids, case["pq_ids"])
    np.testing.assert_array_equal(dists, case["pq_dists"])
    st = index.stats()
    np.testing.assert_array_equal([st.distance_computations, st.hops], case["pq_ctr"])


@pytest.mark.parametrize("locality", [False, True], ids=["reference_order", "cell_order"])
@pytest.mark.parametrize("name", QUANT_CASES)
def test_quantized_search_and_fused_rerank_match_reference(name: str, locality: bool) -> None:
    from hnsw_engine_b200 import QuantizedIndex

    case = load_golden(f"quant_{name}")
    arrays, ep, ml = case_arrays(case, name)
    metric = str(case["metric"])
    M = (arrays["links0"].shape[1] - 1) // 2
    qi = QuantizedIndex(_index(arrays, ep, ml, metric, M, locality))
    for r in case["reranks"]:
        ids, dists = qi.batch_search(case["queries"], k=int(case["k"]), ef=int(case["ef"]), rerank=int(r))
        np.testing.assert_array_equal(ids, case[f"ids_r{r}"], err_msg=f"{name} r{r}")
        np.testing.assert_array_equal(dists, case[f"dists_r{r}"])


@pytest.mark.parametrize("locality", [False, True], ids=["reference_order", "cell_order"])
def test_fused_rerank_of_byte_and_non_byte_queries_matches_oracle(locality: bool) -> None:
    """Fused rerank on a graph holding a byte copy of its vectors: query rows whose values are all
    bytes are re-scored in integers, the others (every second row shifted by 0.25) in float64.
    Both equal the reference's two steps (the code search's candidates, then the float64 re-score,
    numba_engine.py:506-530) run by the oracle."""
    from hnsw_engine_b200 import QuantizedIndex
    from oracle import cpu

    case = load_golden("search_mix10k")
    arrays, ep, ml = case_arrays(case, "mix10k")
    q = np.ascontiguousarray(case["queries"][:64], dtype=np.float32)
    q[1::2] += 0.25
    qi = QuantizedIndex(_index(arrays, ep, ml, "l2", 16, locality))
    ids, dists = qi.batch_search(q, k=10, ef=64, rerank=64)
    codes = qi.quantizer.encode(np.asarray(arrays["vectors"], dtype=np.float32))
    code_q = qi.quantizer.transform_queries(q, "l2")
    cand, _, _ = cpu.search_batch(arrays, ep, ml, code_q, 64, 64, "l2", codes=codes, threads=8)
    o_ids, o_d = cpu.rerank_batch(np.asarray(arrays["vectors"], dtype=np.float32), q, cand, 10, "l2",
                                  threads=8)
    np.testing.assert_array_equal(ids, o_ids)
    np.testing.assert_array_equal(dists, o_d)


@pytest.mark.parametrize("name", ["int_l2", "cont_l2", "cont_ip", "cont_cosine", "mix10k_filtered"])
def test_single_query_search_matches_reference_fixtures(name: str) -> None:
    """HNSWIndex.search, one query at a time (the latency path when unfiltered), against the
    reference's outputs row by row (its search is its batch path on one row, index.py:244-273),
    with the work counters summed over the rows."""
    case = load_golden(f"search_{name}")
    arrays, ep, ml = case_arrays(case, name)
    metric = str(case["metric"])
    M = (arrays["links0"].shape[1] - 1) // 2
    index = _index(arrays, ep, ml, metric, M)
    k = int(case["k"])
    rows = range(min(40, case["queries"].shape[0]))
    for mi, mask, ef in iter_search_runs(case):
        index.reset_counters()
        for row in rows:
            ids, dists = index.search(case["queries"][row], k=k, ef=ef, filter=mask)
            np.testing.assert_array_equal(ids, case[f"ids_m{mi}_ef{ef}"][row],
                                          err_msg=f"{name} m{mi} ef{ef} row {row}")
            np.testing.assert_array_equal(dists, case[f"dists_m{mi}_ef{ef}"][row])
        if len(rows) == case["queries"].shape[0]:
            st = index.stats()
            np.testing.assert_array_equal([st.distance_computations, st.hops],
                                          case[f"ctr_m{mi}_ef{ef}"])


def test_device_queries_are_checked_like_host_queries() -> None:
    """CUDA-tensor queries get the host validator's checks and messages (_validation.py:28-40,
    metrics.py:42-68): NaN/inf, width, dtype, cosine zero rows."""
    import torch

    case = load_golden("search_cont_l2")
    arrays, ep, ml = case_arrays(case, "cont_l2")
    index = _index(arrays, ep, ml, "l2", 8)
    q = np.ascontiguousarray(case["queries"], dtype=np.float32)
    want = index.batch_search(q, k=10, ef=30)
    for dtype in (torch.float32, torch.float64):
        got = index.batch_search(torch.from_numpy(q).to("cuda", dtype), k=10, ef=30)
        for a, b in zip(want, got, strict=True):
            np.testing.assert_array_equal(a, b.cpu().numpy())
        for bad_value in (np.nan, np.inf, -np.inf):
            bad = torch.from_numpy(q).to("cuda", dtype)
            bad[3, 1] = bad_value
            with pytest.raises(ValueError, match="vectors contains NaN or infinite values"):
                index.batch_search(bad, k=10, ef=30)
    with pytest.raises(ValueError, match="expected 10"):
        index.batch_search(torch.zeros((2, 9), device="cuda"), k=10, ef=30)
    with pytest.raises(ValueError, match="2-D"):
        index.batch_search(torch.zeros(10, device="cuda"), k=10, ef=30)
    with pytest.raises(ValueError, match="real numbers"):
        index.batch_search(torch.zeros((2, 10), dtype=torch.bool, device="cuda"), k=10, ef=30)
    cos = load_golden("search_cont_cosine")
    arrays, ep, ml = case_arrays(cos, "cont_cosine")
    cindex = _index(arrays, ep, ml, "cosine", (arrays["links0"].shape[1] - 1) // 2)
    zero = torch.from_numpy(np.ascontiguousarray(cos["queries"][:4], dtype=np.float32)).cuda()
    zero[2] = 0.0
    with pytest.raises(ValueError, match=r"zero vectors \(rows \[2\]\)"):
        cindex.batch_search(zero, k=10, ef=30)


def test_host_query_forms_agree_and_reject_nan_alike() -> None:
    """Contiguous float32 host queries are copied to the GPU as they are and checked there; other
    dtypes and layouts are checked and prepared on the host. Same results, same error."""
    case = load_golden("search_cont_l2")
    arrays, ep, ml = case_arrays(case, "cont_l2")
    index = _index(arrays, ep, ml, "l2", 8)
    q = np.ascontiguousarray(case["queries"], dtype=np.float32)
    want = index.batch_search(q, k=10, ef=30)
    for form in (q.astype(np.float64), np.asfortranarray(q), q.tolist()):
        for a, b in zip(want, index.batch_search(form, k=10, ef=30), strict=True):
            np.testing.assert_array_equal(a, b)
    mask = np.zeros(arrays["vectors"].shape[0], dtype=bool)
    mask[:5] = True
    for bad_value in (np.nan, np.inf):
        bad = q.copy()
        bad[3, 1] = bad_value
        for form in (bad, bad.astype(np.float64)):
            with pytest.raises(ValueError, match="vectors contains NaN or infinite values"):
                index.batch_search(form, k=10, ef=30)
            with pytest.raises(ValueError, match="vectors contains NaN or infinite values"):
                index.batch_search(form, k=10, ef=30, filter=mask, exact_below=0.05)


def test_all_false_filter_pads_without_searching() -> None:
    case = load_golden("search_int_l2")
    arrays, ep, ml = case_arrays(case, "int_l2")
    index = _index(arrays, ep, ml, "l2", 6)
    index.reset_counters()
    ids, dists = index.batch_search(case["queries"][:4], k=3, filter=np.zeros(1500, dtype=bool))
    assert (ids == -1).all() and np.isinf(dists).all()
    assert index.stats().distance_computations == 0


def test_all_true_filter_takes_the_unfiltered_steps() -> None:
    case = load_golden("search_cont_l2")
    arrays, ep, ml = case_arrays(case, "cont_l2")
    index = _index(arrays, ep, ml, "l2", 8)
    index.reset_counters()
    plain = index.batch_search(case["queries"], k=10, ef=30)
    c_plain = (index.distance_computations, index.hops)
    index.reset_counters()
    filt = index.batch_search(case["queries"], k=10, ef=30, filter=np.ones(1500, dtype=bool))
    for a, b in zip(plain, filt, strict=True):
        np.testing.assert_array_equal(a, b)
    assert (index.distance_computations, index.hops) == c_plain


def _oracle_compare(arrays, ep, ml, metric, queries, k, ef, mask=None, codes=None):
    from oracle import cpu

    index = _index(arrays, ep, ml, metric, (arrays["links0"].shape[1] - 1) // 2)
    g = index.device_graph
    if codes is not None:
        g.attach_codes(codes)
    ids, dists, ctr = g.search(queries, k, ef, allowed=mask, use_codes=codes is not None)
    o_ids, o_d, o_c = cpu.search_batch(arrays, ep, ml, queries, k, ef, metric, allowed=mask,
                                       codes=codes, threads=8)
    np.testing.assert_array_equal(ids.cpu().numpy(), o_ids)
    np.testing.assert_array_equal(dists.cpu().numpy(), o_d)
    np.testing.assert_array_equal(ctr.cpu().numpy(), o_c)


def _workload(name: str):
    from hnsw_engine_b200 import graphs

    if not graphs.available(name):
        pytest.skip(f"graph {name} not built")
    meta, arrays = graphs.open_workload(name)
    return arrays, int(meta["entry_point"]), int(meta["max_level"]), meta["params"]["metric"]


def test_start_order_changes_no_result() -> None:
    """Large batches on a cell-ordered graph start longest-predicted first (a priority array the
    library sorts into the first work list): ids, distances and counters equal row order's, before
    and after the per-cell costs are learned, and under arbitrary priorities."""
    import torch

    from hnsw_engine_b200 import graphs
    from hnsw_engine_b200.schedule import MIN_QUERIES
    from hnsw_engine_b200.validation import prepare

    arrays, ep, ml, metric = _workload("mix100k")
    g = _index(arrays, ep, ml, metric, 16).device_graph
    assert g._schedule is not None
    q = torch.from_numpy(prepare(graphs.workload_queries("mix100k", nq=MIN_QUERIES + 904), metric)).cuda()
    g.schedule = False
    want = [t.cpu() for t in g.search(q, 10, 64)]
    g.schedule = True
    sched = g._schedule
    for _ in range(3):  # the first batch starts in row order, the next ones by the learned costs
        for a, b in zip(want, [t.cpu() for t in g.search(q, 10, 64)], strict=True):
            assert torch.equal(a, b)
    assert float(sched.cost[2].sum()) == 3 * q.shape[0]  # plain query counts
    ef = torch.full((q.shape[0],), 64, dtype=torch.int32, device=q.device)
    assert torch.unique(sched.start(q, ef)[1]).numel() > 1
    sched.cost[0].copy_(torch.rand_like(sched.cost[0]) * 300)  # arbitrary, partly clamped priorities
    sched.cost[2].fill_(1.0)
    for a, b in zip(want, [t.cpu() for t in g.search(q, 10, 64)], strict=True):
        assert torch.equal(a, b)
    # filtered batches follow the order without learning from it; code-space batches (with a
    # fused rerank) take their cells from the float32 rerank queries
    mask = np.random.default_rng(4).random(arrays["vectors"].shape[0]) < 0.3
    g.attach_codes(np.asarray(arrays["vectors"], dtype=np.uint8))  # integer 0..255: lossless
    runs = {"filtered": dict(allowed=mask),
            "codes": dict(use_codes=True, k_search=64, rerank_queries=q)}
    for name, kw in runs.items():
        qq = q.double() if name == "codes" else q
        g.schedule = False
        row_order = [t.cpu() for t in g.search(qq, 10, 64, **kw)]
        g.schedule = True
        before = sched.cost.clone()
        started = [t.cpu() for t in g.search(qq, 10, 64, **kw)]
        assert g.last_launches >= 2, name  # the priority kernel ran
        for a, b in zip(row_order, started, strict=True):
            assert torch.equal(a, b), name
        if name == "filtered":
            assert torch.equal(sched.cost, before)


def test_overflow_retries_keep_results_in_start_order() -> None:
    """A filtered batch told its filter allows every node (allowed_fraction = 1) gets scratch sized
    for an unfiltered search: most queries overflow their candidate spill or visited set, are
    flagged (never written past) and re-run with four times the scratch. The results equal those of
    a batch sized for its real selectivity, with the start order on."""
    import torch

    from hnsw_engine_b200 import graphs
    from hnsw_engine_b200.engine import pack_mask
    from hnsw_engine_b200.schedule import MIN_QUERIES
    from hnsw_engine_b200.validation import prepare

    arrays, ep, ml, metric = _workload("mix100k")
    g = _index(arrays, ep, ml, metric, 16).device_graph
    q = torch.from_numpy(prepare(graphs.workload_queries("mix100k", nq=MIN_QUERIES), metric)).cuda()
    mask = np.random.default_rng(6).random(arrays["vectors"].shape[0]) < 0.02
    g.search(q, 10, 64)  # learn some cell costs, so the filtered batches start in an order
    want = [t.cpu() for t in g.search(q, 10, 64, allowed=mask)]
    bits = torch.from_numpy(pack_mask(g.internal_mask(mask)).view(np.int32)).cuda()
    got = [t.cpu() for t in g.search(q, 10, 64, allowed=bits, allowed_fraction=1.0)]
    assert g.last_launches > 3  # overflowed queries were collected and searched again
    for a, b in zip(want, got, strict=True):
        assert torch.equal(a, b)


def test_start_order_without_cell_order_changes_no_result() -> None:
    """A large float graph kept in the reference node order (locality=False; by default it gets the
    cell order like any large graph) gets pivots for the start order alone; fixed and per-query ef
    give row order's ids, distances and counters."""
    import torch

    from hnsw_engine_b200 import graphs, synthetic
    from hnsw_engine_b200.schedule import MIN_QUERIES
    from hnsw_engine_b200.validation import prepare

    arrays, ep, ml, metric = _workload("t100k")
    assert _index(arrays, ep, ml, metric, 16).device_graph.locality
    g = _index(arrays, ep, ml, metric, 16, locality=False).device_graph
    assert g._schedule is not None and not g.locality
    q = torch.from_numpy(prepare(graphs.workload_queries("t100k", nq=MIN_QUERIES), metric)).cuda()
    pq = torch.from_numpy(synthetic.per_query_ef(MIN_QUERIES, seed=3, low=16, high=128)).cuda()
    for ef in (48, pq):
        g.schedule = False
        want = [t.cpu() for t in g.search(q, 10, ef)]
        g.schedule = True
        for _ in range(2):
            for a, b in zip(want, [t.cpu() for t in g.search(q, 10, ef)], strict=True):
                assert torch.equal(a, b)
    assert float(g._schedule.cost[2].sum()) == 4 * MIN_QUERIES


@pytest.mark.parametrize("name", ["mix100k", "t100k"])
def test_large_graph_per_query_ef_matches_oracle(name: str) -> None:
    from hnsw_engine_b200 import graphs, synthetic
    from hnsw_engine_b200.validation import prepare

    arrays, ep, ml, metric = _workload(name)
    q = prepare(graphs.workload_queries(name, nq=400), metric)
    ef = synthetic.per_query_ef(400, seed=5, low=32, high=512)
    _oracle_compare(arrays, ep, ml, metric, q, 10, ef)


@pytest.mark.parametrize("p", [0.5, 0.1, 0.01])
@pytest.mark.parametrize("kind", ["bernoulli", "prefix"])
def test_large_graph_filtered_matches_oracle(p: float, kind: str) -> None:
    from hnsw_engine_b200 import graphs, synthetic

    arrays, ep, ml, metric = _workload("mix100k")
    n = arrays["vectors"].shape[0]
    mask = synthetic.bernoulli_mask(n, p) if kind == "bernoulli" else synthetic.prefix_mask(n, p)
    q = graphs.workload_queries("mix100k", nq=48 if p >= 0.1 else 16)
    _oracle_compare(arrays, ep, ml, metric, q, 10, 64, mask=mask)


def test_large_graph_codes_cosine_match_oracle() -> None:
    from hnsw_engine_b200 import graphs
    from hnsw_engine_b200.quantization import ScalarQuantizer
    from hnsw_engine_b200.validation import prepare

    arrays, ep, ml, metric = _workload("t100k")
    quant = ScalarQuantizer.fit(arrays["vectors"])
    codes = quant.encode(arrays["vectors"])
    q = quant.transform_queries(prepare(graphs.workload_queries("t100k", nq=200), metric), metric)
    _oracle_compare(arrays, ep, ml, metric, q, 10, 128, codes=codes)


def test_large_graph_codes_in_cell_order_match_oracle() -> None:
    """Byte codes on the cell-ordered 100K graph (codes permuted with the rows, internal ids in
    the links, original ids in results and ties), with and without a filter."""
    from hnsw_engine_b200 import graphs, synthetic
    from hnsw_engine_b200.quantization import ScalarQuantizer
    from hnsw_engine_b200.validation import prepare

    arrays, ep, ml, metric = _workload("mix100k")
    quant = ScalarQuantizer.fit(arrays["vectors"])
    codes = quant.encode(arrays["vectors"])
    q = quant.transform_queries(prepare(graphs.workload_queries("mix100k", nq=200), metric), metric)
    _oracle_compare(arrays, ep, ml, metric, q, 10, 96, codes=codes)
    mask = synthetic.bernoulli_mask(arrays["vectors"].shape[0], 0.3)
    _oracle_compare(arrays, ep, ml, metric, q[:64], 10, 48, mask=mask, codes=codes)


@pytest.mark.parametrize("name", ["mix1m", "t1m"])
def test_million_node_graphs_match_oracle(name: str) -> None:
    """The 1M-node workloads (integer L2 and float cosine): ids, distances and counters equal the
    CPU oracle's for a sample of queries at per-query efSearch in 32..512."""
    from hnsw_engine_b200 import graphs, synthetic
    from hnsw_engine_b200.validation import prepare

    arrays, ep, ml, metric = _workload(name)
    q = prepare(graphs.workload_queries(name, nq=96), metric)
    ef = synthetic.per_query_ef(96, seed=6, low=32, high=512)
    _oracle_compare(arrays, ep, ml, metric, q, 10, ef)


@pytest.mark.parametrize("allowed_count", [3, 100])
def test_selective_filter_planner_returns_the_exact_allowed_neighbors(allowed_count: int) -> None:
    """Below the planner's selectivity the batch is answered exactly over the allowed rows: ids and
    distances equal the CPU oracle's exact search of that subset, padded when fewer than k."""
    from oracle import exact

    case = load_golden("search_mix10k")
    arrays, ep, ml = case_arrays(case, "mix10k")
    index = _index(arrays, ep, ml, "l2", 16)
    rng = np.random.default_rng(3)
    mask = np.zeros(arrays["vectors"].shape[0], dtype=bool)
    mask[rng.choice(mask.size, allowed_count, replace=False)] = True
    q = case["queries"][:64]
    index.reset_counters()
    ids, dists = index.batch_search(q, k=10, ef=64, filter=mask, exact_below=0.05)
    sub = np.flatnonzero(mask)
    kk = min(10, allowed_count)
    o_ids, o_d = exact.exact_search(np.asarray(arrays["vectors"])[sub], q, kk, "l2")
    np.testing.assert_array_equal(ids[:, :kk], sub[o_ids])
    np.testing.assert_array_equal(dists[:, :kk], o_d)
    assert (ids[:, kk:] == -1).all() and np.isinf(dists[:, kk:]).all()
    assert index.distance_computations == q.shape[0] * allowed_count
    # above the cutoff the graph walk answers, as the reference does
    g_ids, _ = index.batch_search(q, k=10, ef=64, filter=mask, exact_below=allowed_count / mask.size)
    ref_ids, _ = index.batch_search(q, k=10, ef=64, filter=mask)
    np.testing.assert_array_equal(g_ids, ref_ids)


@pytest.mark.parametrize("name", QUANT_CASES)
def test_device_quantizer_equals_the_reference_codes(name: str) -> None:
    """Fit and encode on the GPU give the reference's offset, step and codes bit for bit."""
    from hnsw_engine_b200 import QuantizedIndex
    from hnsw_engine_b200.quantization import ScalarQuantizer

    case = load_golden(f"quant_{name}")
    arrays, ep, ml = case_arrays(case, name)
    metric = str(case["metric"])
    M = (arrays["links0"].shape[1] - 1) // 2
    qi = QuantizedIndex(_index(arrays, ep, ml, metric, M))
    np.testing.assert_array_equal(qi.quantizer.offset, case["offset"])  # the reference's fit
    assert qi.quantizer.step == float(case["step"])
    vectors = np.asarray(qi._index.native_arrays()["vectors"])
    np.testing.assert_array_equal(qi.codes, ScalarQuantizer(case["offset"], float(case["step"])).encode(vectors))
    if "codes" in case:  # the reference's own codes
        np.testing.assert_array_equal(qi.codes, case["codes"])
