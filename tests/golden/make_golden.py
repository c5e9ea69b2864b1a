"""Generate the golden fixtures under ``tests/golden/`` by running the reference implementation.

The reference (anamankev/hnsw-engine, pure Python + Numba) is importable only where it is checked
out, so its outputs are frozen here as small ``.npz`` files that travel with the tests. Every case
records the reference-built graph (native arrays), the inputs, and the reference's outputs
including the per-call work counters.

Cases follow the reference's own test fixtures:

* bit-identical integer data, filtered at selectivity 1.0 / 0.5 / 0.1 / 0.01 with ef 10 and 50
  (``tests/test_numba_engine.py:37-49, 187-204``);
* continuous data under l2 / ip / cosine with identical ids (``tests/test_numba_engine.py:52-63``);
* the exactness regime, complete graph with ef = n (``tests/test_index.py:157-182, 458-472``);
* padding on a disconnected graph (``tests/test_numba_engine.py:149-162``);
* the 10K x 128 mixture workload at ef 16..256, filtered and with a per-query ef;
* int8 code-space search with and without exact re-rank (``tests/test_quantization.py:69-108``);
* exact brute-force known answers (``tests/test_oracle.py:9-115``).

Usage::

    NUMBA_CACHE_DIR=/tmp/numba python tests/golden/make_golden.py --reference-src <ref>/src
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from hnsw_engine_b200.graphs import workload_queries, workload_vectors  # noqa: E402

GRAPH_KEYS = ("levels", "links0", "count0", "upper_offset", "links_up", "count_up")


def _graph(index) -> dict[str, np.ndarray]:
    arrays = index._engine.native_arrays()
    return {k: np.ascontiguousarray(v) for k, v in arrays.items()}


def _search_case(index, name, queries, k, efs, masks, store_graph=True, per_query_ef=None):
    """Run the reference batch search for each (ef, mask) and store results plus counters.

    Without ``store_graph`` the case names a workload graph stored once in ``graph_<name>.npz``.
    """
    out: dict[str, np.ndarray] = {}
    arrays = _graph(index)
    if store_graph:
        for key in GRAPH_KEYS:
            out[key] = arrays[key]
        out["vectors"] = arrays["vectors"]
    out["entry_point"] = np.int64(index.entry_point)
    out["max_level"] = np.int64(index.max_level)
    out["metric"] = np.array(index.metric)
    out["M"] = np.int64(index.M)
    out["queries"] = np.ascontiguousarray(queries, dtype=np.float32)
    out["k"] = np.int64(k)
    out["efs"] = np.asarray(efs, dtype=np.int64)
    out["n_masks"] = np.int64(len(masks))
    for mi, mask in enumerate(masks):
        if mask is not None:
            out[f"mask{mi}"] = mask
        for ef in efs:
            index.reset_counters()
            ids, dists = index.batch_search(queries, k=k, ef=int(ef), filter=mask)
            st = index.stats()
            out[f"ids_m{mi}_ef{ef}"] = ids
            out[f"dists_m{mi}_ef{ef}"] = dists
            out[f"ctr_m{mi}_ef{ef}"] = np.array([st.distance_computations, st.hops], np.int64)
    if per_query_ef is not None:  # reference takes a scalar ef: one call per distinct value
        nq = queries.shape[0]
        ids = np.empty((nq, k), np.int64)
        dists = np.empty((nq, k), np.float64)
        index.reset_counters()
        for ef in np.unique(per_query_ef):
            rows = np.flatnonzero(per_query_ef == ef)
            a, b = index.batch_search(queries[rows], k=k, ef=int(ef))
            ids[rows], dists[rows] = a, b
        st = index.stats()
        out["pq_ef"] = per_query_ef.astype(np.int32)
        out["pq_ids"] = ids
        out["pq_dists"] = dists
        out["pq_ctr"] = np.array([st.distance_computations, st.hops], np.int64)
    np.savez_compressed(HERE / f"search_{name}.npz", **out)
    print("search", name, {k: v.shape for k, v in out.items() if k.startswith("ids_")})


def _quant_case(index, name, queries, k, ef, reranks, store_graph=True):
    from hnsw_engine import QuantizedIndex

    qi = QuantizedIndex(index)
    out: dict[str, np.ndarray] = {}
    arrays = _graph(index)
    if store_graph:
        for key in GRAPH_KEYS:
            out[key] = arrays[key]
        out["vectors"] = arrays["vectors"]
    out["entry_point"] = np.int64(index.entry_point)
    out["max_level"] = np.int64(index.max_level)
    out["metric"] = np.array(index.metric)
    out["queries"] = np.ascontiguousarray(queries, dtype=np.float32)
    out["k"] = np.int64(k)
    out["ef"] = np.int64(ef)
    if store_graph:
        out["codes"] = qi.codes
    out["offset"] = qi.quantizer.offset
    out["step"] = np.float64(qi.quantizer.step)
    out["reranks"] = np.asarray(reranks, np.int64)
    for r in reranks:
        ids, dists = qi.batch_search(queries, k=k, ef=ef, rerank=r)
        out[f"ids_r{r}"] = ids
        out[f"dists_r{r}"] = dists
    np.savez_compressed(HERE / f"quant_{name}.npz", **out)
    print("quant", name, reranks)


def _exact_cases():
    from hnsw_engine import exact_search

    cases = []
    cases.append(("hand_l2", np.array([[0, 0], [1, 0], [0, 2], [3, 3]], np.float32),
                  np.array([[0.0, 0.0]]), 3, "l2"))
    for metric in ("ip", "cosine"):
        cases.append((f"hand_{metric}", np.array([[1, 0], [0, 3], [2, 2]], np.float32),
                      np.array([[1.0, 1.0]]), 3, metric))
    cases.append(("duplicates", np.array([[5, 5], [1, 1], [5, 5], [1, 1], [9, 9]], np.float32),
                  np.array([[1.0, 1.0], [5.0, 5.0]]), 4, "l2"))
    cases.append(("ties", np.array([[9, 9], [0, -1], [1, 0], [-1, 0], [0, 1]], np.float32),
                  np.zeros((1, 2)), 4, "l2"))
    cases.append(("tie_kth", np.array([[2, 0], [0, 0], [-2, 0], [0, 2]], np.float32),
                  np.array([[0.0, 0.0]]), 2, "l2"))
    rng = np.random.default_rng(7)
    data = rng.integers(1, 5, size=(80, 4)).astype(np.float32)
    queries = rng.integers(1, 5, size=(15, 4)).astype(np.float32)
    for metric in ("l2", "ip", "cosine"):
        cases.append((f"int_{metric}", data, queries, 10, metric))
    rng = np.random.default_rng(11)
    data = rng.standard_normal((200, 6)).astype(np.float32)
    queries = rng.standard_normal((10, 6)).astype(np.float32)
    for metric in ("l2", "ip", "cosine"):
        cases.append((f"float_{metric}", data, queries, 7, metric))
    rng = np.random.default_rng(3)
    data = (1e4 + rng.integers(0, 4, size=(300, 8))).astype(np.float32)
    queries = (1e4 + rng.integers(0, 4, size=(20, 8)) + 0.5).astype(np.float32)
    cases.append(("cancellation", data, queries, 5, "l2"))
    cases.append(("uint8", np.array([[0, 0], [3, 4], [1, 1]], np.uint8),
                  np.array([[0, 0]], np.uint8), 3, "l2"))
    mix = workload_vectors("mix10k")
    mq = workload_queries("mix10k")[:200]
    cases.append(("mix10k_k100", mix, mq, 100, "l2"))
    out: dict[str, np.ndarray] = {}
    names = []
    for name, data, queries, k, metric in cases:
        ids, dists = exact_search(data, queries, k, metric)
        names.append(name)
        if name != "mix10k_k100":
            out[f"{name}_data"] = data
        out[f"{name}_queries"] = queries
        out[f"{name}_k"] = np.int64(k)
        out[f"{name}_metric"] = np.array(metric)
        out[f"{name}_ids"] = ids
        out[f"{name}_dists"] = dists
    out["names"] = np.array(names)
    np.savez_compressed(HERE / "exact.npz", **out)
    print("exact", names)


def per_query_counters_case(rows: int = 200, ef: int = 192) -> None:
    """The reference's own work counters query by query: one ``HNSWIndex.search`` per query on the
    10K mixture graph at ef = 192 (the efSearch of the 1M benchmark's plain operating point), the
    counters reset before each call. ``search_mix10k_counters.npz``."""
    import tempfile

    from hnsw_engine import HNSWIndex

    from hnsw_engine_b200.graphs import graph_dir, stored_vectors

    src = graph_dir("mix10k")
    with tempfile.TemporaryDirectory() as tmp:  # the graph directory ships without vectors.npy
        for f in src.iterdir():
            if f.is_file():
                (Path(tmp) / f.name).symlink_to(f)
        if not (src / "vectors.npy").is_file():
            np.save(Path(tmp) / "vectors.npy", stored_vectors("mix10k"))
        index = HNSWIndex.load_native(tmp, mmap=False)
    q = workload_queries("mix10k")[:rows]
    ids = np.empty((rows, 10), np.int64)
    dists = np.empty((rows, 10), np.float64)
    ctr = np.empty((rows, 2), np.int64)
    for r in range(rows):
        index.reset_counters()
        ids[r], dists[r] = index.search(q[r], k=10, ef=ef)
        st = index.stats()
        ctr[r] = (st.distance_computations, st.hops)
    np.savez_compressed(HERE / "search_mix10k_counters.npz", queries=q, ef=np.int64(ef), ids=ids,
                        dists=dists, counters=ctr)


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference-src", required=True)
    parser.add_argument("--only", choices=("per_query_counters",), default=None,
                        help="write only this fixture")
    args = parser.parse_args()
    sys.path.insert(0, args.reference_src)
    if args.only == "per_query_counters":
        per_query_counters_case()
        return
    from hnsw_engine import GraphState, HNSWIndex
    from hnsw_engine.synthetic import clustered, gaussian, small_integers

    # Integer data: bit-identical, filtered at four selectivities.
    data = small_integers(1500, 6, seed=21, high=5)
    queries = small_integers(50, 6, seed=22, high=5)
    masks = [None] + [np.random.default_rng(24).random(1500) < s for s in (1.0, 0.5, 0.1, 0.01)]
    for metric in ("l2", "ip"):
        index = HNSWIndex(6, metric=metric, M=6, ef_construction=40, seed=23)
        index.add(data)
        _search_case(index, f"int_{metric}", queries, 10, (10, 50), masks)

    # Continuous data under every metric (heuristic selection, as the reference default).
    data, queries = clustered(1500, 10, seed=4), clustered(80, 10, seed=5)
    mask = np.random.default_rng(0).random(1500) < 0.2
    for metric in ("l2", "ip", "cosine"):
        index = HNSWIndex(10, metric=metric, M=8, ef_construction=50, seed=6)
        index.add(data)
        _search_case(index, f"cont_{metric}", queries, 10, (10, 50), [None, mask])

    # Exactness regime: complete graph, ef = n.
    n = 60
    for metric in ("l2", "ip"):
        d = small_integers(n, 4, seed=8, high=5)
        q = small_integers(25, 4, seed=9, high=5)
        index = HNSWIndex(4, metric=metric, M=n, ef_construction=n, selection="simple", seed=1)
        index.add(d)
        allowed = np.random.default_rng(0).random(n) < 0.4
        _search_case(index, f"complete_{metric}", q, 10, (n,), [None, allowed])

    # Padding: a disconnected three-node graph.
    index = HNSWIndex(2, M=2, seed=0)
    vectors = np.array([[0, 0], [1, 0], [5, 5]], dtype=np.float32)
    state = GraphState.from_adjacency(vectors, np.zeros(3, np.int64), 0, 0, [{0: [1], 1: [0], 2: [0]}])
    index._engine.load_state(state)
    _search_case(index, "padding", np.array([[5.0, 5.0]], np.float32), 3, (10,),
                 [None, np.array([True, False, True])])

    # Fewer allowed than k, and the gaussian single/batch case.
    data = gaussian(300, 4, seed=6)
    index = HNSWIndex(4, M=6, seed=0)
    index.add(data)
    allowed = np.zeros(300, dtype=bool)
    allowed[[7, 70, 170]] = True
    _search_case(index, "few_allowed", data[[70, 7, 1]], 5, (10,), [None, allowed])

    # The 10K x 128 mixture workload (vectors regenerate from the seed; not stored).
    from hnsw_engine_b200 import synthetic

    index = HNSWIndex.load_native(HERE.parent.parent / "graphs" / "mix10k")
    g = _graph(index)
    np.savez_compressed(
        HERE / "graph_mix10k.npz",
        entry_point=np.int64(index.entry_point),
        max_level=np.int64(index.max_level),
        **{key: g[key] for key in GRAPH_KEYS},
    )
    q = workload_queries("mix10k")
    pq = synthetic.per_query_ef(q.shape[0], seed=11, low=16, high=256)
    masks = [None, synthetic.bernoulli_mask(10_000, 0.1, seed=12), synthetic.prefix_mask(10_000, 0.1)]
    _search_case(index, "mix10k", q, 10, (16, 32, 64, 128, 256), masks[:1], store_graph=False,
                 per_query_ef=pq)
    _search_case(index, "mix10k_filtered", q[:300], 10, (64,), masks, store_graph=False)

    # Quantized: lossless integer codes; lossy codes under cosine and ip.
    _quant_case(index, "mix10k", q[:300], 10, 32, (0, 40), store_graph=False)
    data, queries = clustered(1500, 10, seed=4), clustered(80, 10, seed=5)
    for metric in ("cosine", "ip", "l2"):
        idx = HNSWIndex(10, metric=metric, M=8, ef_construction=50, seed=6)
        idx.add(data if metric != "l2" else gaussian(1500, 10, seed=4) * 3.0)
        _quant_case(idx, f"cont_{metric}", queries, 10, 40, (0, 50))

    _exact_cases()
    per_query_counters_case()


if __name__ == "__main__":
    main()
