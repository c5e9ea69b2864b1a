"""The batched search recorded in a CUDA graph and replayed gives the synchronous search's ids,
distances and counters, batch after batch; the asynchronous entry point refuses to allocate."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import case_arrays, load_golden

pytestmark = pytest.mark.gpu


def _check_replays(g, batches, k, ef, stop=None) -> None:
    import torch

    from hnsw_engine_b200.engine import CapturedSearch

    cap = CapturedSearch(g, batches[0], k, ef, stop=stop)
    for b in batches + batches[:1]:  # a new batch each replay, then the first one again
        cap.queries.copy_(b)
        cap.replay()
        got = [t.cpu().numpy() for t in cap.results()]
        want = [t.cpu().numpy() for t in g.search(b, k, ef, stop=stop,
                                                  kernel_config=cap.kernel_config)]
        for x, y in zip(got, want, strict=True):
            np.testing.assert_array_equal(x, y)
    torch.cuda.synchronize()


def test_captured_search_matches_synchronous_search_small_graph() -> None:
    import torch

    from hnsw_engine_b200 import HNSWIndex

    case = load_golden("search_mix10k")
    arrays, ep, ml = case_arrays(case, "mix10k")
    g = HNSWIndex.from_arrays(arrays, ep, ml, dim=128, metric="l2", M=16).device_graph
    q = torch.from_numpy(case["queries"]).cuda()
    _check_replays(g, [q[:500].contiguous(), q[500:].contiguous()], 10, 64)
    ids = g.search(q[:500], 10, 64)[0].cpu().numpy()
    np.testing.assert_array_equal(ids, case["ids_m0_ef64"][:500])


def test_captured_search_with_start_order_and_learned_stop() -> None:
    import torch

    from hnsw_engine_b200 import HNSWIndex, graphs
    from hnsw_engine_b200.learned_stop import StopNetwork
    from hnsw_engine_b200.schedule import MIN_QUERIES
    from hnsw_engine_b200.validation import prepare

    if not graphs.available("mix100k"):
        pytest.skip("graph mix100k not built")
    meta, arrays = graphs.open_workload("mix100k")
    params = {k: v for k, v in meta["params"].items() if k != "engine"}
    g = HNSWIndex.from_arrays(arrays, int(meta["entry_point"]), int(meta["max_level"]),
                              **params).device_graph
    assert g._schedule is not None
    qs = [torch.from_numpy(prepare(graphs.workload_queries("mix100k", nq=MIN_QUERIES, seed=s), "l2")).cuda()
          for s in (1, 2)]
    _check_replays(g, qs, 10, 96)
    net = StopNetwork(g.device, seed=3)  # untrained weights still stop queries deterministically
    _check_replays(g, qs, 10, 96, stop=net.stop_args(0.5))


def test_async_search_needs_reserved_scratch() -> None:
    import torch

    from hnsw_engine_b200 import HNSWIndex, _lib

    case = load_golden("search_mix10k")
    arrays, ep, ml = case_arrays(case, "mix10k")
    g = HNSWIndex.from_arrays(arrays, ep, ml, dim=128, metric="l2", M=16).device_graph
    q = torch.from_numpy(case["queries"]).cuda()
    with pytest.raises(_lib.HnswB200Error, match="not reserved"):
        g.search(q, 10, 64, dist_mode=2, kernel_config=0, asynchronous=True)
    g.search(q, 10, 64, dist_mode=2, kernel_config=0)
    ids, _, _ = g.search(q, 10, 64, dist_mode=2, kernel_config=0, asynchronous=True)
    assert g.search_failed() == 0
    np.testing.assert_array_equal(ids.cpu().numpy(), case["ids_m0_ef64"])
    with pytest.raises(ValueError, match="dist_mode and kernel_config"):
        g.search(q, 10, 64, asynchronous=True)
