"""The allocation-free search entry point gives the same results as the regular one.

``hnsw_b200_search_noalloc`` serves callers that may not allocate device memory: real-time serving
loops where an allocation would stall the loop, plugins whose host owns every device allocation,
processes under a hard memory budget. It runs the same kernel with its working memory in a fixed
array inside the library. This file is collected last so that a failure here never hides the other
tests, and it passes in a fresh process as well as after them.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import load_golden, mix10k_arrays


def _args(q, ef_t, k, outs, dist_mode):
    from hnsw_engine_b200 import _lib

    ids, dists, ctr = outs
    return _lib.SearchArgs(
        queries=q.data_ptr(), queries_f64=0, use_codes=0, nq=q.shape[0], k=k, k_search=k,
        ef=ef_t.data_ptr(), ef_max=int(ef_t.max().item()), dist_mode=dist_mode, allowed=None,
        allowed_fraction=1.0, rerank_queries=None, out_ids=ids.data_ptr(),
        out_dists=dists.data_ptr(), out_counters=ctr.data_ptr(), stop_mlp=None,
        stop_threshold=0.0, trace_cap=0, trace_feat=None, trace_dk=None, trace_count=None,
        trace_hops=None,
    )


def _outs(nq: int, k: int, fill_ids: int = 7):
    import torch

    return (torch.full((nq, k), fill_ids, dtype=torch.int64, device="cuda"),
            torch.zeros((nq, k), dtype=torch.float64, device="cuda"),
            torch.zeros((nq, 2), dtype=torch.int64, device="cuda"))


@pytest.mark.gpu
@pytest.mark.parametrize("dist_mode", [0, 2])
def test_noalloc_search_matches_regular_search_twice(dist_mode: int) -> None:
    import torch

    from hnsw_engine_b200 import HNSWIndex, _lib

    arrays, ep, ml = mix10k_arrays()
    index = HNSWIndex.from_arrays(arrays, ep, ml, dim=128, metric="l2", M=16)
    g = index.device_graph
    lib = _lib.load()
    case = load_golden("search_mix10k")
    q = torch.from_numpy(case["queries"]).cuda()
    ef = torch.from_numpy(case["pq_ef"]).cuda()
    k = 10
    nq = q.shape[0]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ref = _outs(nq, k)
    a = _args(q, ef, k, ref, dist_mode)
    _lib.check(lib.hnsw_b200_search(g._handle, ctypes.byref(a), stream))
    graph = g._graph_struct()
    for call in range(2):  # the shared array keeps the previous call's contents
        out = _outs(nq, k)
        b = _args(q, ef, k, out, dist_mode)
        _lib.check(lib.hnsw_b200_search_noalloc(ctypes.byref(graph), ctypes.byref(b), stream))
        for x, y in zip(out, ref, strict=True):  # integer and exact float64 results: tolerance 0
            np.testing.assert_array_equal(x.cpu().numpy(), y.cpu().numpy(), err_msg=f"call {call}")
    np.testing.assert_array_equal(ref[0].cpu().numpy(), case["pq_ids"])


@pytest.mark.gpu
def test_noalloc_rejects_requests_beyond_its_limits() -> None:
    import torch

    from hnsw_engine_b200 import HNSWIndex, _lib

    arrays, ep, ml = mix10k_arrays()
    g = HNSWIndex.from_arrays(arrays, ep, ml, dim=128, metric="l2", M=16).device_graph
    lib = _lib.load()
    q = torch.zeros((1, 128), device="cuda")
    ef = torch.full((1,), 16, dtype=torch.int32, device="cuda")
    outs = _outs(1, 10)
    graph = g._graph_struct()
    a = _args(q, ef, 10, outs, 0)
    a.nq = (1 << 20) + 1  # more queries than the fixed status area holds: rejected before any launch
    assert lib.hnsw_b200_search_noalloc(ctypes.byref(graph), ctypes.byref(a), None) == _lib.EINVAL
    assert b"at most" in lib.hnsw_b200_last_error()
    a = _args(q, ef, 10, outs, 0)
    a.priority = ef.data_ptr()  # a start order is not supported: refused, not silently ignored
    assert lib.hnsw_b200_search_noalloc(ctypes.byref(graph), ctypes.byref(a), None) == _lib.EINVAL
    assert b"priority" in lib.hnsw_b200_last_error()


def test_noalloc_rejects_a_graph_too_large_for_its_array_before_any_gpu_work() -> None:
    """Host-only: a graph whose per-warp visited bitmap cannot fit the fixed array is refused by the
    size check, which runs before any CUDA call (the pointers are never dereferenced)."""
    from hnsw_engine_b200 import _lib, build

    build.build()
    lib = _lib.load()
    fake = 4096
    graph = _lib.Graph(vectors=fake, links0=fake, count0=fake, upper_offset=fake, n=(1 << 31) - 2,
                       dim=128, links0_stride=33, links_up_stride=17, metric=0, entry_point=0,
                       max_level=0)
    a = _lib.SearchArgs(queries=fake, nq=1, k=10, k_search=10, ef=fake, ef_max=16, dist_mode=0,
                        out_ids=fake, out_dists=fake, allowed_fraction=1.0)
    assert lib.hnsw_b200_search_noalloc(ctypes.byref(graph), ctypes.byref(a), None) == _lib.EINVAL
    assert b"needs more than the fixed" in lib.hnsw_b200_last_error()


def _chain_graph(path: int = 100, dummies: int = 14):
    """A graph whose upper layer is a long chain: path node i sits at x = 10 i and links to i - 1,
    i + 1 and `dummies` private far-away nodes. A greedy descent from the far end of the chain visits
    about (dummies + 1) nodes per hop, so queries near x = 0 outgrow a 1024-entry upper-layer hash."""
    n = path * (1 + dummies)
    vec = np.zeros((n, 4), np.float32)
    vec[:path, 0] = 10.0 * np.arange(path)
    links_up = np.full((n, 17), -1, np.int32)
    count_up = np.zeros(n, np.int32)
    links0 = np.full((n, 33), -1, np.int32)
    count0 = np.zeros(n, np.int32)
    for i in range(path):
        own = [path + i * dummies + j for j in range(dummies)]
        for j, d in enumerate(own):
            vec[d] = (10.0 * i, 10000.0 + j, 0.0, 0.0)
            links_up[d, 0] = i
            count_up[d] = 1
            links0[d, 0] = i
            count0[d] = 1
        nb = [x for x in (i - 1, i + 1) if 0 <= x < path]
        row = nb + own
        links_up[i, : len(row)] = row
        count_up[i] = len(row)
        links0[i, : len(nb)] = nb
        count0[i] = len(nb)
    arrays = {"vectors": vec, "levels": np.ones(n, np.int64), "links0": links0, "count0": count0,
              "upper_offset": np.arange(n, dtype=np.int64), "links_up": links_up,
              "count_up": count_up}
    return arrays, path - 1, 1


@pytest.mark.gpu
def test_noalloc_overflow_returns_eretry_and_keeps_the_other_queries_exact() -> None:
    import torch

    from hnsw_engine_b200 import _lib
    from hnsw_engine_b200.engine import DeviceGraph

    arrays, ep, ml = _chain_graph()
    g = DeviceGraph(arrays, ep, ml, "l2")
    lib = _lib.load()
    # x = 0 and 100 walk most of the chain (overflow); 970 and 990 start next to the entry point
    xs = np.array([0.0, 970.0, 100.0, 990.0], np.float32)
    q = torch.from_numpy(np.stack([xs, np.zeros(4), np.zeros(4), np.zeros(4)], 1)
                         .astype(np.float32)).cuda()
    ef = torch.full((4,), 10, dtype=torch.int32, device="cuda")
    k = 5
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ref = _outs(4, k)
    _lib.check(lib.hnsw_b200_search(g._handle, ctypes.byref(_args(q, ef, k, ref, 0)), stream))
    graph = g._graph_struct()
    sentinel = -7
    for _call in range(2):
        out = _outs(4, k, fill_ids=sentinel)
        rc = lib.hnsw_b200_search_noalloc(ctypes.byref(graph), ctypes.byref(_args(q, ef, k, out, 0)),
                                          stream)
        assert rc == _lib.ERETRY
        assert b"2 queries overflowed" in lib.hnsw_b200_last_error()
        ids = out[0].cpu().numpy()
        assert (ids[[0, 2]] == sentinel).all()  # overflowed queries are left unwritten
        for x, y in zip(out, ref, strict=True):
            np.testing.assert_array_equal(x.cpu().numpy()[[1, 3]], y.cpu().numpy()[[1, 3]])
    # the regular entry point retried the overflowed queries with a larger hash
    assert ref[0].cpu().numpy()[0, 0] == 0 and ref[0].cpu().numpy()[2, 0] == 10
