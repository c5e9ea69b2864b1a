"""The allocation-free search entry point gives the same results as the regular one.

``hnsw_b200_search_noalloc`` serves callers that may not allocate device memory (captured or
real-time serving loops, plugins whose host owns all device allocations, processes under a hard
memory budget): it runs the same kernel with its working memory in a fixed array inside the
library. This file is collected last so that a failure here never hides the other tests, and it
passes in a fresh process as well as after them.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import load_golden, mix10k_arrays

pytestmark = pytest.mark.gpu


def _args(g, q, ef_t, k, outs, dist_mode):
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
    ref = (torch.empty((nq, k), dtype=torch.int64, device="cuda"),
           torch.empty((nq, k), dtype=torch.float64, device="cuda"),
           torch.empty((nq, 2), dtype=torch.int64, device="cuda"))
    a = _args(g, q, ef, k, ref, dist_mode)
    _lib.check(lib.hnsw_b200_search(g._handle, ctypes.byref(a), stream))
    graph = g._graph_struct()
    for call in range(2):  # the shared array keeps the previous call's contents
        out = (torch.full((nq, k), 7, dtype=torch.int64, device="cuda"),
               torch.zeros((nq, k), dtype=torch.float64, device="cuda"),
               torch.zeros((nq, 2), dtype=torch.int64, device="cuda"))
        b = _args(g, q, ef, k, out, dist_mode)
        _lib.check(lib.hnsw_b200_search_noalloc(ctypes.byref(graph), ctypes.byref(b), stream))
        for x, y in zip(out, ref, strict=True):  # integer and exact float64 results: tolerance 0
            np.testing.assert_array_equal(x.cpu().numpy(), y.cpu().numpy(), err_msg=f"call {call}")
    np.testing.assert_array_equal(ref[0].cpu().numpy(), case["pq_ids"])


def test_noalloc_rejects_requests_beyond_its_limits() -> None:
    import torch

    from hnsw_engine_b200 import HNSWIndex, _lib

    arrays, ep, ml = mix10k_arrays()
    g = HNSWIndex.from_arrays(arrays, ep, ml, dim=128, metric="l2", M=16).device_graph
    lib = _lib.load()
    q = torch.zeros((1, 128), device="cuda")
    ef = torch.full((1,), 16, dtype=torch.int32, device="cuda")
    outs = (torch.empty((1, 10), dtype=torch.int64, device="cuda"),
            torch.empty((1, 10), dtype=torch.float64, device="cuda"),
            torch.empty((1, 2), dtype=torch.int64, device="cuda"))
    a = _args(g, q, ef, 10, outs, 0)
    a.nq = (1 << 20) + 1  # more queries than the fixed status area holds: rejected before any launch
    graph = g._graph_struct()
    rc = lib.hnsw_b200_search_noalloc(ctypes.byref(graph), ctypes.byref(a), None)
    assert rc == _lib.EINVAL
    assert b"at most" in lib.hnsw_b200_last_error()
