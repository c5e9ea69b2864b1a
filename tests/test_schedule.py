"""The start order's kernels against float64 NumPy references: each query's nearest pivot, the
priority read from the per-cell cost table, and the table the search kernel learns."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _start(piv: np.ndarray, q: np.ndarray, ef: np.ndarray, cost: np.ndarray | None = None):
    import torch

    from hnsw_engine_b200.schedule import CellSchedule

    s = CellSchedule(torch.from_numpy(np.ascontiguousarray(piv, dtype=np.float32)).cuda())
    if cost is not None:
        s.cost.copy_(torch.from_numpy(cost))
    cells, prio = s.start(torch.from_numpy(np.ascontiguousarray(q, dtype=np.float32)).cuda(),
                          torch.from_numpy(ef.astype(np.int32)).cuda())
    torch.cuda.synchronize()
    return cells.cpu().numpy(), prio.cpu().numpy()


def test_cells_are_the_nearest_pivots() -> None:
    rng = np.random.default_rng(0)
    piv = rng.standard_normal((300, 40)).astype(np.float32)  # two pivot groups, a partial chunk
    q = rng.standard_normal((1000, 40)).astype(np.float32)   # a partial block of queries
    cells, prio = _start(piv, q, np.full(1000, 50))
    d = ((q[:, None, :].astype(np.float64) - piv[None, :, :]) ** 2).sum(-1)
    chosen = d[np.arange(1000), cells]
    assert np.all(chosen <= d.min(1) * (1 + 1e-5) + 1e-6)  # float32 sums: equal up to rounding
    assert (prio == 0).all()  # nothing learned yet


def test_byte_valued_cells_are_exact_at_d128() -> None:
    # the benchmark's shape (256 pivots x 128 dimensions, pivots staged as 16-byte pieces):
    # byte-valued data make every float32 sum exact, so the cells equal the float64 argmin,
    # ties to the lower pivot
    rng = np.random.default_rng(5)
    piv = rng.integers(0, 256, (256, 128)).astype(np.float32)
    piv[17] = piv[3]  # a tied pair
    q = rng.integers(0, 256, (700, 128)).astype(np.float32)
    q[:5] = piv[3]
    cells, _ = _start(piv, q, np.full(700, 64))
    d = ((q[:, None, :].astype(np.float64) - piv[None, :, :]) ** 2).sum(-1)
    assert cells.tolist() == d.argmin(1).tolist()
    assert (cells[:5] == 3).all()


def test_equal_distances_pick_the_lower_pivot() -> None:
    piv = np.array([[0, 0], [1, 0], [0, 0], [1, 0]], np.float32)
    q = np.array([[0, 0], [1, 0], [0.5, 0]], np.float32)
    cells, _ = _start(piv, q, np.full(3, 10))
    assert cells.tolist() == [0, 1, 0]


def test_priority_is_the_cell_ratio_times_ef() -> None:
    from hnsw_engine_b200.schedule import PRIORITY_SCALE

    piv = np.array([[0, 0], [10, 0], [0, 10]], np.float32)
    # plain sums, stopped sums, plain counts, stopped counts; cell 2 has only stopped searches
    cost = np.array([[2.2, 8.0, 0.0], [0.0, 0.0, 6.0], [2.0, 2.0, 0.0], [0.0, 0.0, 3.0]])
    q = piv[[0, 1, 2, 1]]
    ef = np.array([100, 100, 100, 50])
    _, prio = _start(piv, q, ef, cost)
    ratio = [1.1, 4.0, 2.0, 4.0]
    assert prio.tolist() == [int(r * e * PRIORITY_SCALE) for r, e in zip(ratio, ef, strict=True)]
    cost[0, 1] = 1e9  # clamped to the 16-bit key range
    _, prio = _start(piv, q, ef, cost)
    assert prio[1] == 65535 and prio[3] == 65535


def test_search_learns_the_cost_table() -> None:
    """Every finished query adds hops / ef and 1 to its cell, in the plain or the stopped half."""
    import torch

    from hnsw_engine_b200 import graphs
    from hnsw_engine_b200.schedule import MIN_QUERIES
    from hnsw_engine_b200.validation import prepare
    from test_search_gpu import _index, _workload

    arrays, ep, ml, metric = _workload("mix100k")
    g = _index(arrays, ep, ml, metric, 16).device_graph
    s = g._schedule
    q = torch.from_numpy(prepare(graphs.workload_queries("mix100k", nq=MIN_QUERIES), metric)).cuda()
    ef = torch.randint(20, 120, (q.shape[0],), dtype=torch.int32, device="cuda")
    s.reset()
    cells, _ = s.start(q, ef)
    _, _, ctr = g.search(q, 10, ef)
    want = torch.zeros(s.n_cells, dtype=torch.float64, device="cuda")
    want.index_add_(0, cells.long(), ctr[:, 1].double() / ef.double())
    counts = torch.bincount(cells.long(), minlength=s.n_cells).double()
    torch.testing.assert_close(s.cost[0], want, rtol=1e-12, atol=1e-9)
    assert torch.equal(s.cost[2], counts)
    assert float(s.cost[1].abs().sum()) == 0.0 and float(s.cost[3].sum()) == 0.0
