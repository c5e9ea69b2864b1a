"""The start-order predictor on the host (torch CPU tensors, no GPU): nearest pivots, per-cell
mean expansions and the 16-bit priority they give."""

from __future__ import annotations

import numpy as np
import torch

from hnsw_engine_b200.schedule import PRIORITY_SCALE, CellSchedule


def test_cells_are_the_nearest_pivots() -> None:
    rng = np.random.default_rng(0)
    piv = rng.integers(0, 256, (64, 16)).astype(np.float32)
    q = rng.integers(0, 256, (500, 16)).astype(np.float32)
    s = CellSchedule(torch.from_numpy(piv))
    got = s.cells(torch.from_numpy(q)).numpy()
    d = ((q[:, None, :].astype(np.float64) - piv[None, :, :]) ** 2).sum(-1)
    # the chosen pivot is at the minimum distance (ties may pick either)
    np.testing.assert_array_equal(d[np.arange(500), got], d.min(1))


def test_priority_is_the_learned_cell_ratio_times_ef() -> None:
    piv = torch.tensor([[0.0, 0.0], [10.0, 0.0], [0.0, 10.0]])
    s = CellSchedule(piv)
    cells = torch.tensor([0, 1, 1, 2, 0])
    ef = torch.full((5,), 100, dtype=torch.int32)
    assert s.priority(cells, ef).tolist() == [0, 0, 0, 0, 0]  # nothing learned: row order
    s.learn(cells, torch.tensor([100, 300, 500, 200, 120]), ef)
    ratio = [1.1, 4.0, 2.0]  # expansions per unit of ef, per cell
    want = [int(ratio[c] * 100 * PRIORITY_SCALE) for c in cells.tolist()]
    assert s.priority(cells, ef).tolist() == want
    # the query's own ef scales its prediction
    assert s.priority(torch.tensor([1]), torch.tensor([50])).tolist() == [int(4.0 * 50 * PRIORITY_SCALE)]
    # stopped searches learn and read a table of their own
    assert s.priority(cells, ef, stopped=True).tolist() == [0, 0, 0, 0, 0]
    s.learn(torch.tensor([2]), torch.tensor([10**7]), torch.tensor([1]))  # clamped to 16 bits
    assert int(s.priority(torch.tensor([2]), torch.tensor([1]))) == 65535
    s.reset()
    assert s.priority(cells, ef).tolist() == [0, 0, 0, 0, 0]
