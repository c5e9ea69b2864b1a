"""Start order of a search batch: the queries predicted to be longest start first.

The search kernel is persistent: each warp takes the next query from a queue until it is empty.
Per query the work is a chain of dependent memory round trips, so a warp's time grows with the
query's layer-0 expansions whatever the load, and the batch ends with the warps that drew a long
query late. On the 1M x 128 mixture at ef = 192 the expansions are 204 at the median and up to
514; in row order the batch takes about 1.48x the evenly spread time, and starting the longest
first would take 1.17x (a model of 2,960 warps with time proportional to expansions).

A query's length is predicted from its cell: its nearest pivot row, the pivots that also define
the graph's memory order. The prediction is the mean expansions of the queries of that cell in
earlier batches, accumulated on the GPU from the search's own counters (no host round trip). The
searches are independent of one another, so the order changes no result, counter or trace.
"""

from __future__ import annotations

import torch

# Smallest batch worth ordering: below about the resident warps (2,960 on a B200 with the byte
# kernel) every query starts at once anyway.
MIN_QUERIES = 4096
# Priority = predicted expansions x 4, in the library's 16-bit key range.
PRIORITY_SCALE = 4.0


class CellSchedule:
    """Per-cell expansions per unit of efSearch, learned on the GPU, and the start priority they
    give a batch: predicted expansions = ratio[cell] x the query's efSearch. The query's own ef
    dominates when it varies per query; the cell ranks queries of equal ef. Searches that stop
    early on the learned network keep a table of their own (``stopped``)."""

    def __init__(self, pivots: torch.Tensor) -> None:
        p = pivots.to(torch.float32)
        self.pivots_t = p.t().contiguous()  # (dim, cells)
        self.pivot_norms = (p.double() ** 2).sum(dim=1).float()
        cells = int(p.shape[0])
        # [plain, stopped] x cells: summed expansions / ef, and query counts
        self.total = torch.zeros((2, cells), dtype=torch.float64, device=p.device)
        self.count = torch.zeros((2, cells), dtype=torch.float64, device=p.device)

    def cells(self, queries: torch.Tensor) -> torch.Tensor:
        """Nearest pivot of each float32 query (|p|^2 - 2 q.p; a prediction input, so float32
        rounding is of no consequence)."""
        score = torch.addmm(self.pivot_norms, queries, self.pivots_t, alpha=-2.0)
        return score.argmin(dim=1)

    def priority(self, cells: torch.Tensor, ef: torch.Tensor, stopped: bool = False) -> torch.Tensor:
        """int32 start priority per query (higher starts earlier); 0 for cells not yet seen."""
        t = int(stopped)
        ratio = self.total[t] / self.count[t].clamp(min=1.0)
        key = (ratio[cells] * ef.to(torch.float64) * PRIORITY_SCALE).clamp(max=65535.0)
        return key.to(torch.int32)

    def learn(self, cells: torch.Tensor, hops: torch.Tensor, ef: torch.Tensor,
              stopped: bool = False) -> None:
        """Add a finished batch's expansions (the counters' hops column) to its cells."""
        t = int(stopped)
        self.total[t].index_add_(0, cells, hops.to(torch.float64) / ef.to(torch.float64))
        self.count[t].index_add_(0, cells, torch.ones_like(hops, dtype=torch.float64))

    def reset(self) -> None:
        self.total.zero_()
        self.count.zero_()
