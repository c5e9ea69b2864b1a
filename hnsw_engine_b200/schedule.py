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

import ctypes

import torch

from . import _lib

# Smallest batch worth ordering: below about the resident warps (2,960 on a B200 with the byte
# kernel) every query starts at once anyway.
MIN_QUERIES = 4096
# Priority = predicted expansions x 4, in the library's 16-bit key range.
PRIORITY_SCALE = 4.0


class CellSchedule:
    """Per-cell expansions per unit of efSearch, learned on the GPU, and the start priority they
    give a batch: predicted expansions = ratio[cell] x the query's efSearch. The query's own ef
    dominates when it varies per query; the cell ranks queries of equal ef.

    ``hnsw_b200_start_priority`` computes cells and priorities in one launch; the search kernel
    adds each finished query to ``cost`` ((4, cells) float64: plain sums, stopped sums, plain
    counts, stopped counts). Searches that stop early on the learned network learn into a table
    of their own, which is read only for cells that plain searches have not reached: the plain
    table ranks cells better for stopped searches too (learned stop on the 1M mixture, cap 192:
    3.87 ms ordered by its own table, the same as row order, against 3.67 ms ordered by the plain
    one; a stopped table learned only at the final threshold orders them in 3.59 ms against 3.48
    ms by the plain one)."""

    def __init__(self, pivots: torch.Tensor) -> None:
        self.pivots = pivots.to(torch.float32).contiguous()  # (cells, dim), on the graph's GPU
        self.n_cells = int(self.pivots.shape[0])
        self.cost = torch.zeros((4, self.n_cells), dtype=torch.float64, device=self.pivots.device)

    def start(self, queries: torch.Tensor, ef: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """(cells, priority) of a float32 device batch with its (nq,) int32 efSearch, on the
        current stream."""
        nq, dim = int(queries.shape[0]), int(queries.shape[1])
        dev = self.pivots.device
        cells = torch.empty(nq, dtype=torch.int32, device=dev)
        prio = torch.empty(nq, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(_lib.load().hnsw_b200_start_priority(
            queries.data_ptr(), nq, dim, self.pivots.data_ptr(), self.n_cells, self.cost.data_ptr(),
            ef.data_ptr(), PRIORITY_SCALE, cells.data_ptr(), prio.data_ptr(),
            ctypes.c_void_p(stream)))
        return cells, prio

    def reset(self) -> None:
        self.cost.zero_()
