"""int8 scalar quantization and the code-space search with fused exact re-rank.

:class:`ScalarQuantizer` reproduces the reference's codes exactly (``src/hnsw_engine/
quantization.py:29-83``): per-dimension minimum offsets, one step shared by every dimension
(``widest / 255``, or 1 for integer data spanning at most 256 values), ``rint`` then clip to
``[0, 255]``. For L2 the code-space query is ``(q - offset) / step`` (not clipped); for inner product
and cosine the query is unchanged, so ranking against codes equals ranking against decoded vectors.

:class:`QuantizedIndex` (``quantization.py:86-138``) searches the float32-built graph with
distances to the codes on the GPU. With ``rerank = R`` the beam collects ``fetch = min(max(R, k), n)``
candidates and the same kernel re-scores them with exact float64 distances to the float32 vectors,
keeping the best ``k`` by ``(distance, id)`` -- the reference's ``_rerank_batch`` fused into the
search launch. Extension: ``filter=`` (hnswlib pass-through semantics on layer 0), which the
reference's ``QuantizedIndex`` does not expose although its compiled kernel supports it.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import ctypes

import numpy as np
import torch
from numpy.typing import ArrayLike, NDArray

from . import _lib
from .index import HNSWIndex
from .validation import as_matrix, check_int

CODE_LEVELS = 256


@dataclass(frozen=True)
class ScalarQuantizer:
    """Per-dimension offset and one shared step; codes are uint8."""

    offset: NDArray[np.float64]
    step: float

    @classmethod
    def fit(cls, vectors: ArrayLike) -> ScalarQuantizer:
        x = np.asarray(as_matrix(vectors, "vectors"), dtype=np.float64)
        if x.shape[0] == 0:
            raise ValueError("cannot fit a quantizer on zero vectors")
        low = x.min(axis=0)
        widest = float((x.max(axis=0) - low).max())
        lossless = bool(np.array_equal(x, np.rint(x))) and widest <= CODE_LEVELS - 1
        step = 1.0 if (lossless or widest == 0.0) else widest / (CODE_LEVELS - 1)
        return cls(low, step)

    @classmethod
    def fit_device(cls, vectors: torch.Tensor) -> ScalarQuantizer:
        """:meth:`fit` of float32 rows resident on a GPU: one pass of the library's column
        statistics kernel (minima, maxima, integrality), then the same step rule."""
        n, dim = vectors.shape
        if n == 0:
            raise ValueError("cannot fit a quantizer on zero vectors")
        lib = _lib.load()
        dev = vectors.device
        x = vectors.to(torch.float32).contiguous()
        with torch.cuda.device(dev):
            lo = torch.empty(dim, dtype=torch.float64, device=dev)
            hi = torch.empty(dim, dtype=torch.float64, device=dev)
            scratch = torch.empty(int(lib.hnsw_b200_quant_scratch_bytes(dim)), dtype=torch.uint8, device=dev)
            integer = ctypes.c_int32(0)
            stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
            _lib.check(lib.hnsw_b200_quant_stats(x.data_ptr(), n, dim, lo.data_ptr(), hi.data_ptr(),
                                                 ctypes.byref(integer), scratch.data_ptr(), stream))
        low = lo.cpu().numpy()
        widest = float((hi.cpu().numpy() - low).max())
        lossless = bool(integer.value) and widest <= CODE_LEVELS - 1
        step = 1.0 if (lossless or widest == 0.0) else widest / (CODE_LEVELS - 1)
        return cls(low, step)

    def encode(self, vectors: ArrayLike) -> NDArray[np.uint8]:
        x = np.asarray(vectors, dtype=np.float64)
        codes = np.clip(np.rint((x - self.offset) / self.step), 0, CODE_LEVELS - 1)
        return np.ascontiguousarray(codes, dtype=np.uint8)

    def encode_device(self, vectors: torch.Tensor) -> torch.Tensor:
        """:meth:`encode` of float32 rows resident on a GPU (the same float64 arithmetic)."""
        lib = _lib.load()
        dev = vectors.device
        x = vectors.to(torch.float32).contiguous()
        n, dim = x.shape
        with torch.cuda.device(dev):
            codes = torch.empty((n, dim), dtype=torch.uint8, device=dev)
            if n:
                off = torch.from_numpy(np.ascontiguousarray(self.offset, dtype=np.float64)).to(dev)
                stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
                _lib.check(lib.hnsw_b200_quant_encode(x.data_ptr(), n, dim, off.data_ptr(),
                                                      float(self.step), codes.data_ptr(), stream))
        return codes

    def decode(self, codes: NDArray[np.uint8]) -> NDArray[np.float64]:
        return self.offset + self.step * codes.astype(np.float64)

    def transform_queries(self, queries: ArrayLike, metric: str) -> NDArray[np.float64]:
        q = np.asarray(queries, dtype=np.float64)
        if metric == "l2":
            return np.ascontiguousarray((q - self.offset) / self.step)
        return np.ascontiguousarray(q)

    def to_distance(self, code_distances: NDArray[np.float64], queries: ArrayLike,
                    metric: str) -> NDArray[np.float64]:
        """Code-space distances (one row per query) -> distances to the decoded vectors."""
        if metric == "l2":
            return code_distances * self.step**2
        shift = np.asarray(queries, dtype=np.float64) @ self.offset
        if metric == "ip":
            return self.step * code_distances - shift[:, None]
        return 1.0 - shift[:, None] - self.step + self.step * code_distances


class QuantizedIndex:
    """Searches the graph of a :class:`HNSWIndex` with distances to int8 codes on the GPU."""

    def __init__(self, index: HNSWIndex) -> None:
        if len(index) == 0:
            raise ValueError("cannot quantize an empty index")
        self._index = index
        # fit and encode on the GPU, over the rows already resident for searching
        g = index.device_graph
        self.quantizer = ScalarQuantizer.fit_device(g.vectors)
        self._codes_device = self.quantizer.encode_device(g.vectors)
        self._n = len(index)
        g.attach_codes(self._codes_device)
        self._codes_host: NDArray[np.uint8] | None = None

    @property
    def codes(self) -> NDArray[np.uint8]:
        """The (n, dim) uint8 codes (the reference's ``QuantizedIndex.codes``)."""
        if self._codes_host is None:
            self._codes_host = self._codes_device.cpu().numpy()
        return self._codes_host

    @property
    def code_bytes(self) -> int:
        return int(self._codes_device.numel())

    @property
    def vector_bytes(self) -> int:
        return len(self._index) * self._index.dim * 4

    def batch_search(
        self, queries: ArrayLike, k: int = 10, ef: Any = None, rerank: int = 0,
        filter: ArrayLike | None = None,
    ) -> tuple[NDArray[np.int64], NDArray[np.float64]]:
        """Approximate ``k`` nearest neighbours of each query row (reference ``quantization.py:114-138``).

        Without re-ranking the distances are those to the decoded vectors. With ``rerank = R`` the
        search collects ``max(R, k)`` candidates (with at least that ``ef``) and returns the best
        ``k`` by exact distance, ties to the lower id.
        """
        if len(self._index) != self._n:
            raise ValueError("the index changed after quantization; build a new QuantizedIndex")
        k_valid, ef_valid = self._index._check_search_args(k, ef)
        r = check_int(rerank, "rerank", minimum=0)
        allowed = self._index._check_filter(filter)
        metric = self._index.metric
        prepared = self._index._prepare(queries)
        nq = prepared.shape[0]
        fetch = min(max(r, k_valid), len(self._index))
        if allowed is not None and not allowed.any():
            return np.full((nq, k_valid), -1, np.int64), np.full((nq, k_valid), np.inf)
        ef_fetch = np.maximum(np.asarray(ef_valid, dtype=np.int64), fetch)
        code_q = self.quantizer.transform_queries(prepared, metric)
        g = self._index.device_graph
        if r == 0:
            ids, dists, ctr = g.search(code_q, fetch, ef_fetch, allowed=allowed, use_codes=True)
            self._index._accumulate(ctr)
            return ids.cpu().numpy(), self.quantizer.to_distance(dists.cpu().numpy(), prepared, metric)
        ids, dists, ctr = g.search(
            code_q, k_valid, ef_fetch, allowed=allowed, use_codes=True, k_search=fetch,
            rerank_queries=prepared,
        )
        self._index._accumulate(ctr)
        return ids.cpu().numpy(), dists.cpu().numpy()

    def batch_search_device(self, code_queries: torch.Tensor, prepared: torch.Tensor, k: int,
                            ef: Any, rerank: int) -> tuple[torch.Tensor, torch.Tensor]:
        """Device-resident variant: code-space and prepared queries already on the GPU."""
        fetch = min(max(rerank, k), len(self._index))
        g = self._index.device_graph
        ids, dists, _ = g.search(code_queries, k, ef, use_codes=True, k_search=fetch,
                                 rerank_queries=prepared if rerank else None, counters=False)
        return ids, dists
