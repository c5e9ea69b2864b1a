"""The GPU engine: the reference's native graph arrays resident in HBM, searched through the C ABI.

:class:`DeviceGraph` uploads the seven native arrays (``src/hnsw_engine/numba_engine.py:36-44``)
unchanged -- the device copies are byte-identical to the ``.npy`` files -- and opens a
``libhnsw_b200`` handle over them. Torch is used only for device memory and streams; every search
is one call into the library, whose kernels do all the work.

The distance arithmetic of a call is chosen per batch (:func:`DeviceGraph.exact_f32_ok`): when data
and queries are integer-valued and every partial sum of the distance stays below 2**24, float32
arithmetic is exact in any order and reproduces the reference's float64 value bit for bit, so the
fast warp-parallel float32 kernel runs; otherwise the kernel accumulates in float64 sequentially
over the dimensions, which is the reference's own arithmetic (``_distance``, numba_engine.py:57-70).
"""

from __future__ import annotations

import ctypes
import warnings
from typing import Any

import numpy as np
import torch
from numpy.typing import NDArray

from . import _lib
from .schedule import MIN_QUERIES, CellSchedule

EXACT_LIMIT = float(2**24)
# Host threads that read an uploaded query batch for its statistics (the library's pool size caps it).
UPLOAD_THREADS = 8
# Graphs of at least this many nodes are stored on the GPU in a locality order (see
# DeviceGraph._build_internal_order); smaller ones fit in L2 and keep the reference's order.
LOCALITY_MIN_NODES = 65536
LOCALITY_CELLS = 256
# Autotuner: a configuration replaces the default only when it is this much faster.
TUNE_MARGIN = 0.02
TUNE_REPS = 3


def pick_config(ms: list[float], default: int = 0, margin: float = TUNE_MARGIN) -> int:
    """The kernel configuration to keep from measured times (one per configuration, same batch):
    the fastest, if it beats the default by more than ``margin``, else the default. A function of
    the timings alone, so the same measurements always give the same choice."""
    if not ms:
        return default
    best = min(range(len(ms)), key=lambda c: (ms[c], c))
    return best if ms[best] < (1.0 - margin) * ms[default] else default


def tune_key(dist_mode: int, use_codes: bool, filtered: bool, ef_cap: int, stop: bool,
             rerank: bool) -> tuple:
    """What a tuned choice is kept for: the kernel (distance mode, rows, filter), the learned stop
    and the rerank epilogue, and the efSearch cap rounded up to a power of two."""
    bucket = 1 << max(0, int(ef_cap) - 1).bit_length()
    return (int(dist_mode), bool(use_codes), bool(filtered), bucket, bool(stop), bool(rerank))


def _dev_ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else int(t.data_ptr())


def pack_mask(mask: NDArray[np.bool_]) -> NDArray[np.uint32]:
    """Bool mask -> little-endian bitmap words (bit i of word w is node 32 w + i)."""
    n = mask.shape[0]
    words = (n + 31) // 32
    packed = np.packbits(np.ascontiguousarray(mask, dtype=np.bool_), bitorder="little")
    padded = np.zeros(words * 4, dtype=np.uint8)
    padded[: packed.shape[0]] = packed
    return padded.view(np.uint32)


def to_device(a: Any, dtype: torch.dtype, device: torch.device) -> torch.Tensor:
    """Host array or device tensor -> contiguous device tensor of ``dtype`` (H2D copy if host; an
    asynchronous one on the current stream from a page-locked tensor of that dtype)."""
    if isinstance(a, torch.Tensor):
        if not a.is_cuda and a.dtype == dtype and a.is_contiguous() and a.is_pinned():
            return a.to(device=device, non_blocking=True)
        return a.to(device=device, dtype=dtype).contiguous()
    arr = np.ascontiguousarray(a)
    if arr.flags.writeable:
        t = torch.from_numpy(arr)
    else:
        # Read-only source (an mmap of a native .npy): the tensor is only read, by the copy below,
        # so torch's warning about writes through non-writable memory does not apply.
        with warnings.catch_warnings():
            warnings.filterwarnings("ignore", message="The given NumPy array is not writable")
            t = torch.from_numpy(arr)
    if t.dtype != dtype:
        t = t.to(dtype)
    return t.to(device, non_blocking=False).contiguous()


class CapturedSearch:
    """One batched search recorded as a CUDA graph and replayed: the start-order launches, the
    counters' reset and the search kernel, with no host work between them.

    The queries live in a fixed device buffer (``self.queries``): copy each new batch into it,
    then :meth:`replay`. Construction runs the search once synchronously with the same arguments,
    which sizes the scratch, picks the distance arithmetic from the buffer's current contents and
    lets the autotuner choose the kernel configuration; the graph keeps those choices, so later
    batches must suit the same arithmetic (byte mode: integer queries in [0, 255]).
    :meth:`results` returns the outputs after checking on the host that no query overflowed its
    scratch, re-running the batch synchronously in that rare case."""

    def __init__(self, graph: "DeviceGraph", queries: torch.Tensor, k: int, ef: int, *,
                 stop: tuple | None = None) -> None:
        self.graph = graph
        # the graph reads this buffer: its own copy, never an alias of the caller's tensor
        self.queries = torch.empty(tuple(queries.shape), dtype=torch.float32, device=graph.device)
        self.queries.copy_(queries)
        self.k, self.ef, self.stop = int(k), int(ef), stop
        nq = self.queries.shape[0]
        dev = graph.device
        with torch.cuda.device(dev):
            self.out = (torch.empty((nq, k), dtype=torch.int64, device=dev),
                        torch.empty((nq, k), dtype=torch.float64, device=dev),
                        torch.empty((nq, 2), dtype=torch.int64, device=dev))
            graph.search(self.queries, k, ef, stop=stop, out=self.out)
            self.dist_mode = graph.last_call["dist_mode"]
            self.kernel_config = graph.last_call["kernel_config"]
            torch.cuda.synchronize(dev)
            self.cuda_graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.cuda_graph):
                graph.search(self.queries, k, ef, stop=stop, out=self.out, dist_mode=self.dist_mode,
                             kernel_config=self.kernel_config, asynchronous=True)
            graph._priority_launches = 0

    def replay(self) -> None:
        """Run the recorded search on the buffer's current queries (asynchronous)."""
        self.cuda_graph.replay()

    def results(self) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """(ids, distances, counters) of the last replay; overflowed queries (none in practice)
        are searched again synchronously."""
        if self.graph.search_failed():
            self.graph.search(self.queries, self.k, self.ef, stop=self.stop, out=self.out,
                              dist_mode=self.dist_mode, kernel_config=self.kernel_config)
        return self.out


class DeviceGraph:
    """A reference-built HNSW graph resident on one GPU, plus its library handle."""

    def __init__(
        self,
        arrays: dict[str, NDArray[Any]],
        entry_point: int,
        max_level: int,
        metric: str,
        device: str | torch.device = "cuda",
        locality: bool | None = None,
        validate_M: int | None = None,
    ) -> None:
        self.lib = _lib.load()
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("the B200 engine needs a CUDA device")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.metric = metric
        self.n, self.dim = arrays["vectors"].shape
        self.entry_point = int(entry_point)
        self.max_level = int(max_level)
        host_vectors = np.ascontiguousarray(arrays["vectors"], dtype=np.float32)
        self.host_vectors = host_vectors
        with torch.cuda.device(self.device):
            self.vectors = to_device(host_vectors, torch.float32, self.device)
            self.links0 = to_device(arrays["links0"], torch.int32, self.device)
            self.count0 = to_device(arrays["count0"], torch.int32, self.device)
            self.upper_offset = to_device(arrays["upper_offset"], torch.int64, self.device)
            links_up = np.asarray(arrays["links_up"])
            count_up = np.asarray(arrays["count_up"])
            self.rows = int(links_up.shape[0])
            self.links_up_stride = int(links_up.shape[1]) if links_up.ndim == 2 else 1
            if self.rows == 0:  # keep valid (unused) pointers
                links_up = np.zeros((1, self.links_up_stride), dtype=np.int32)
                count_up = np.zeros(1, dtype=np.int32)
            self.links_up = to_device(links_up, torch.int32, self.device)
            self.count_up = to_device(count_up, torch.int32, self.device)
        self.links0_stride = int(arrays["links0"].shape[1])
        self.codes: torch.Tensor | None = None
        # Host facts for choosing the exact integer kernels.
        self._integer = bool(np.array_equal(host_vectors, np.rint(host_vectors)))
        self._lo = host_vectors.min(axis=0).astype(np.float64) if self.n else np.zeros(self.dim)
        self._hi = host_vectors.max(axis=0).astype(np.float64) if self.n else np.zeros(self.dim)
        # Integer vectors in [0, 255] are the same values as bytes: keep a uint8 copy so the byte
        # kernel (exact integer dot products) can search them with a quarter of the traffic.
        self.vector_bytes: torch.Tensor | None = None
        if (self._integer and self.n and self.dim % 4 == 0 and self._lo.min() >= 0
                and self._hi.max() <= 255):
            with torch.cuda.device(self.device):
                self.vector_bytes = to_device(host_vectors.astype(np.uint8), torch.uint8, self.device)
        # Automatic: every large graph. Each kernel's expansions wait on their gathers, the float64
        # one's included once its rows are prefetched (1M x 100 cosine, 10K queries: ef = 64 3.61 ->
        # 2.91 ms, ef = 256 9.59 -> 8.91 ms; identical results).
        if locality is None:
            locality = self.n >= LOCALITY_MIN_NODES
        self.locality = bool(locality) and self.n > 1
        self.order: torch.Tensor | None = None  # internal node -> original id (None: identity)
        self._order_host: NDArray[np.int64] | None = None
        # Longest-predicted-first start order of large batches (graphs with cells only); set
        # False to start queries in row order. Results are the same either way.
        self.schedule = True
        self._schedule: CellSchedule | None = None
        self._priority_launches = 0
        # page-locked staging of uploaded query batches, and the end of the last DMA from it
        self._stage: torch.Tensor | None = None
        self._stage_done = torch.cuda.Event()
        self._internal: dict[str, Any] = {}
        # Runtime autotuner (see search): kernel configuration per tune_key, with the timings that
        # chose it.
        self.autotune = True
        self.last_call: dict[str, int] = {}  # dist_mode and kernel_config of the last search
        self.tuned: dict[tuple, int] = {}
        self.tune_log: dict[tuple, list[float]] = {}
        if validate_M is not None:  # before anything follows the links
            self._validate_on_device(arrays["levels"], int(validate_M))
        if self.locality:
            self._build_internal_order()
        elif self.n >= LOCALITY_MIN_NODES:  # the start order alone: pivots, no memory reorder
            with torch.cuda.device(self.device):
                self._schedule = CellSchedule(self._pivot_rows())
        self._handle = ctypes.c_void_p()
        self._open()

    def _validate_on_device(self, levels: NDArray[np.int64], M: int) -> None:
        """The checks of the reference's _validate_native on the uploaded arrays (one kernel pass);
        raises its ValueError for the first failed check."""
        from .validation import device_validation_message

        dev = self.device
        with torch.cuda.device(dev):
            lv = to_device(levels, torch.int64, dev)
            scratch = torch.empty(int(self.lib.hnsw_b200_validate_scratch_bytes(self.rows)),
                                  dtype=torch.uint8, device=dev)
            flags = ctypes.c_uint32(0)
            g = self._graph_struct()
            stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
            _lib.check(self.lib.hnsw_b200_validate_graph(ctypes.byref(g), _dev_ptr(lv), M,
                                                         _dev_ptr(scratch), ctypes.byref(flags), stream))
        message = device_validation_message(int(flags.value), M)
        if message is not None:
            raise ValueError(message)

    # ------------------------------------------------------------------------ node order
    def _build_internal_order(self) -> None:
        """Store the graph in cell order: nodes grouped by their nearest of 256 sampled pivot rows
        (ties to the lower original id), so that a search's visited nodes, rows and link rows fall
        in a few contiguous ranges. The library reads every array in this internal order and maps
        back to original ids for results and for ties between equal distances, so results are the
        reference's exactly; only memory locality changes."""
        from .exact_knn import exact_search

        dev = self.device
        n = self.n
        with torch.cuda.device(dev):
            pivots = self._pivot_rows()
            nearest, _ = exact_search(pivots, self.vectors, 1, "l2")
            order = torch.sort(nearest[:, 0], stable=True).indices  # internal -> original
            new_of_old = torch.empty_like(order)
            new_of_old[order] = torch.arange(n, device=dev)

            def relink(links: torch.Tensor, counts: torch.Tensor) -> torch.Tensor:
                valid = torch.arange(links.shape[1], device=dev)[None, :] < counts[:, None]
                mapped = new_of_old[links.clamp(0, n - 1).long()].to(torch.int32)
                return torch.where(valid, mapped, links).contiguous()

            inner = self._internal
            inner["vectors"] = self.vectors[order].contiguous()
            inner["vector_bytes"] = (self.vector_bytes[order].contiguous()
                                     if self.vector_bytes is not None else None)
            inner["count0"] = self.count0[order].contiguous()
            links0 = relink(self.links0[order], inner["count0"])
            links_up = relink(self.links_up, self.count_up)
            # The native rows hold one slot more than a link count can reach (2M + 1 and M + 1):
            # without it a layer-0 row of M = 16 is exactly one 128-byte line.
            w0, wu = links0.shape[1] - 1, links_up.shape[1] - 1
            if w0 >= 1 and int(inner["count0"].max()) <= w0:
                links0 = links0[:, :w0]
            if wu >= 1 and (self.rows == 0 or int(self.count_up.max()) <= wu):
                links_up = links_up[:, :wu]
            inner["links0"] = links0.contiguous()
            inner["links_up"] = links_up.contiguous()
            inner["upper_offset"] = self.upper_offset[order].contiguous()
            inner["entry_point"] = int(new_of_old[self.entry_point].item())
            inner["node_ids"] = order.to(torch.int32).contiguous()
            self._schedule = CellSchedule(pivots)
        self.order = order
        self._order_host = order.cpu().numpy()

    def _pivot_rows(self) -> torch.Tensor:
        """The cells' pivots: LOCALITY_CELLS rows sampled without replacement (seed 0), in row
        order, as float32 device rows."""
        cells = min(LOCALITY_CELLS, self.n)
        pick = np.sort(np.random.default_rng(0).choice(self.n, cells, replace=False))
        return self.vectors[torch.from_numpy(pick).to(self.device)].contiguous()

    def internal_mask(self, mask: NDArray[np.bool_]) -> NDArray[np.bool_]:
        """A filter mask over original ids, rearranged into the internal node order."""
        return mask if self._order_host is None else np.ascontiguousarray(mask[self._order_host])

    def _graph_struct(self) -> _lib.Graph:
        inner = self._internal
        if inner:
            return _lib.Graph(
                vectors=_dev_ptr(inner["vectors"]),
                codes=_dev_ptr(inner.get("codes")),
                links0=_dev_ptr(inner["links0"]),
                count0=_dev_ptr(inner["count0"]),
                upper_offset=_dev_ptr(inner["upper_offset"]),
                links_up=_dev_ptr(inner["links_up"]),
                count_up=_dev_ptr(self.count_up),
                n=self.n,
                rows=self.rows,
                dim=self.dim,
                links0_stride=int(inner["links0"].shape[1]),
                links_up_stride=int(inner["links_up"].shape[1]),
                metric=_lib.METRIC_CODES[self.metric],
                entry_point=inner["entry_point"],
                max_level=self.max_level,
                reserved=0,
                vector_bytes=_dev_ptr(inner["vector_bytes"]),
                node_ids=_dev_ptr(inner["node_ids"]),
            )
        return _lib.Graph(
            vectors=_dev_ptr(self.vectors),
            codes=_dev_ptr(self.codes),
            links0=_dev_ptr(self.links0),
            count0=_dev_ptr(self.count0),
            upper_offset=_dev_ptr(self.upper_offset),
            links_up=_dev_ptr(self.links_up),
            count_up=_dev_ptr(self.count_up),
            n=self.n,
            rows=self.rows,
            dim=self.dim,
            links0_stride=self.links0_stride,
            links_up_stride=self.links_up_stride,
            metric=_lib.METRIC_CODES[self.metric],
            entry_point=self.entry_point,
            max_level=self.max_level,
            reserved=0,
            vector_bytes=_dev_ptr(self.vector_bytes),
            node_ids=None,
        )

    def _open(self) -> None:
        if self._handle:
            self.lib.hnsw_b200_close(self._handle)
            self._handle = ctypes.c_void_p()
        g = self._graph_struct()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.hnsw_b200_open(ctypes.byref(g), ctypes.byref(self._handle)))

    def attach_codes(self, codes: NDArray[np.uint8] | torch.Tensor) -> None:
        """Attach scalar-quantizer codes (n, dim) uint8 (host array or device tensor, original node
        order) for code-space searches."""
        is_u8 = codes.dtype == (torch.uint8 if isinstance(codes, torch.Tensor) else np.uint8)
        if tuple(codes.shape) != (self.n, self.dim) or not is_u8:
            raise ValueError(f"codes must be uint8 with shape {(self.n, self.dim)}")
        with torch.cuda.device(self.device):
            self.codes = to_device(codes, torch.uint8, self.device)
            if self._internal:
                self._internal["codes"] = self.codes[self.order].contiguous()
        self._open()

    def close(self) -> None:
        if getattr(self, "_handle", None):
            self.lib.hnsw_b200_close(self._handle)
            self._handle = ctypes.c_void_p()

    def __del__(self) -> None:  # pragma: no cover - interpreter teardown order varies
        try:
            self.close()
        except Exception:
            pass

    @property
    def last_launches(self) -> int:
        """This library's kernel launches in the last search: the start-priority kernel, when it
        ran, and those of hnsw_b200_search."""
        return int(self.lib.hnsw_b200_last_launches(self._handle)) + self._priority_launches

    # ------------------------------------------------------------------ arithmetic selection
    def choose_mode(self, queries: NDArray[Any], codes: bool) -> int:
        """Fastest exact arithmetic for this batch: bytes, exact float32, or float64 sequential."""
        if self.metric != "cosine" and self.dim % 4 == 0:
            rows_ok = codes or self.vector_bytes is not None
            q = np.asarray(queries)
            if rows_ok and q.size and np.array_equal(q, np.rint(q)) and q.min() >= 0 and q.max() <= 255:
                return _lib.DIST_BYTES
        return _lib.DIST_EXACT_F32 if self.exact_f32_ok(queries, codes) else _lib.DIST_F64

    def exact_f32_ok(self, queries: NDArray[Any], codes: bool, step_lo_hi=None) -> bool:
        """Whether float32 arithmetic is exact for this batch (integer data, partial sums < 2**24)."""
        if self.metric == "cosine":
            return False
        if codes:
            lo, hi = np.zeros(self.dim), np.full(self.dim, 255.0)
        else:
            if not self._integer:
                return False
            lo, hi = self._lo, self._hi
        q = np.asarray(queries, dtype=np.float64)
        if q.size == 0:
            return True
        if not np.array_equal(q, np.rint(q)):
            return False
        if self.metric == "l2":
            span = np.maximum(np.abs(q - lo), np.abs(hi - q))
            bound = (span * span).sum(axis=1).max()
        else:
            bound = (np.abs(q) * np.maximum(np.abs(lo), np.abs(hi))).sum(axis=1).max()
        return bool(bound < EXACT_LIMIT)

    def upload_queries(self, src: NDArray[np.float32], dst: torch.Tensor | None,
                       threads: int = UPLOAD_THREADS, staged: bool = True) -> _lib.ValueStats:
        """Copy C-contiguous float32 host queries into the device tensor ``dst`` on the current
        stream (``None``: no copy) and return their statistics (finite, integer, min, max), read
        on host threads in the library.

        ``staged``: the threads also copy the rows into this graph's page-locked staging buffer
        and one asynchronous DMA follows (faster than the pageable copy); the buffer is reused
        only once the previous DMA from it has completed."""
        st = _lib.ValueStats()
        if dst is None:
            _lib.check(self.lib.hnsw_b200_upload_queries(src.ctypes.data, None, src.size,
                                                          int(threads), ctypes.byref(st), None, None))
            return st
        if dst.numel() != src.size or dst.dtype != torch.float32 or not dst.is_contiguous():
            raise ValueError("dst must be a contiguous float32 device tensor of src's size")
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device)
            stage = None
            if staged:
                if self._stage is None or self._stage.numel() < src.size:
                    self._stage = torch.empty(max(src.size, 1 << 20), dtype=torch.float32,
                                              pin_memory=True)
                else:
                    self._stage_done.synchronize()  # the previous DMA from it has finished
                stage = self._stage
            _lib.check(self.lib.hnsw_b200_upload_queries(
                src.ctypes.data, _dev_ptr(dst), src.size, int(threads), ctypes.byref(st),
                _dev_ptr(stage), ctypes.c_void_p(stream.cuda_stream)))
            if stage is not None:
                self._stage_done.record(stream)
        return st

    def mode_from_stats(self, st: _lib.ValueStats, queries: NDArray[np.float32]) -> int:
        """:meth:`choose_mode` from :meth:`upload_queries` statistics (uncoded queries): the same
        rules; only integer data outside the byte range still needs the host's per-row bound."""
        if queries.size == 0 or self.metric == "cosine" or not st.integer:
            return _lib.DIST_F64
        if self.dim % 4 == 0 and self.vector_bytes is not None and st.min >= 0 and st.max <= 255:
            return _lib.DIST_BYTES
        return _lib.DIST_EXACT_F32 if self.exact_f32_ok(queries, False) else _lib.DIST_F64

    def choose_mode_device(self, q: torch.Tensor, codes: bool,
                           stats: tuple[bool, float, float] | None = None) -> int:
        """:meth:`choose_mode` for queries already on this GPU: the same rules, evaluated by a few
        device reductions and one small copy back, instead of a host pass over the batch.
        ``stats``: ``(integer, min, max)`` of ``q`` when the caller has read them already."""
        if q.numel() == 0:
            return _lib.DIST_F64
        if stats is None:
            # integrality, minimum and maximum in q's own dtype (exact for float32 and float64 alike)
            lo_q, hi_q = torch.aminmax(q)
            st = torch.stack([(q != torch.round(q)).any().to(q.dtype), lo_q, hi_q]).to(torch.float64).cpu()
            stats = (not bool(st[0]), float(st[1]), float(st[2]))
        integer, q_lo, q_hi = stats
        if self.metric == "cosine" or not integer:
            return _lib.DIST_F64
        rows_ok = codes or self.vector_bytes is not None
        if self.dim % 4 == 0 and rows_ok and q_lo >= 0 and q_hi <= 255:
            return _lib.DIST_BYTES
        if codes:
            lo, hi = np.zeros(self.dim), np.full(self.dim, 255.0)
        elif self._integer:
            lo, hi = self._lo, self._hi
        else:
            return _lib.DIST_F64
        qd = q.to(torch.float64)
        lo_t = torch.from_numpy(np.asarray(lo, dtype=np.float64)).to(qd.device)
        hi_t = torch.from_numpy(np.asarray(hi, dtype=np.float64)).to(qd.device)
        if self.metric == "l2":
            span = torch.maximum((qd - lo_t).abs(), (hi_t - qd).abs())
            bound = (span * span).sum(dim=1).max()
        else:
            bound = (qd.abs() * torch.maximum(lo_t.abs(), hi_t.abs())).sum(dim=1).max()
        return _lib.DIST_EXACT_F32 if float(bound) < EXACT_LIMIT else _lib.DIST_F64

    # ------------------------------------------------------------------- single-query path
    def search_one(self, query: NDArray[np.float32], k: int, ef: int) -> tuple[NDArray[np.int64],
                                                                              NDArray[np.float64],
                                                                              NDArray[np.int64]]:
        """One prepared float32 query (dim,), unfiltered, for latency: preallocated device and
        pinned host buffers, the arithmetic chosen on the host from the query's own values, one
        library call (which synchronises once) and asynchronous copies either side. Returns host
        arrays (ids (k,), distances (k,), counters (2,))."""
        dev = self.device
        key = int(k)
        buf = getattr(self, "_one", None)
        if buf is None or buf["k"] != key:
            with torch.cuda.device(dev):
                buf = {
                    "k": key,
                    "q": torch.empty((1, self.dim), dtype=torch.float32, device=dev),
                    "ef": torch.empty(1, dtype=torch.int32, device=dev),
                    "ids": torch.empty((1, key), dtype=torch.int64, device=dev),
                    "dists": torch.empty((1, key), dtype=torch.float64, device=dev),
                    "ctr": torch.empty((1, 2), dtype=torch.int64, device=dev),
                    "h_q": torch.empty((1, self.dim), dtype=torch.float32).pin_memory(),
                    "h_ef": torch.empty(1, dtype=torch.int32).pin_memory(),
                    "h_ids": torch.empty((1, key), dtype=torch.int64).pin_memory(),
                    "h_dists": torch.empty((1, key), dtype=torch.float64).pin_memory(),
                    "h_ctr": torch.empty((1, 2), dtype=torch.int64).pin_memory(),
                }
            self._one = buf
        q = np.asarray(query, dtype=np.float32).reshape(1, self.dim)
        mode = self.choose_mode(q, False)
        buf["h_q"].numpy()[:] = q
        buf["h_ef"].numpy()[0] = max(int(ef), key)
        stream = torch.cuda.current_stream(dev)
        with torch.cuda.device(dev):
            buf["q"].copy_(buf["h_q"], non_blocking=True)
            buf["ef"].copy_(buf["h_ef"], non_blocking=True)
            args = _lib.SearchArgs(
                queries=buf["q"].data_ptr(), queries_f64=0, use_codes=0, nq=1, k=key, k_search=key,
                ef=buf["ef"].data_ptr(), ef_max=max(int(ef), key), dist_mode=int(mode), allowed=None,
                allowed_fraction=1.0, rerank_queries=None, out_ids=buf["ids"].data_ptr(),
                out_dists=buf["dists"].data_ptr(), out_counters=buf["ctr"].data_ptr(),
                stop_mlp=None, stop_threshold=0.0, trace_cap=0, trace_feat=None, trace_dk=None,
                trace_count=None, trace_hops=None,
            )
            _lib.check(self.lib.hnsw_b200_search(self._handle, ctypes.byref(args),
                                                 ctypes.c_void_p(stream.cuda_stream)))
            buf["h_ids"].copy_(buf["ids"], non_blocking=True)
            buf["h_dists"].copy_(buf["dists"], non_blocking=True)
            buf["h_ctr"].copy_(buf["ctr"], non_blocking=True)
            stream.synchronize()
        return (buf["h_ids"].numpy()[0].copy(), buf["h_dists"].numpy()[0].copy(),
                buf["h_ctr"].numpy()[0].copy())

    # ------------------------------------------------------------------------------ search
    def search(
        self,
        queries: Any,
        k: int,
        ef: Any,
        *,
        allowed: NDArray[np.bool_] | torch.Tensor | None = None,
        allowed_fraction: float | None = None,
        use_codes: bool = False,
        k_search: int | None = None,
        rerank_queries: Any = None,
        dist_mode: int | None = None,
        counters: bool = True,
        out: tuple[torch.Tensor, ...] | None = None,
        stop: tuple[torch.Tensor, float] | None = None,
        trace: tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor] | None = None,
        kernel_config: int | None = None,
        asynchronous: bool = False,
        ef_max: int | None = None,
    ) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor | None]:
        """One batched search; returns device tensors ``(ids, dists, counters)``.

        ``queries``: (nq, dim) float32 prepared queries, or float64 code-space queries with
        ``use_codes``. ``ef``: scalar or (nq,) raw efSearch (layer 0 uses ``max(ef, k_search)``).
        ``allowed``: bool mask (n,) over original ids, or a device uint32 bitmap over internal
        ids (``pack_mask(internal_mask(mask))``). ``rerank_queries``: float32 prepared
        queries for the fused exact re-rank of the first ``k_search`` beam entries. ``stop``:
        ``(packed network, threshold[, slope, slope_from])`` for the learned early termination (the
        threshold rises by ``slope`` per 64 layer-0 expansions beyond ``slope_from``); ``trace``: device
        buffers ``(features (nq, cap, 12) f32, first 16 result distances (nq, cap, 16) f64,
        count (nq,) i32, hops (nq,) i32)``
        filled with the stop features every 16 layer-0 expansions.

        Batches of at least ``schedule.MIN_QUERIES`` on graphs of at least ``LOCALITY_MIN_NODES``
        nodes start longest-predicted first (``self.schedule``; see :mod:`.schedule`); results
        do not depend on it.

        ``kernel_config``: the kernel configuration (``hnsw_b200_kernel_configs``); by default the
        autotuner's choice for this kind of batch. With ``self.autotune`` the first batch of at
        least ``schedule.MIN_QUERIES`` queries of each kind (:func:`tune_key`) is searched once
        per configuration, ``TUNE_REPS`` times each, timed with CUDA events, and the choice of
        :func:`pick_config` is kept for later batches. Results do not depend on the configuration.

        ``asynchronous``: issue the search with no host synchronisation, allocation or read-back
        (``hnsw_b200_search_async``), so that it can be recorded in a CUDA graph
        (:class:`CapturedSearch`). It needs ``dist_mode`` and ``kernel_config`` given, a
        device float tensor of queries, ``ef`` an int or a device tensor with ``ef_max``, no host
        filter mask, and scratch sized by an earlier synchronous call of the same size.
        Overflowed queries are left unwritten; :meth:`search_failed` counts them.
        """
        dev = self.device
        nq = int(queries.shape[0])
        ks = int(k if k_search is None else k_search)
        q_f64 = use_codes
        with torch.cuda.device(dev):
            q = to_device(queries, torch.float64 if q_f64 else torch.float32, dev)
            if asynchronous and (dist_mode is None or kernel_config is None):
                raise ValueError("an asynchronous search needs dist_mode and kernel_config")
            if dist_mode is None:
                dist_mode = self.choose_mode_device(q, use_codes)
            if isinstance(ef, torch.Tensor):
                ef_t = ef.to(device=dev, dtype=torch.int32).contiguous()
                if ef_max is None:
                    if asynchronous:
                        raise ValueError("an asynchronous search with per-query ef needs ef_max")
                    ef_max = int(ef_t.max().item()) if nq else 1
            elif np.ndim(ef) == 0:
                ef_max = int(ef) if nq else 1
                ef_t = torch.full((nq,), int(ef), dtype=torch.int32, device=dev)
            else:
                ef_arr = np.broadcast_to(np.asarray(ef, dtype=np.int32), (nq,))
                ef_max = int(ef_arr.max()) if nq else 1
                ef_t = to_device(np.ascontiguousarray(ef_arr), torch.int32, dev)
            bitmap = None
            frac = 1.0
            if allowed is not None:
                if isinstance(allowed, torch.Tensor) and allowed.dtype == torch.int32:
                    bitmap = allowed.contiguous()
                    frac = 1.0 if allowed_fraction is None else float(allowed_fraction)
                else:
                    mask = np.asarray(allowed.cpu() if isinstance(allowed, torch.Tensor) else allowed)
                    frac = float(mask.mean()) if mask.size else 1.0
                    bitmap = to_device(pack_mask(self.internal_mask(mask)).view(np.int32), torch.int32, dev)
            rq = None
            if rerank_queries is not None:
                rq = to_device(rerank_queries, torch.float32, dev)
            # Start order: cells from the float32 queries (code-space searches: their rerank
            # queries). Filtered searches read the order but do not learn: a filter scales every
            # query's cost by about the same factor, so the unfiltered cell ranking still holds,
            # but their expansions would distort the table.
            cell_q = q if not use_codes else rq
            sched = self._schedule if (self.schedule and self._schedule is not None
                                       and nq >= MIN_QUERIES and trace is None
                                       and cell_q is not None) else None
            cells = prio = None
            self._priority_launches = 0
            if sched is not None:
                cells, prio = sched.start(cell_q, ef_t)
                self._priority_launches = 1
            learn = sched is not None and bitmap is None
            if out is None:
                ids = torch.empty((nq, k), dtype=torch.int64, device=dev)
                dists = torch.empty((nq, k), dtype=torch.float64, device=dev)
                ctr = torch.empty((nq, 2), dtype=torch.int64, device=dev) if counters else None
            else:
                ids, dists, ctr = out
            args = _lib.SearchArgs(
                queries=_dev_ptr(q),
                queries_f64=int(q_f64),
                use_codes=int(use_codes),
                nq=nq,
                k=int(k),
                k_search=ks,
                ef=_dev_ptr(ef_t),
                ef_max=max(ef_max, ks),
                dist_mode=int(dist_mode),
                allowed=_dev_ptr(bitmap),
                allowed_fraction=frac,
                rerank_queries=_dev_ptr(rq),
                out_ids=_dev_ptr(ids),
                out_dists=_dev_ptr(dists),
                out_counters=_dev_ptr(ctr),
                stop_mlp=_dev_ptr(stop[0]) if stop is not None else None,
                stop_threshold=float(stop[1]) if stop is not None else 0.0,
                stop_slope=float(stop[2]) if stop is not None and len(stop) > 2 else 0.0,
                stop_slope_from=int(stop[3]) if stop is not None and len(stop) > 3 else 0,
                trace_cap=int(trace[0].shape[1]) if trace is not None else 0,
                trace_feat=_dev_ptr(trace[0]) if trace is not None else None,
                trace_dk=_dev_ptr(trace[1]) if trace is not None else None,
                trace_count=_dev_ptr(trace[2]) if trace is not None else None,
                trace_hops=_dev_ptr(trace[3]) if trace is not None else None,
                priority=_dev_ptr(prio),
                cells=_dev_ptr(cells) if learn else None,
                cell_cost=_dev_ptr(sched.cost) if learn else None,
                n_cells=sched.n_cells if learn else 0,
            )
            stream = torch.cuda.current_stream(dev)
            key = tune_key(dist_mode, use_codes, bitmap is not None, max(ef_max, ks), stop is not None,
                           rq is not None)
            if kernel_config is None:
                n_cfg = int(self.lib.hnsw_b200_kernel_configs(int(dist_mode)))
                if (self.autotune and key not in self.tuned and n_cfg > 1 and nq >= MIN_QUERIES
                        and trace is None):
                    self._tune(args, key, n_cfg, stream)
                kernel_config = self.tuned.get(key, 0)
            args.kernel_config = int(kernel_config)
            self.last_call = {"dist_mode": int(dist_mode), "kernel_config": int(kernel_config)}
            fn = self.lib.hnsw_b200_search_async if asynchronous else self.lib.hnsw_b200_search
            _lib.check(fn(self._handle, ctypes.byref(args), ctypes.c_void_p(stream.cuda_stream)))
        return ids, dists, ctr

    def search_failed(self) -> int:
        """Queries the last asynchronous search left unwritten (their scratch overflowed); waits
        for the current stream."""
        out = ctypes.c_int32(0)
        with torch.cuda.device(self.device):
            stream = torch.cuda.current_stream(self.device).cuda_stream
            _lib.check(self.lib.hnsw_b200_search_failed(self._handle, ctypes.byref(out),
                                                        ctypes.c_void_p(stream)))
        return int(out.value)

    def _tune(self, args: _lib.SearchArgs, key: tuple, n_cfg: int, stream: torch.cuda.Stream) -> None:
        """Time every kernel configuration on this batch (median of ``TUNE_REPS`` launches each)
        and keep :func:`pick_config`'s choice for ``key``. The timing runs do not learn into the
        start order's cost table (the search that follows does, once)."""
        ms = []
        learn = (args.cells, args.cell_cost, args.n_cells)
        args.cells, args.cell_cost, args.n_cells = None, None, 0
        for cfg in range(n_cfg):
            args.kernel_config = cfg
            times = []
            for _ in range(TUNE_REPS):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                _lib.check(self.lib.hnsw_b200_search(self._handle, ctypes.byref(args),
                                                     ctypes.c_void_p(stream.cuda_stream)))
                b.record(stream)
                b.synchronize()
                times.append(a.elapsed_time(b))
            ms.append(float(np.median(times)))
        args.cells, args.cell_cost, args.n_cells = learn
        self.tuned[key] = pick_config(ms)
        self.tune_log[key] = ms
