"""Search-side drop-in for the reference's ``HNSWIndex`` (``src/hnsw_engine/index.py:96-466``).

The index opens a graph written by the reference's ``save_native`` (``index.py:390-425``,
``persistence.py:192-243``) and searches it on the GPU with exactly the reference's results. The
public search surface keeps the reference's names, defaults, argument meaning, validation and
error messages:

* ``search(query, k=10, ef=None, filter=None)`` and ``batch_search(queries, k=10, ef=None,
  filter=None)`` (``index.py:244-292``), with ``ef <- max(ef or ef_search, k)`` and an all-false
  filter returning padding without searching (``:289-291``);
* cumulative ``distance_computations`` / ``hops`` counters, ``stats()`` and ``reset_counters()``
  (``:329-365``) with the reference's definitions;
* extension: ``ef`` may also be an integer array with one efSearch per query, and inputs may be
  torch device tensors (``batch_search`` then returns device tensors).

Graph construction is not part of this engine: graphs are built by the reference host build, whose
sequential insertion defines them, and ``add`` says so.
"""

from __future__ import annotations

import json
import math
from dataclasses import asdict, dataclass
from pathlib import Path
from typing import Any

import numpy as np
import torch
from numpy.typing import ArrayLike, NDArray

from . import _lib
from .engine import DeviceGraph
from .validation import (
    NATIVE_ARRAYS,
    as_matrix,
    as_vector,
    check_int,
    check_k,
    check_native_shapes,
    prepare,
    validate_metric,
    validate_native,
)

NATIVE_FORMAT = "hnsw-engine-native"
NATIVE_FORMAT_VERSION = 1
NATIVE_HEADER = "header.json"
SELECTIONS = ("simple", "heuristic")


@dataclass(frozen=True)
class _Uploaded:
    """Checked, prepared queries already on the GPU, with their distance arithmetic."""

    rows: torch.Tensor
    dist_mode: int


@dataclass(frozen=True)
class IndexStats:
    """Summary of an index, with the fields of the reference's ``IndexStats`` (index.py:63-93)."""

    size: int
    dim: int
    metric: str
    engine: str
    M: int
    max_links_layer0: int
    ef_construction: int
    ef_search: int
    m_L: float
    selection: str
    extend_candidates: bool
    keep_pruned_connections: bool
    max_level: int
    entry_point: int
    nodes_per_layer: tuple[int, ...]
    links_per_layer: tuple[int, ...]
    mean_degree_per_layer: tuple[float, ...]
    memory_bytes: int
    distance_computations: int
    hops: int

    def as_dict(self) -> dict[str, Any]:
        return asdict(self)


def read_native(directory: str | Path, mmap: bool = True) -> tuple[dict[str, Any], dict[str, NDArray[Any]]]:
    """Read a ``save_native`` directory; same checks and messages as ``persistence.load_native``."""
    root = Path(directory)
    header_path = root / NATIVE_HEADER
    if not header_path.is_file():
        raise ValueError(f"{root} is not an hnsw-engine native index (no {NATIVE_HEADER})")
    meta: dict[str, Any] = json.loads(header_path.read_text())
    if meta.pop("format", None) != NATIVE_FORMAT:
        raise ValueError(f"{root} is not an hnsw-engine native index")
    version = meta.pop("format_version", None)
    if version != NATIVE_FORMAT_VERSION:
        raise ValueError(f"unsupported native format version {version!r}")
    arrays: dict[str, NDArray[Any]] = {}
    for name, expected in meta.pop("arrays").items():
        array = np.load(root / f"{name}.npy", mmap_mode="r" if mmap else None, allow_pickle=False)
        if str(array.dtype) != expected["dtype"] or list(array.shape) != expected["shape"]:
            raise ValueError(
                f"{name}.npy has dtype {array.dtype} and shape {array.shape}, header says "
                f"{expected['dtype']} and {tuple(expected['shape'])}"
            )
        arrays[name] = np.asarray(array)
    return meta, arrays


class HNSWIndex:
    """An HNSW graph built by the reference, searched on one B200.

    Open one with :meth:`load_native` (a ``save_native`` directory) or :meth:`from_arrays`.
    Constructor parameters mirror the reference's (``index.py:115-149``); only ``ef_search`` and
    ``metric`` affect searching. Extensions: ``device``, and ``locality`` (store the graph on the
    GPU in a cell order for memory locality; ``None`` turns it on from 65,536 nodes; results are
    the same either way).
    """

    def __init__(
        self,
        dim: int,
        metric: str = "l2",
        M: int = 16,
        ef_construction: int = 200,
        ef_search: int = 50,
        seed: int | None = None,
        selection: str = "heuristic",
        extend_candidates: bool = False,
        keep_pruned_connections: bool = False,
        m_L: float | None = None,
        engine: str = "b200",
        device: str | torch.device = "cuda",
        locality: bool | None = None,
    ) -> None:
        self._dim = check_int(dim, "dim", minimum=1)
        self._metric = validate_metric(metric)
        self._M = check_int(M, "M", minimum=2)
        self._ef_construction = check_int(ef_construction, "ef_construction", minimum=1)
        self._ef_search = check_int(ef_search, "ef_search", minimum=1)
        self._seed = None if seed is None else check_int(seed, "seed", minimum=0)
        if selection not in SELECTIONS:
            raise ValueError(f"unknown selection {selection!r}; expected one of {SELECTIONS}")
        self._selection = selection
        self._extend_candidates = bool(extend_candidates)
        self._keep_pruned = bool(keep_pruned_connections)
        self._m_L = 1.0 / math.log(self._M) if m_L is None else float(m_L)
        self._engine_name = engine
        self._device = device
        self._locality = locality  # device node order: None = automatic (see engine.DeviceGraph)
        self._graph: DeviceGraph | None = None
        self._arrays: dict[str, NDArray[Any]] | None = None
        self._size = 0
        self._counters = np.zeros(2, dtype=np.int64)  # distance computations, hops
        self._counters_dev: torch.Tensor | None = None  # device-side share not yet read back
        self._meta_extra: dict[str, Any] = {}

    # ----------------------------------------------------------------------- opening
    @classmethod
    def load_native(
        cls, directory: str | Path, mmap: bool = True, validate: bool = True,
        device: str | torch.device = "cuda", locality: bool | None = None,
    ) -> HNSWIndex:
        """Open a directory written by the reference's ``HNSWIndex.save_native``."""
        meta, arrays = read_native(directory, mmap=mmap)
        params = {k: v for k, v in meta["params"].items() if k != "engine"}
        index = cls(**params, device=device, locality=locality)
        index._meta_extra = {"rng_state": meta.get("rng_state")}
        index._attach(arrays, int(meta["entry_point"]), int(meta["max_level"]), validate)
        return index

    @classmethod
    def from_arrays(
        cls, arrays: dict[str, NDArray[Any]], entry_point: int, max_level: int, *, validate: bool = True,
        **params: Any,
    ) -> HNSWIndex:
        """Wrap native arrays (``NumbaEngine.native_arrays()`` layout) already in memory."""
        index = cls(**params)
        index._attach(arrays, int(entry_point), int(max_level), validate)
        return index

    def _attach(self, arrays: dict[str, NDArray[Any]], entry_point: int, max_level: int,
                validate: bool) -> None:
        check_native_shapes(arrays, self._dim, self._M)
        size = int(arrays["vectors"].shape[0])
        if validate and size == 0:
            validate_native(arrays, entry_point, max_level, self._M)
        self._arrays = {name: arrays[name] for name in NATIVE_ARRAYS}
        if size:
            # validate: the reference's checks, run on the GPU over the uploaded arrays
            self._graph = DeviceGraph(self._arrays, entry_point, max_level, self._metric, self._device,
                                      locality=self._locality, validate_M=self._M if validate else None)
        self._size = size
        self._entry_point = entry_point
        self._max_level = max_level

    # ---------------------------------------------------------------------- properties
    @property
    def dim(self) -> int:
        return self._dim

    @property
    def metric(self) -> str:
        return self._metric

    @property
    def M(self) -> int:
        return self._M

    @property
    def ef_search(self) -> int:
        return self._ef_search

    @ef_search.setter
    def ef_search(self, value: int) -> None:
        self._ef_search = check_int(value, "ef_search", minimum=1)

    @property
    def engine(self) -> str:
        return self._engine_name

    @property
    def entry_point(self) -> int:
        return self._entry_point if self._size else -1

    @property
    def max_level(self) -> int:
        return self._max_level if self._size else -1

    @property
    def device_graph(self) -> DeviceGraph:
        if self._graph is None:
            raise ValueError("cannot search an empty index")
        return self._graph

    @property
    def distance_computations(self) -> int:
        return int(self._read_counters()[0])

    @property
    def hops(self) -> int:
        return int(self._read_counters()[1])

    def _read_counters(self) -> NDArray[np.int64]:
        """Fold the searches' device-side counter sums into the host totals (one small copy)."""
        if self._counters_dev is not None:
            self._counters += self._counters_dev.cpu().numpy()
            self._counters_dev = None
        return self._counters

    def native_arrays(self) -> dict[str, NDArray[Any]]:
        if self._arrays is None:
            raise ValueError("the index holds no graph")
        return self._arrays

    def __len__(self) -> int:
        return self._size

    def __repr__(self) -> str:
        return (
            f"HNSWIndex(dim={self._dim}, metric={self._metric!r}, M={self._M}, "
            f"ef_search={self._ef_search}, engine={self._engine_name!r}, size={len(self)})"
        )

    # -------------------------------------------------------------------- construction
    def add(self, vectors: ArrayLike) -> NDArray[np.int64]:
        raise NotImplementedError(
            "graph construction stays on the reference host build (hnsw_engine.HNSWIndex.add, "
            "then save_native); open the result with HNSWIndex.load_native"
        )

    # --------------------------------------------------------------------------- search
    def _prepare(self, vectors: ArrayLike) -> NDArray[np.float32]:
        return prepare(as_matrix(vectors, "vectors", dim=self._dim), self._metric)

    def _upload(self, vectors: ArrayLike) -> Any:
        """Host queries for a device search, with :meth:`_prepare`'s checks, messages and values.

        C-contiguous float32 rows of the right width under l2 or ip are already their prepared
        form: the library copies them to the GPU while its host threads read them for the NaN/inf
        check and for the statistics that pick the distance arithmetic, so nothing is read back
        from the GPU (``_Uploaded``). Every other input is checked and prepared by NumPy, straight
        into page-locked memory."""
        a = np.asarray(vectors)
        if (self._metric != "cosine" and a.dtype == np.float32 and a.ndim == 2
                and a.shape[1] == self._dim and a.flags.c_contiguous):
            g = self.device_graph
            rows = torch.empty(a.shape, dtype=torch.float32, device=g.device)
            st = g.upload_queries(a, rows)
            if not st.finite:
                raise ValueError("vectors contains NaN or infinite values")
            return _Uploaded(rows, g.mode_from_stats(st, a))
        rows = as_matrix(a, "vectors", dim=self._dim)
        staged = torch.empty(rows.shape, dtype=torch.float32, pin_memory=True)
        prepare(rows, self._metric, out=staged.numpy(), checked_finite=True)
        return staged

    def _device_queries(self, queries: torch.Tensor) -> _Uploaded:
        """Queries already on the GPU, with :meth:`_prepare`'s checks and messages (shape, real
        dtype, width, NaN/inf, cosine zero rows, float32 overflow) and its values, read back as one
        small copy that also carries the statistics picking the distance arithmetic."""
        if queries.ndim != 2:
            raise ValueError(f"vectors must be a 2-D array, got shape {tuple(queries.shape)}")
        if queries.dtype == torch.bool or queries.is_complex():
            dtype = str(queries.dtype).removeprefix("torch.")
            raise ValueError(f"vectors must contain real numbers, got dtype {dtype}")
        if queries.shape[1] != self._dim:
            raise ValueError(f"vectors has dimension {queries.shape[1]}, expected {self._dim}")
        g = self.device_graph
        with torch.cuda.device(queries.device):
            if queries.numel() == 0:
                return _Uploaded(queries.to(torch.float32).contiguous(), _lib.DIST_F64)
            raw_finite = torch.isfinite(queries).all()
            zero_rows = torch.zeros((), dtype=torch.bool, device=queries.device)
            if self._metric == "cosine":
                q64 = queries.to(torch.float64)
                norms = torch.linalg.norm(q64, dim=1, keepdim=True)
                zero_rows = (norms == 0).any()
                rows = (q64 / norms).to(torch.float32).contiguous()
            else:
                rows = queries.to(torch.float32).contiguous()
            lo, hi = torch.aminmax(rows)
            flags = torch.stack([raw_finite.double(), zero_rows.double(),
                                 torch.isfinite(rows).all().double(),
                                 (rows != torch.round(rows)).any().double(), lo.double(),
                                 hi.double()]).cpu().tolist()
        if not flags[0]:
            raise ValueError("vectors contains NaN or infinite values")
        if flags[1]:
            rows_host = torch.nonzero(norms[:, 0] == 0).flatten()[:5].cpu().tolist()
            raise ValueError(f"cosine distance is undefined for zero vectors (rows {rows_host})")
        if not flags[2]:
            raise ValueError("vectors overflow float32 (values beyond about 3.4e38)")
        mode = g.choose_mode_device(rows, False, stats=(not flags[3], flags[4], flags[5]))
        return _Uploaded(rows, mode)

    def _check_search_args(self, k: int, ef: Any) -> tuple[int, Any]:
        if len(self) == 0:
            raise ValueError("cannot search an empty index")
        k_valid = check_k(k, len(self))
        if ef is None:
            return k_valid, max(self._ef_search, k_valid)
        if isinstance(ef, (np.ndarray, torch.Tensor, list, tuple)):
            arr = np.asarray(ef.cpu() if isinstance(ef, torch.Tensor) else ef)
            if arr.ndim != 1 or not np.issubdtype(arr.dtype, np.integer):
                raise TypeError("ef must be an integer or a 1-D integer array (one per query)")
            if arr.size and arr.min() < 1:
                raise ValueError(f"ef must be >= 1, got {int(arr.min())}")
            return k_valid, np.maximum(arr.astype(np.int32), k_valid)
        return k_valid, max(check_int(ef, "ef", minimum=1), k_valid)

    def _check_filter(self, filter: ArrayLike | None) -> NDArray[np.bool_] | None:
        if filter is None:
            return None
        mask = np.asarray(filter.cpu() if isinstance(filter, torch.Tensor) else filter)
        if mask.dtype != np.bool_:
            raise TypeError(f"filter must be a boolean array, got dtype {mask.dtype}")
        if mask.shape != (len(self),):
            raise ValueError(
                f"filter must have one entry per indexed vector ({len(self)}), got shape "
                f"{mask.shape}"
            )
        return np.ascontiguousarray(mask)

    def search(
        self, query: ArrayLike, k: int = 10, ef: int | None = None, filter: ArrayLike | None = None
    ) -> tuple[NDArray[np.int64], NDArray[np.float64]]:
        """Approximate ``k`` nearest neighbours of one ``(dim,)`` query (reference ``index.py:244-273``)."""
        k_valid, ef_valid = self._check_search_args(k, ef)
        allowed = self._check_filter(filter)
        prepared = self._prepare(as_vector(query, "query", dim=self._dim)[None, :])
        if allowed is not None and not allowed.any():
            return np.full(k_valid, -1, dtype=np.int64), np.full(k_valid, np.inf)
        if allowed is None and np.isscalar(ef_valid):  # the latency path
            ids, dists, ctr = self.device_graph.search_one(prepared[0], k_valid, int(ef_valid))
            self._counters += ctr
            return ids, dists
        ids, dists = self._run(prepared, k_valid, ef_valid, allowed)
        return ids[0], dists[0]

    def batch_search(
        self, queries: Any, k: int = 10, ef: Any = None, filter: ArrayLike | None = None,
        stop: Any = None, exact_below: float | None = None,
    ) -> tuple[Any, Any]:
        """:meth:`search` for each row of ``(nq, dim)`` queries (reference ``index.py:275-292``).

        ``ef`` may be one integer or an array of one efSearch per query. Torch device queries give
        device results (no host round trip); host queries give numpy results.

        Extensions:

        * ``stop``: a trained :class:`~hnsw_engine_b200.learned_stop.StopNetwork` ends each
          unfiltered query early once the network predicts no further recall gain (``ef`` is then
          the cap).
        * ``exact_below``: a selectivity planner. When the filter allows fewer than this share of
          the nodes, the batch is answered by the tensor-core exact k-NN over the allowed rows
          instead of the graph walk, which must pass through about 1/share nodes per result
          (the policy of the reference's ``benchmarks/run_filtered.py:76-106``). The results are
          then the exact neighbours among the allowed nodes, as ``oracle.exact_search`` gives them;
          the distance counter adds one per (query, allowed node).
        """
        k_valid, ef_valid = self._check_search_args(k, ef)
        allowed = self._check_filter(filter)
        on_device = isinstance(queries, torch.Tensor) and queries.is_cuda
        if on_device:
            prepared: Any = self._device_queries(queries)
        elif allowed is not None and not allowed.any():
            prepared = self._prepare(queries)  # validated; no device work follows
        else:
            prepared = self._upload(queries)
        dist_mode = None
        if isinstance(prepared, _Uploaded):
            prepared, dist_mode = prepared.rows, prepared.dist_mode
        nq = prepared.shape[0]
        if allowed is not None and not allowed.any():
            ids = np.full((nq, k_valid), -1, dtype=np.int64)
            dists = np.full((nq, k_valid), np.inf)
            if on_device:
                return torch.from_numpy(ids).to(queries.device), torch.from_numpy(dists).to(queries.device)
            return ids, dists
        if allowed is not None and exact_below is not None and allowed.mean() < float(exact_below):
            return self._exact_subset(prepared, k_valid, allowed, keep_device=on_device)
        ids_t, dists_t = self._run(prepared, k_valid, ef_valid, allowed, keep_device=on_device,
                                   stop=stop, dist_mode=dist_mode)
        return ids_t, dists_t

    def _exact_subset(self, prepared: Any, k: int, allowed: NDArray[np.bool_],
                      keep_device: bool = False) -> tuple[Any, Any]:
        """Exact k nearest allowed nodes (ties to the lower id), padded with -1 / inf."""
        from .exact_knn import exact_search

        g = self.device_graph
        dev = g.device
        sub = torch.from_numpy(np.flatnonzero(allowed)).to(dev)
        q = prepared if isinstance(prepared, torch.Tensor) else torch.from_numpy(prepared)
        q = q.to(device=dev, dtype=torch.float32).contiguous()
        nq = q.shape[0]
        kk = min(k, int(sub.numel()))
        ids = torch.full((nq, k), -1, dtype=torch.int64, device=dev)
        dists = torch.full((nq, k), float("inf"), dtype=torch.float64, device=dev)
        if nq and kk:
            sub_ids, sub_d = exact_search(g.vectors[sub].contiguous(), q, kk, self._metric)
            ids[:, :kk] = sub[sub_ids]
            dists[:, :kk] = sub_d
        self._counters[0] += nq * int(sub.numel())
        if keep_device:
            return ids, dists
        return ids.cpu().numpy(), dists.cpu().numpy()

    def _run(self, prepared: Any, k: int, ef: Any, allowed: NDArray[np.bool_] | None,
             keep_device: bool = False, stop: Any = None,
             dist_mode: int | None = None) -> tuple[Any, Any]:
        g = self.device_graph
        stop_arg = None
        if stop is not None and allowed is None:
            packed = getattr(stop, "_packed_cache", None)
            if packed is None:
                packed = stop.packed()
                stop._packed_cache = packed
            stop_arg = (packed, stop.threshold, stop.slope, stop.slope_from)
        ids, dists, ctr = g.search(prepared, k, ef, allowed=allowed, stop=stop_arg,
                                   dist_mode=dist_mode)
        self._accumulate(ctr)
        if keep_device:
            return ids, dists
        # results into page-locked host memory, one synchronisation for both copies
        ids_h = torch.empty(ids.shape, dtype=ids.dtype, pin_memory=True)
        dists_h = torch.empty(dists.shape, dtype=dists.dtype, pin_memory=True)
        ids_h.copy_(ids, non_blocking=True)
        dists_h.copy_(dists, non_blocking=True)
        torch.cuda.current_stream(g.device).synchronize()
        return ids_h.numpy(), dists_h.numpy()

    def _accumulate(self, ctr: torch.Tensor | None) -> None:
        """Add a search's per-query counters to the running totals on the device (no sync)."""
        if ctr is not None and ctr.numel():
            s = ctr.sum(dim=0)
            self._counters_dev = s if self._counters_dev is None else self._counters_dev + s

    # ----------------------------------------------------------------------- inspection
    def stats(self) -> IndexStats:
        """Sizes, layer structure, degrees, memory estimate and cumulative counters (index.py:329-360)."""
        arrays = self._arrays
        if arrays is None or self._size == 0:
            nodes: tuple[int, ...] = ()
            links: tuple[int, ...] = ()
        else:
            levels = arrays["levels"]
            top = int(levels.max())
            nodes = tuple(int((levels >= layer).sum()) for layer in range(top + 1))
            link_counts = [int(arrays["count0"].sum())]
            if top > 0:
                upper = np.flatnonzero(levels > 0)
                offs = arrays["upper_offset"][upper]
                lv = levels[upper]
                for layer in range(1, top + 1):
                    sel = lv >= layer
                    link_counts.append(int(arrays["count_up"][offs[sel] + layer - 1].sum()))
            links = tuple(link_counts)
        degrees = tuple(lk / nd if nd else 0.0 for lk, nd in zip(links, nodes, strict=True))
        slots = sum(nd * ((2 * self._M if layer == 0 else self._M) + 1) for layer, nd in enumerate(nodes))
        memory = self._size * self._dim * 4 + slots * 4 + self._size * 4
        return IndexStats(
            size=self._size, dim=self._dim, metric=self._metric, engine=self._engine_name, M=self._M,
            max_links_layer0=2 * self._M, ef_construction=self._ef_construction,
            ef_search=self._ef_search, m_L=self._m_L, selection=self._selection,
            extend_candidates=self._extend_candidates, keep_pruned_connections=self._keep_pruned,
            max_level=self.max_level, entry_point=self.entry_point, nodes_per_layer=nodes,
            links_per_layer=links, mean_degree_per_layer=degrees, memory_bytes=memory,
            distance_computations=self.distance_computations, hops=self.hops,
        )

    def reset_counters(self) -> None:
        self._counters[:] = 0
        self._counters_dev = None

    def _params(self) -> dict[str, Any]:
        return {
            "dim": self._dim, "metric": self._metric, "M": self._M,
            "ef_construction": self._ef_construction, "ef_search": self._ef_search,
            "seed": self._seed, "selection": self._selection,
            "extend_candidates": self._extend_candidates,
            "keep_pruned_connections": self._keep_pruned, "m_L": self._m_L, "engine": "numba",
        }

    def save_native(self, directory: str | Path) -> None:
        """Write the graph back in the reference's native layout (header written last)."""
        arrays = self.native_arrays()
        root = Path(directory)
        root.mkdir(parents=True, exist_ok=True)
        (root / NATIVE_HEADER).unlink(missing_ok=True)
        layout = {}
        for name in NATIVE_ARRAYS:
            np.save(root / f"{name}.npy", np.ascontiguousarray(arrays[name]), allow_pickle=False)
            layout[name] = {"dtype": str(arrays[name].dtype), "shape": list(arrays[name].shape)}
        header = {
            "format": NATIVE_FORMAT, "format_version": NATIVE_FORMAT_VERSION, "arrays": layout,
            "params": self._params(), "rng_state": self._meta_extra.get("rng_state"),
            "entry_point": self.entry_point, "max_level": self.max_level,
        }
        (root / NATIVE_HEADER).write_text(json.dumps(header, indent=2))
