"""Exact brute-force k-NN on the tensor cores: the GPU counterpart of ``oracle.exact_search``.

``exact_search(data, queries, k, metric)`` keeps the reference's signature and result contract
(``src/hnsw_engine/oracle.py:35-126``): ``(ids int64 (nq, k), distances float64 (nq, k))`` sorted
by ascending distance with ties broken by ascending id. The work runs in ``libhnsw_b200``
(``hnsw_b200_exact_knn``): a tensor-core distance filter, then the k best survivors by
(distance, id). Byte rows (uint8, or float32 rows of integers in [0, 255]) under L2 or inner
product take the integer filter (tcgen05 kind::i8), whose values are the exact distances; other
rows take a BF16 filter with FP32 accumulation and a derived error margin, and their survivors are
re-ranked in float64.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Any

import numpy as np
import torch
from numpy.typing import NDArray

from . import _lib
from .validation import as_matrix, check_k, validate_metric


@dataclass
class ExactStats:
    filter_max_error: float    # measured: largest |filter value - float64 distance| re-scored
    candidates: int
    launches: int
    filter_error_bound: float  # derived bound of the filter's error (margins are twice it)


def exact_search(
    data: Any, queries: Any, k: int, metric: str = "l2", *, device: str | torch.device = "cuda",
    return_stats: bool = False,
) -> Any:
    """Exact ``k`` nearest neighbours of each query; arguments and results as ``oracle.exact_search``.

    ``data``/``queries`` may be numpy arrays (uploaded) or CUDA tensors (used in place); float32
    and uint8 rows are supported (other real dtypes are converted to float32). Results are numpy
    arrays for numpy inputs, device tensors for tensor inputs.
    """
    lib = _lib.load()
    metric = validate_metric(metric)
    on_device = isinstance(data, torch.Tensor) and data.is_cuda
    dev = data.device if on_device else torch.device(device)
    if not on_device:
        x_np = as_matrix(data, "data")
        n, dim = x_np.shape
        if n == 0 or dim == 0:
            raise ValueError(f"data must be non-empty with at least one dimension, got {x_np.shape}")
        q_np = as_matrix(queries, "queries", dim=dim)
        k = check_k(k, n)
        if x_np.dtype == np.uint8 and q_np.dtype == np.uint8:
            x = torch.from_numpy(np.ascontiguousarray(x_np)).to(dev)
            q = torch.from_numpy(np.ascontiguousarray(q_np)).to(dev)
        else:
            x = torch.from_numpy(np.ascontiguousarray(x_np, dtype=np.float32)).to(dev)
            q = torch.from_numpy(np.ascontiguousarray(q_np, dtype=np.float32)).to(dev)
        if metric == "cosine":
            for name, arr in (("data", x_np), ("queries", q_np)):
                norms = np.linalg.norm(np.asarray(arr, np.float64), axis=1)
                zero = np.flatnonzero(norms == 0.0)
                if zero.size:
                    raise ValueError(
                        f"cosine distance is undefined for zero vectors ({name} rows {zero[:5].tolist()})"
                    )
    else:
        x, q = data.contiguous(), queries.to(dev).contiguous()
        n, dim = x.shape
        k = check_k(k, n)
        if not (x.dtype == torch.uint8 and q.dtype == torch.uint8):
            x, q = x.to(torch.float32), q.to(torch.float32)
    nq = q.shape[0]
    ids = torch.empty((nq, k), dtype=torch.int64, device=dev)
    dists = torch.empty((nq, k), dtype=torch.float64, device=dev)
    err = ctypes.c_double(0.0)
    bound = ctypes.c_double(0.0)
    cand = ctypes.c_int64(0)
    launches = ctypes.c_int64(0)
    args = _lib.ExactArgs(
        data=x.data_ptr(), queries=q.data_ptr(),
        dtype=_lib_dtype(x), dim=dim, n=n, nq=nq, k=k, metric=_lib.METRIC_CODES[metric],
        integer_valued=-1, reserved=0, out_ids=ids.data_ptr(), out_dists=dists.data_ptr(),
        out_filter_max_error=ctypes.addressof(err), out_candidates=ctypes.addressof(cand),
        out_launches=ctypes.addressof(launches), out_filter_error_bound=ctypes.addressof(bound),
    )
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.hnsw_b200_exact_knn(ctypes.byref(args), ctypes.c_void_p(stream)))
    stats = ExactStats(err.value, cand.value, launches.value, bound.value)
    out: Any = (ids, dists) if on_device else (ids.cpu().numpy(), dists.cpu().numpy())
    return (*out, stats) if return_stats else out


def _lib_dtype(t: torch.Tensor) -> int:
    return 1 if t.dtype == torch.uint8 else 0


def exact_distances(data: NDArray, queries: NDArray, ids: NDArray, metric: str = "l2") -> NDArray[np.float64]:
    """Float64 distances of given ids (``-1`` -> ``+inf``), host-side, as ``oracle.exact_distances``."""
    x = np.asarray(data)
    q = np.asarray(queries, dtype=np.float64)
    idx = np.asarray(ids, dtype=np.int64)
    out = np.full(idx.shape, np.inf)
    for row in range(q.shape[0]):
        ok = idx[row] >= 0
        if not ok.any():
            continue
        rows = np.asarray(x[idx[row, ok]], dtype=np.float64)
        if metric == "l2":
            diff = rows - q[row]
            out[row, ok] = np.einsum("ij,ij->i", diff, diff)
        elif metric == "ip":
            out[row, ok] = -(rows @ q[row])
        else:
            rows = rows / np.linalg.norm(rows, axis=1)[:, None]
            out[row, ok] = 1.0 - rows @ (q[row] / np.linalg.norm(q[row]))
    return out
