"""Host-side validation and query preparation, with the reference's semantics and messages.

Restates, in this package's own code:

* ``check_int``, ``as_matrix``, ``as_vector``, ``check_k`` -- ``src/hnsw_engine/_validation.py:16-66``
  (same exception types and message wording, so callers see identical errors);
* ``prepare`` -- ``src/hnsw_engine/metrics.py:42-68`` (float32 cast; cosine divides by the float64
  norm first and rejects zero rows);
* ``validate_native`` -- the checks ``NumbaEngine.attach_native`` and ``_validate_native`` run before
  the compiled search may follow a link (``src/hnsw_engine/numba_engine.py:841-927``). The CUDA
  kernels do not bounds-check link ids either, so every graph is validated here before upload.
"""

from __future__ import annotations

import numbers
from typing import Any

import numpy as np
from numpy.typing import ArrayLike, NDArray

METRICS = ("l2", "cosine", "ip")
NATIVE_ARRAYS = ("vectors", "levels", "links0", "count0", "upper_offset", "links_up", "count_up")


def validate_metric(metric: object) -> str:
    if metric not in METRICS:
        raise ValueError(f"unknown metric {metric!r}; expected one of {METRICS}")
    return str(metric)


def check_int(value: object, name: str, *, minimum: int | None = None) -> int:
    if isinstance(value, bool) or not isinstance(value, numbers.Integral):
        raise TypeError(f"{name} must be an integer, got {type(value).__name__}")
    result = int(value)
    if minimum is not None and result < minimum:
        raise ValueError(f"{name} must be >= {minimum}, got {result}")
    return result


def _real_and_finite(array: NDArray[Any], name: str) -> None:
    if not (np.issubdtype(array.dtype, np.integer) or np.issubdtype(array.dtype, np.floating)):
        raise ValueError(f"{name} must contain real numbers, got dtype {array.dtype}")
    if np.issubdtype(array.dtype, np.floating) and not np.isfinite(array).all():
        raise ValueError(f"{name} contains NaN or infinite values")


def as_matrix(values: ArrayLike, name: str, *, dim: int | None = None) -> NDArray[Any]:
    array = np.asarray(values)
    if array.ndim != 2:
        raise ValueError(f"{name} must be a 2-D array, got shape {array.shape}")
    _real_and_finite(array, name)
    if dim is not None and array.shape[1] != dim:
        raise ValueError(f"{name} has dimension {array.shape[1]}, expected {dim}")
    return array


def as_vector(values: ArrayLike, name: str, *, dim: int) -> NDArray[Any]:
    array = np.asarray(values)
    if array.ndim != 1:
        raise ValueError(f"{name} must be a 1-D array, got shape {array.shape}")
    _real_and_finite(array, name)
    if array.shape[0] != dim:
        raise ValueError(f"{name} has dimension {array.shape[0]}, expected {dim}")
    return array


def check_k(k: object, n: int) -> int:
    k_int = check_int(k, "k", minimum=1)
    if k_int > n:
        raise ValueError(f"k={k_int} exceeds the number of indexed vectors ({n})")
    return k_int


def _exact_in_float32(dtype: np.dtype) -> bool:
    """Finite values of this dtype stay finite in float32 (no overflow on the cast)."""
    return bool(np.issubdtype(dtype, np.integer) or dtype in (np.float16, np.float32))


def prepare(vectors: NDArray[Any], metric: str, out: NDArray[np.float32] | None = None,
            checked_finite: bool = False) -> NDArray[np.float32]:
    """Stored representation of validated rows: contiguous float32 (cosine: float64-normalised).

    ``out``: a C-contiguous float32 array of the same shape to write into (a pinned staging
    buffer), else a new array (or ``vectors`` itself when already contiguous float32).
    ``checked_finite``: the rows already passed :func:`as_matrix`, so the overflow check after a
    cast that cannot overflow (integers, float16, float32) is skipped."""
    if metric != "cosine":
        with np.errstate(over="ignore"):
            if out is None:
                direct = np.ascontiguousarray(vectors, dtype=np.float32)
            else:
                np.copyto(out, vectors, casting="unsafe")
                direct = out
        skip = checked_finite and _exact_in_float32(np.asarray(vectors).dtype)
        if not skip and not np.isfinite(direct).all():
            raise ValueError("vectors overflow float32 (values beyond about 3.4e38)")
        return direct
    as64 = np.asarray(vectors, dtype=np.float64)
    norms = np.linalg.norm(as64, axis=1)
    zero_rows = np.flatnonzero(norms == 0.0)
    if zero_rows.size:
        raise ValueError(
            f"cosine distance is undefined for zero vectors (rows {zero_rows[:5].tolist()})"
        )
    with np.errstate(over="ignore"):
        if out is None:
            out = np.ascontiguousarray(as64 / norms[:, None], dtype=np.float32)
        else:
            np.copyto(out, as64 / norms[:, None], casting="unsafe")
    if not np.isfinite(out).all():
        raise ValueError("vectors overflow float32 (values beyond about 3.4e38)")
    return out


def check_native_shapes(arrays: dict[str, NDArray[Any]], dim: int, M: int) -> None:
    """Dtype/shape table of the native layout, and levels summing to the upper rows."""
    n = arrays["vectors"].shape[0]
    rows = arrays["links_up"].shape[0]
    expected = {
        "vectors": (np.float32, (n, dim)),
        "levels": (np.int64, (n,)),
        "links0": (np.int32, (n, 2 * M + 1)),
        "count0": (np.int32, (n,)),
        "upper_offset": (np.int64, (n,)),
        "links_up": (np.int32, (rows, M + 1)),
        "count_up": (np.int32, (rows,)),
    }
    for name, (dtype, shape) in expected.items():
        array = arrays[name]
        if array.dtype != dtype or array.shape != shape:
            raise ValueError(
                f"{name} has dtype {array.dtype} and shape {array.shape}, expected "
                f"{np.dtype(dtype)} and {shape}"
            )
    if int(arrays["levels"].sum()) != rows:
        raise ValueError("upper-layer rows do not match the node levels")


def _used_links(links: NDArray[np.int32], counts: NDArray[np.int32], n: int, cap: int,
                where: str) -> NDArray[np.int32]:
    if (counts < 0).any() or (counts > cap).any():
        raise ValueError(f"{where}: link counts outside [0, {cap}]")
    used = np.arange(links.shape[1])[None, :] < counts[:, None]
    values = links[used]
    if values.size and ((values < 0).any() or (values >= n).any()):
        raise ValueError(f"{where}: a link points outside the graph")
    return values


def validate_native(arrays: dict[str, NDArray[Any]], entry_point: int, max_level: int,
                    M: int) -> None:
    """Raise ``ValueError`` unless every link the search can follow is a valid node on its layer."""
    levels = arrays["levels"]
    n, rows = levels.shape[0], arrays["links_up"].shape[0]
    if n == 0:
        if rows or entry_point != -1 or max_level != -1:
            raise ValueError("an empty graph has no entry point and no layers")
        return
    if (levels < 0).any():
        raise ValueError("negative node level")
    top = int(levels.max())
    if max_level != top or not 0 <= entry_point < n or int(levels[entry_point]) != top:
        raise ValueError("the entry point is not a node of the top layer")
    _used_links(arrays["links0"], arrays["count0"], n, 2 * M, "layer 0")
    upper = np.flatnonzero(levels > 0)
    offsets = arrays["upper_offset"][upper]
    order = np.argsort(offsets, kind="stable")
    starts, sizes = offsets[order], levels[upper][order]
    ends = starts + sizes
    tiles = starts.size == 0 or (
        starts[0] == 0 and ends[-1] == rows and bool((starts[1:] == ends[:-1]).all())
    )
    if not tiles or (starts.size == 0 and rows):
        raise ValueError("upper-layer rows of the nodes overlap or leave gaps")
    count_up = arrays["count_up"]
    targets = _used_links(arrays["links_up"], count_up, n, M, "upper layers")
    layer_of_row = np.arange(rows) - np.repeat(starts, sizes) + 1
    if (levels[targets] < np.repeat(layer_of_row, count_up)).any():
        raise ValueError("an upper-layer link points to a node absent from that layer")


# Messages of validate_native, in its order of checks, for the failure bits of the on-device
# validator (hnsw_b200_validate_graph, HNSW_B200_BAD_* in include/hnsw_b200.h).
def device_validation_message(flags: int, M: int) -> str | None:
    """The message validate_native raises for the first failed check, or None if none failed."""
    messages = (
        "negative node level",
        "the entry point is not a node of the top layer",
        f"layer 0: link counts outside [0, {2 * M}]",
        "layer 0: a link points outside the graph",
        "upper-layer rows of the nodes overlap or leave gaps",
        f"upper layers: link counts outside [0, {M}]",
        "upper layers: a link points outside the graph",
        "an upper-layer link points to a node absent from that layer",
    )
    for bit, message in enumerate(messages):
        if flags >> bit & 1:
            return message
    return None
