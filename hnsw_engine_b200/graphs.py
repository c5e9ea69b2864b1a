"""The standard workloads: synthetic data plus the reference-built graph over it.

Each workload names a generator, its seeds and the build parameters the reference host build
used (``graphs/build_graphs.py``). :func:`open_workload` returns the native directory's arrays
with the vectors regenerated from the seed when the directory ships without ``vectors.npy``; the
regenerated bytes are checked against the SHA-256 the build recorded, so a mismatch in the
generator can never silently pair a graph with the wrong vectors.
"""

from __future__ import annotations

import hashlib
import json
from pathlib import Path
from typing import Any

import numpy as np
from numpy.typing import NDArray

from . import synthetic

GRAPH_ROOT = Path(__file__).resolve().parent.parent / "graphs"

WORKLOADS: dict[str, dict[str, Any]] = {
    # 10K x 128 integer mixture, L2 (the reference's CPU-runnable case).
    "mix10k": {"gen": "mixture", "n": 10_000, "dim": 128, "metric": "l2", "M": 16,
               "ef_construction": 200, "level_seed": 42, "data_seed": synthetic.DATA_SEED,
               "query_seed": synthetic.QUERY_SEED, "nq": 1_000},
    # 100K x 128 integer mixture, L2 (mid-size development case).
    "mix100k": {"gen": "mixture", "n": 100_000, "dim": 128, "metric": "l2", "M": 16,
                "ef_construction": 200, "level_seed": 42, "data_seed": synthetic.DATA_SEED,
                "query_seed": synthetic.QUERY_SEED, "nq": 10_000},
    # 1M x 128 integer mixture, L2 (the batched-at-scale workload).
    "mix1m": {"gen": "mixture", "n": 1_000_000, "dim": 128, "metric": "l2", "M": 16,
              "ef_construction": 200, "level_seed": 42, "data_seed": synthetic.DATA_SEED,
              "query_seed": synthetic.QUERY_SEED, "nq": 10_000},
    # 1M x 100 Student-t unit vectors, cosine.
    "t1m": {"gen": "student_t", "n": 1_000_000, "dim": 100, "metric": "cosine", "M": 16,
            "ef_construction": 200, "level_seed": 42, "data_seed": synthetic.T_DATA_SEED,
            "query_seed": synthetic.T_QUERY_SEED, "nq": 10_000},
    # 100K x 100 Student-t unit vectors, cosine (mid-size development case).
    "t100k": {"gen": "student_t", "n": 100_000, "dim": 100, "metric": "cosine", "M": 16,
              "ef_construction": 200, "level_seed": 42, "data_seed": synthetic.T_DATA_SEED,
              "query_seed": synthetic.T_QUERY_SEED, "nq": 10_000},
}


def _generate(gen: str, n: int, dim: int, seed: int) -> NDArray[np.float32]:
    if gen == "mixture":
        return synthetic.mixture(n, seed, dim)
    if gen == "student_t":
        return synthetic.student_t_unit(n, seed, dim)
    if gen == "image":
        return synthetic.image_like(n, seed)
    raise ValueError(f"unknown generator {gen!r}")


def workload_vectors(name: str) -> NDArray[np.float32]:
    """The workload's data rows as handed to the reference's ``HNSWIndex.add`` by the build.

    For cosine workloads the generator's rows are normalised once more here (float64, then cast),
    so the data given to the build is already unit-length; the reference's ``prepare`` then
    normalises again when it stores them (:func:`stored_vectors`).
    """
    spec = WORKLOADS[name]
    x = _generate(spec["gen"], spec["n"], spec["dim"], spec["data_seed"])
    if spec["metric"] == "cosine":  # metrics.prepare: float64 normalise then cast
        x64 = x.astype(np.float64)
        x = np.ascontiguousarray(x64 / np.linalg.norm(x64, axis=1)[:, None], dtype=np.float32)
    return x


def stored_vectors(name: str) -> NDArray[np.float32]:
    """The rows the built graph holds: the reference's ``prepare`` of :func:`workload_vectors`."""
    from .validation import prepare

    return prepare(workload_vectors(name), WORKLOADS[name]["metric"])


def workload_queries(name: str, nq: int | None = None, seed: int | None = None) -> NDArray[np.float32]:
    """The workload's query rows (raw generator output; the index prepares them)."""
    spec = WORKLOADS[name]
    count = spec["nq"] if nq is None else nq
    return _generate(spec["gen"], count, spec["dim"], spec["query_seed"] if seed is None else seed)


def graph_dir(name: str) -> Path:
    return GRAPH_ROOT / name


def available(name: str) -> bool:
    return (graph_dir(name) / "header.json").is_file()


def open_workload(name: str, mmap: bool = True) -> tuple[dict[str, Any], dict[str, NDArray[Any]]]:
    """``(meta, arrays)`` of a built workload graph, in the reference's native layout.

    Raises ``FileNotFoundError`` if the graph has not been built.
    """
    root = graph_dir(name)
    header_path = root / "header.json"
    if not header_path.is_file():
        raise FileNotFoundError(f"graph {name!r} is not built ({root}); run graphs/build_graphs.py")
    meta = json.loads(header_path.read_text())
    arrays: dict[str, NDArray[Any]] = {}
    for array_name, expected in meta["arrays"].items():
        path = root / f"{array_name}.npy"
        if array_name == "vectors" and not path.is_file():
            vec = stored_vectors(name)
            digest = hashlib.sha256(vec.tobytes()).hexdigest()
            want = (root / "vectors.sha256").read_text().strip()
            if digest != want:
                raise ValueError(f"regenerated vectors of {name!r} do not match the built graph")
            arrays[array_name] = vec
            continue
        arr = np.load(path, mmap_mode="r" if mmap else None, allow_pickle=False)
        if str(arr.dtype) != expected["dtype"] or list(arr.shape) != expected["shape"]:
            raise ValueError(f"{path} does not match its header")
        arrays[array_name] = np.asarray(arr)
    return meta, arrays
