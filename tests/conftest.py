"""Shared fixtures: golden reference outputs and the graphs they were produced on."""

from __future__ import annotations

import sys
from pathlib import Path
from typing import Any

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GRAPH_KEYS = ("levels", "links0", "count0", "upper_offset", "links_up", "count_up")


def pytest_configure(config: pytest.Config) -> None:
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests of the CUDA path")
    config.addinivalue_line("markers", "slow: long-running")


def load_golden(name: str) -> dict[str, Any]:
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


_MIX10K: dict[str, Any] | None = None


def mix10k_arrays() -> tuple[dict[str, np.ndarray], int, int]:
    """Native arrays of the 10K mixture graph (links from the fixture, vectors regenerated)."""
    global _MIX10K
    if _MIX10K is None:
        from hnsw_engine_b200.graphs import workload_vectors

        g = load_golden("graph_mix10k")
        arrays = {k: g[k] for k in GRAPH_KEYS}
        arrays["vectors"] = workload_vectors("mix10k")
        _MIX10K = {"arrays": arrays, "ep": int(g["entry_point"]), "ml": int(g["max_level"])}
    return _MIX10K["arrays"], _MIX10K["ep"], _MIX10K["ml"]


def case_arrays(case: dict[str, Any], name: str) -> tuple[dict[str, np.ndarray], int, int]:
    if "links0" in case:
        arrays = {k: case[k] for k in GRAPH_KEYS}
        arrays["vectors"] = case["vectors"]
        return arrays, int(case["entry_point"]), int(case["max_level"])
    assert name.startswith("mix10k"), name
    return mix10k_arrays()


SEARCH_CASES = [
    "int_l2", "int_ip", "cont_l2", "cont_ip", "cont_cosine", "complete_l2", "complete_ip",
    "padding", "few_allowed", "mix10k", "mix10k_filtered",
]
QUANT_CASES = ["mix10k", "cont_cosine", "cont_ip", "cont_l2"]


def iter_search_runs(case: dict[str, Any]):
    """(mask_index, mask or None, ef) for every stored run of a search case."""
    for mi in range(int(case["n_masks"])):
        mask = case.get(f"mask{mi}")
        for ef in case["efs"]:
            yield mi, mask, int(ef)


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False
