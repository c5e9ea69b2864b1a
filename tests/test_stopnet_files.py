"""The stop network shipped with the package, read as files (no GPU): its metadata carries the
threshold schedule the trainer uses and the feature list the kernel computes."""

from __future__ import annotations

import json

import numpy as np


def test_shipped_network_carries_its_threshold_schedule() -> None:
    from hnsw_engine_b200.learned_stop import FEATURE_NAMES
    from hnsw_engine_b200.train_stop import SHIPPED, STOP_SLOPE, STOP_SLOPE_FROM

    root = SHIPPED / "mix1m"
    meta = json.loads((root / "meta.json").read_text())
    assert tuple(meta["features"]) == FEATURE_NAMES
    assert (meta["slope"], meta["slope_from"]) == (STOP_SLOPE, STOP_SLOPE_FROM)
    assert meta["ef_cap"] == 192 and np.isfinite(meta["threshold"])
    params = np.load(root / "params.npy")
    assert params.dtype == np.float32 and params.size == 12 * 64 + 64 + 64 * 64 + 64 + 64 + 1
    assert np.isfinite(params).all()


def test_shipped_student_t_network_uses_a_constant_threshold_at_cap_512() -> None:
    """The network for the 1M Student-t cosine graph (which reaches recall 0.832 at ef = 512) is
    tuned to recall 0.80 with a constant threshold: a rising one stops its long searches before
    they reach what the graph allows."""
    from hnsw_engine_b200.learned_stop import FEATURE_NAMES
    from hnsw_engine_b200.train_stop import SHIPPED

    root = SHIPPED / "t1m"
    meta = json.loads((root / "meta.json").read_text())
    log = json.loads((root / "train_log.json").read_text())
    assert tuple(meta["features"]) == FEATURE_NAMES
    assert (meta["slope"], meta["ef_cap"]) == (0.0, 512)
    assert log["target"] == 0.8 and log["validation_recall"] >= 0.8
    params = np.load(root / "params.npy")
    assert params.dtype == np.float32 and np.isfinite(params).all()
