"""The runtime autotuner: its choice is a function of the measured timings alone (CPU), and every
kernel configuration it chooses among returns the same ids, distances and counters (GPU)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import case_arrays, load_golden


def test_pick_config_keeps_the_default_unless_clearly_faster() -> None:
    from hnsw_engine_b200.engine import pick_config

    assert pick_config([3.30, 3.40, 3.60, 5.00]) == 0
    assert pick_config([3.30, 3.26, 3.60, 5.00]) == 0  # 1.2% faster: within the margin
    assert pick_config([3.30, 3.10, 3.60, 5.00]) == 1
    assert pick_config([3.30, 3.10, 3.00, 5.00]) == 2
    assert pick_config([3.30, 3.00, 3.00, 5.00]) == 1  # ties go to the lower index
    assert pick_config([]) == 0
    times = [3.3, 3.1, 3.2, 4.0]
    assert pick_config(times) == pick_config(list(times))  # same timings, same choice


def test_tune_key_buckets_the_ef_cap() -> None:
    from hnsw_engine_b200.engine import tune_key

    assert tune_key(2, False, False, 192, False, False) == tune_key(2, False, False, 256, False, False)
    assert tune_key(2, False, False, 192, False, False) != tune_key(2, False, False, 257, False, False)
    assert tune_key(2, False, False, 64, True, False) != tune_key(2, False, False, 64, False, False)
    assert tune_key(2, False, False, 1, False, False)[3] == 1


@pytest.mark.gpu
@pytest.mark.parametrize("filtered", [False, True])
def test_every_kernel_configuration_gives_identical_results(filtered: bool) -> None:
    from hnsw_engine_b200 import HNSWIndex, _lib

    case = load_golden("search_mix10k")
    arrays, ep, ml = case_arrays(case, "mix10k")
    g = HNSWIndex.from_arrays(arrays, ep, ml, dim=128, metric="l2", M=16).device_graph
    lib = _lib.load()
    n_cfg = int(lib.hnsw_b200_kernel_configs(_lib.DIST_BYTES))
    assert n_cfg == 4 and int(lib.hnsw_b200_kernel_configs(_lib.DIST_F64)) == 1
    assert all(lib.hnsw_b200_kernel_config_name(_lib.DIST_BYTES, c) for c in range(n_cfg))
    mask = np.random.default_rng(5).random(10_000) < 0.3 if filtered else None
    q = case["queries"]
    want = [t.cpu().numpy() for t in g.search(q, 10, 96, allowed=mask, dist_mode=2, kernel_config=0)]
    for cfg in range(1, n_cfg):
        got = [t.cpu().numpy() for t in g.search(q, 10, 96, allowed=mask, dist_mode=2, kernel_config=cfg)]
        for a, b in zip(want, got, strict=True):
            np.testing.assert_array_equal(a, b, err_msg=f"config {cfg}")
    if not filtered:
        np.testing.assert_array_equal(want[0], g.search(q, 10, 96, dist_mode=0)[0].cpu().numpy())
    with pytest.raises(_lib.HnswB200Error, match="kernel_config"):
        g.search(q, 10, 96, dist_mode=2, kernel_config=n_cfg)
    with pytest.raises(_lib.HnswB200Error, match="kernel_config"):
        g.search(q, 10, 96, dist_mode=0, kernel_config=1)


@pytest.mark.gpu
def test_autotuner_tunes_large_batches_once_and_keeps_its_choice() -> None:
    import torch

    from hnsw_engine_b200 import HNSWIndex, graphs
    from hnsw_engine_b200.engine import pick_config, tune_key
    from hnsw_engine_b200.schedule import MIN_QUERIES
    from hnsw_engine_b200.validation import prepare

    if not graphs.available("mix100k"):
        pytest.skip("graph mix100k not built")
    meta, arrays = graphs.open_workload("mix100k")
    params = {k: v for k, v in meta["params"].items() if k != "engine"}
    g = HNSWIndex.from_arrays(arrays, int(meta["entry_point"]), int(meta["max_level"]),
                              **params).device_graph
    q = torch.from_numpy(prepare(graphs.workload_queries("mix100k", nq=MIN_QUERIES), "l2")).cuda()
    g.autotune = False
    want = [t.cpu().numpy() for t in g.search(q, 10, 64)]
    assert not g.tuned
    g.autotune = True
    got = [t.cpu().numpy() for t in g.search(q, 10, 64)]
    key = tune_key(2, False, False, 64, False, False)
    assert key in g.tuned and len(g.tune_log[key]) == 4
    assert g.tuned[key] == pick_config(g.tune_log[key])
    for a, b in zip(want, got, strict=True):
        np.testing.assert_array_equal(a, b)
    g.search(q, 10, 64)  # tuned once: the next batch of the same kind only searches
    assert list(g.tuned) == [key]
    small = g.search(q[:100], 10, 200)  # below MIN_QUERIES: never tuned, default configuration
    assert small[0].shape == (100, 10) and len(g.tuned) == 1
