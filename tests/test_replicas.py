"""Multi-GPU host logic (one process per GPU, graph replicas) on CPU: gloo, world size 2."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from hnsw_engine_b200.replicas import job_throughput, query_slice, rank_env


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out: dict) -> None:
    import datetime

    import torch.distributed as dist

    from hnsw_engine_b200.replicas import gather_results, max_over_ranks

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        r, w, local = rank_env()
        # a rank's device time; the job's time is the slowest rank's
        slowest = max_over_ranks(dist, 10.0 + 5.0 * r, "cpu")
        # one batch split across ranks: each searches its slice, results come back in query order
        nq, k = 11, 3
        sl = query_slice(nq, r, w)
        qids = np.arange(nq)[sl]
        ids = np.repeat(qids[:, None] * 100, k, axis=1) + np.arange(k)
        dists = ids.astype(np.float64) / 7.0
        all_ids, all_d = gather_results(dist, ids, dists)
        out[rank] = (r, w, local, slowest, all_ids, all_d)
    finally:
        dist.destroy_process_group()


def test_two_ranks_agree_on_time_and_gather_results_in_query_order() -> None:
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True,
                           start_method="spawn")
        res = dict(out)
    assert sorted(res) == [0, 1]
    want_ids = np.repeat(np.arange(11)[:, None] * 100, 3, axis=1) + np.arange(3)
    for rank, (r, w, local, slowest, ids, d) in res.items():
        assert (r, w, local) == (rank, 2, rank)
        assert slowest == 15.0
        np.testing.assert_array_equal(ids, want_ids)
        np.testing.assert_array_equal(d, want_ids / 7.0)


@pytest.mark.parametrize("nq,world", [(0, 1), (5, 1), (11, 2), (10, 3), (3, 8), (10_000, 8)])
def test_query_slices_tile_the_batch(nq: int, world: int) -> None:
    sizes = []
    covered = []
    for r in range(world):
        sl = query_slice(nq, r, world)
        covered.extend(range(nq)[sl])
        sizes.append(sl.stop - sl.start)
    assert covered == list(range(nq))
    assert max(sizes) - min(sizes) <= 1


def test_job_throughput_counts_every_rank() -> None:
    # 2 ranks x 10,000 queries x 4 steps in 80 ms (slowest rank)
    assert job_throughput(2, 10_000, 4, 80.0) == pytest.approx(1_000_000.0)
    with pytest.raises(ValueError):
        job_throughput(1, 1, 1, 0.0)


def test_rank_env_rejects_inconsistent_launch(monkeypatch) -> None:
    monkeypatch.setenv("RANK", "2")
    monkeypatch.setenv("WORLD_SIZE", "2")
    with pytest.raises(ValueError):
        rank_env()
