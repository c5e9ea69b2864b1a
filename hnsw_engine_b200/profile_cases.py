"""Small, fixed cases of the two hot kernels for profilers (the commands in ``profiles/``).

    python -m hnsw_engine_b200.profile_cases search --nq 2000 --ef 192 [--stop] [--workload t1m]
    python -m hnsw_engine_b200.profile_cases exact --nq 1024 [--image] [--calls 2]

``search``: the 1M x 128 mixture graph (``--workload t1m``: the 1M x 100 Student-t cosine graph,
float64 rows) with ``nq`` of its benchmark queries, three synchronous searches at ``ef`` (the
learned stop with the shipped network when ``--stop``), autotuning off, so the search kernel's
launches are the 3 searches in order (with the start order's launches before each when
``nq >= 4096``). ``exact``: the tensor-core exact k-NN (k = 100) of ``nq`` mixture queries over the
1M x 128 mixture rows (``--image``: 60K x 784 image-like rows), ``calls`` times;
each call launches the filter kernel twice (the prefix pass, then every row).
"""

from __future__ import annotations

import argparse

import numpy as np
import torch

from . import graphs, synthetic
from .exact_knn import exact_search
from .index import HNSWIndex
from .validation import prepare


def search_case(nq: int, ef: int, stop: bool, workload: str = "mix1m") -> None:
    from .train_stop import load_or_train

    meta, arrays = graphs.open_workload(workload)
    params = {k: v for k, v in meta["params"].items() if k != "engine"}
    g = HNSWIndex.from_arrays(arrays, int(meta["entry_point"]), int(meta["max_level"]),
                              **params).device_graph
    g.autotune = False
    q = torch.from_numpy(prepare(graphs.workload_queries(workload, nq=nq), meta["params"]["metric"])).cuda()
    kw = {}
    if stop:
        net = load_or_train(workload)
        kw["stop"] = (net.packed(), net.threshold, net.slope, net.slope_from)
    for _ in range(3):
        ids, d, c = g.search(q, 10, ef, **kw)
    torch.cuda.synchronize()
    print("search", nq, ef, "stop" if stop else "plain", float(c[:, 0].float().mean()),
          float(c[:, 1].float().mean()), flush=True)


def exact_case(nq: int, image: bool, calls: int) -> None:
    if image:
        x = torch.from_numpy(synthetic.image_like(60000, seed=synthetic.IMAGE_DATA_SEED)
                             .astype(np.uint8)).cuda()
        q = torch.from_numpy(synthetic.image_like(nq, seed=synthetic.IMAGE_QUERY_SEED)
                             .astype(np.uint8)).cuda()
    else:
        x = torch.from_numpy(synthetic.mixture(1_000_000, seed=synthetic.DATA_SEED)).cuda()
        q = torch.from_numpy(synthetic.mixture(nq, seed=synthetic.QUERY_SEED)).cuda()
    for _ in range(calls):
        _, _, st = exact_search(x, q, 100, return_stats=True)
    torch.cuda.synchronize()
    print("exact", nq, "image" if image else "mixture", st, flush=True)


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("case", choices=("search", "exact"))
    p.add_argument("--nq", type=int, default=2000)
    p.add_argument("--ef", type=int, default=192)
    p.add_argument("--stop", action="store_true")
    p.add_argument("--image", action="store_true")
    p.add_argument("--calls", type=int, default=1)
    p.add_argument("--workload", default="mix1m", help="search: the graph (mix1m, or t1m for float64 rows)")
    a = p.parse_args()
    if a.case == "search":
        search_case(a.nq, a.ef, a.stop, a.workload)
    else:
        exact_case(a.nq, a.image, a.calls)


if __name__ == "__main__":
    main()
