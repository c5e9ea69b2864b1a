"""Measurements of every workload configuration, one JSON line each (``python -m hnsw_engine_b200.suite``).

The headline metric is ``bench.py``'s; this suite measures the other configurations of the same
engine on one GPU with device-resident inputs (CUDA events, median of repeated launches) and the
recall measured against the tensor-core exact k-NN:

* ``sweep``: plain search at a list of efSearch values (10K and 1M mixture, 1M Student-t);
* ``modes``: the same search with byte rows, exact float32 rows and float64 rows (1M mixture);
* ``per_query_ef``: efSearch uniform in 32..512 per query;
* ``quantized``: int8 codes with the fused exact re-rank of the beam (rerank = ef);
* ``filtered``: Bernoulli and prefix masks, recall against the exact k-NN of the allowed rows;
  below 5% selectivity also the planner (``batch_search(..., exact_below=0.05)``);
* ``exact``: the tensor-core exact k-NN (k = 100) on the 1M mixture and on 60K x 784 image-like data.
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import graphs, synthetic
from .exact_knn import exact_search
from .index import HNSWIndex
from .learned_stop import recall_of
from .quantization import QuantizedIndex
from .validation import prepare


def _timed(fn, reps: int = 3) -> tuple[float, object]:
    out = fn()
    torch.cuda.synchronize()
    ms = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        out = fn()
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    return float(np.median(ms)), out


def _emit(**kw) -> None:
    print(json.dumps(kw), flush=True)


def _open(name: str):
    meta, arrays = graphs.open_workload(name)
    params = {k: v for k, v in meta["params"].items() if k != "engine"}
    index = HNSWIndex.from_arrays(arrays, int(meta["entry_point"]), int(meta["max_level"]), **params)
    return index, arrays, params["metric"]


def sweep(name: str, efs, k: int = 10, modes=(None,)) -> None:
    index, arrays, metric = _open(name)
    g = index.device_graph
    q = prepare(graphs.workload_queries(name), metric)
    qd = torch.from_numpy(q).cuda()
    _, gt = exact_search(g.vectors, qd, k, metric)
    gt = gt.cpu().numpy()
    for mode in modes:
        for ef in efs:
            ms, (ids, d, c) = _timed(lambda: g.search(qd, k, ef, dist_mode=mode))
            _emit(config="sweep", workload=name, mode=mode if mode is not None else g.choose_mode(q, False),
                  ef=ef, qps=q.shape[0] / ms * 1e3, ms=ms,
                  recall=recall_of(ids.cpu().numpy(), d.cpu().numpy(), gt, k),
                  dist_per_query=float(c[:, 0].float().mean()), hops_per_query=float(c[:, 1].float().mean()))
    if name.endswith("1m") or name.endswith("100k"):
        pq = torch.from_numpy(synthetic.per_query_ef(q.shape[0], seed=11, low=32, high=512)).cuda()
        ms, (ids, d, c) = _timed(lambda: g.search(qd, k, pq))
        _emit(config="per_query_ef", workload=name, ef="uniform 32..512", qps=q.shape[0] / ms * 1e3, ms=ms,
              recall=recall_of(ids.cpu().numpy(), d.cpu().numpy(), gt, k),
              dist_per_query=float(c[:, 0].float().mean()))


def quantized(name: str, efs, k: int = 10) -> None:
    index, arrays, metric = _open(name)
    g = index.device_graph
    qi = QuantizedIndex(index)
    raw = graphs.workload_queries(name)
    q = prepare(raw, metric)
    qd = torch.from_numpy(q).cuda()
    _, gt = exact_search(g.vectors, qd, k, metric)
    gt = gt.cpu().numpy()
    code_q = torch.from_numpy(qi.quantizer.transform_queries(q, metric)).cuda()
    for ef in efs:
        for rerank in (0, ef):
            fetch = max(rerank, k)

            def run():
                return g.search(code_q, k if rerank else fetch, ef, use_codes=True, k_search=fetch,
                                rerank_queries=qd if rerank else None)

            ms, (ids, d, c) = _timed(run)
            dd = d.cpu().numpy()
            if rerank == 0:
                dd = qi.quantizer.to_distance(dd, q, metric)
            _emit(config="quantized", workload=name, ef=ef, rerank=rerank, step=qi.quantizer.step,
                  mode=g.choose_mode(code_q.cpu().numpy(), True), qps=q.shape[0] / ms * 1e3, ms=ms,
                  recall=recall_of(ids.cpu().numpy()[:, :k], dd[:, :k], gt, k))


def filtered(name: str, ef: int = 64, k: int = 10) -> None:
    index, arrays, metric = _open(name)
    g = index.device_graph
    q = prepare(graphs.workload_queries(name), metric)
    qd = torch.from_numpy(q).cuda()
    n = arrays["vectors"].shape[0]
    for kind in ("bernoulli", "prefix"):
        for p in (0.5, 0.1, 0.01):
            mask = synthetic.bernoulli_mask(n, p) if kind == "bernoulli" else synthetic.prefix_mask(n, p)
            sub = np.flatnonzero(mask)
            _, gtd = exact_search(g.vectors[torch.from_numpy(sub).cuda()], qd, k, metric)
            gtd = gtd.cpu().numpy()
            ms, (ids, d, c) = _timed(lambda: g.search(qd, k, ef, allowed=mask), reps=1)
            _emit(config="filtered", workload=name, mask=kind, p=p, ef=ef, qps=q.shape[0] / ms * 1e3,
                  ms=ms, recall=recall_of(ids.cpu().numpy(), d.cpu().numpy(), gtd, k),
                  dist_per_query=float(c[:, 0].float().mean()))
            if p < 0.05:  # the selectivity planner: exact k-NN over the allowed rows
                ms, (ids, d) = _timed(lambda: index.batch_search(qd, k, ef, filter=mask, exact_below=0.05))
                _emit(config="filtered_planner", workload=name, mask=kind, p=p, qps=q.shape[0] / ms * 1e3,
                      ms=ms, recall=recall_of(ids.cpu().numpy(), d.cpu().numpy(), gtd, k))


def exact(k: int = 100) -> None:
    x = graphs.stored_vectors("mix1m")
    q = graphs.workload_queries("mix1m")
    xd, qd = torch.from_numpy(x).cuda(), torch.from_numpy(q).cuda()
    for label, data, queries in (("mixture 1M x 128", xd, qd),):
        exact_search(data, queries, k)  # warm-up at full size: scratch allocated outside the timing
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ids, d, st = exact_search(data, queries, k, return_stats=True)
        torch.cuda.synchronize()
        s = time.perf_counter() - t0
        flops = 2.0 * queries.shape[0] * data.shape[0] * data.shape[1]
        _emit(config="exact", data=label, nq=queries.shape[0], k=k, seconds=s, qps=queries.shape[0] / s,
              gemm_tflops=flops / s / 1e12, filter_max_error=st.filter_max_error,
              filter_error_bound=st.filter_error_bound,
              candidates_per_query=st.candidates / queries.shape[0])
    img = synthetic.image_like(60000, seed=synthetic.IMAGE_DATA_SEED)
    iq = synthetic.image_like(10000, seed=synthetic.IMAGE_QUERY_SEED)
    xi, qi = torch.from_numpy(img.astype(np.uint8)).cuda(), torch.from_numpy(iq.astype(np.uint8)).cuda()
    exact_search(xi, qi, k)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ids, d, st = exact_search(xi, qi, k, return_stats=True)
    torch.cuda.synchronize()
    s = time.perf_counter() - t0
    flops = 2.0 * 10000 * 60000 * 784
    _emit(config="exact", data="image-like 60K x 784 uint8", nq=10000, k=k, seconds=s, qps=10000 / s,
          gemm_tflops=flops / s / 1e12, filter_max_error=st.filter_max_error,
              filter_error_bound=st.filter_error_bound,
          candidates_per_query=st.candidates / 10000)


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--only", nargs="*", default=None,
                   help="subset of: small mix1m modes quantized filtered t1m exact")
    args = p.parse_args()
    want = set(args.only or ["small", "mix1m", "modes", "quantized", "filtered", "t1m", "exact"])
    if "small" in want and graphs.available("mix10k"):
        sweep("mix10k", (16, 32, 64, 128, 256))
    if "mix1m" in want and graphs.available("mix1m"):
        sweep("mix1m", (32, 64, 128, 192, 256, 512))
    if "modes" in want and graphs.available("mix1m"):
        sweep("mix1m", (192,), modes=(2, 1, 0))
    if "quantized" in want and graphs.available("mix1m"):
        quantized("mix1m", (64, 192))
    if "filtered" in want and graphs.available("mix1m"):
        filtered("mix1m")
    if "t1m" in want and graphs.available("t1m"):
        sweep("t1m", (64, 128, 256, 512))
        quantized("t1m", (64, 128, 256, 512))
    if "exact" in want:
        exact()


if __name__ == "__main__":
    main()
