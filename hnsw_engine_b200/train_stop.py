"""Train the early-termination network for a workload graph.

    python -m hnsw_engine_b200.train_stop --workload mix1m

1. 200,000 training queries from the workload's generator (seed 2 for the mixture, 5 for the
   Student-t data) are searched by the plain GPU kernel at the cap efSearch (192) with the trace on;
2. the tensor-core exact k-NN gives each query's exact k-th distance; each checkpoint is labelled
   with the recall@10 hits the search would still gain by running to the cap;
3. the network is trained with the library's CUDA forward/backward/Adam kernels;
4. the stop threshold is tuned on 10,000 validation queries (seed 9) for recall@10 >= 0.95, with
   the threshold rising by ``STOP_SLOPE`` per 64 layer-0 expansions beyond ``STOP_SLOPE_FROM``
   (long searches stop more readily; the batch's makespan is set by its longest queries).

    python -m hnsw_engine_b200.train_stop --workload mix1m --retune

re-tunes the threshold of the stored network (with its stored threshold schedule) without
retraining.

The model is written to ``graphs/<workload>/stopnet/`` (git-ignored, next to the graph).
"""

from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np
import torch

from . import graphs, synthetic
from .exact_knn import exact_search
from .index import HNSWIndex
from .learned_stop import StopNetwork, collect_traces, label_traces, tune_threshold
from .validation import prepare

VALIDATION_SEED = 9
# Threshold schedule of the trained networks: measured on mix1m at cap 192 and recall 0.95, a slope
# of 3.2 from 192 expansions cut the batch time 4.35 -> 4.01 ms against a constant threshold
# (slopes 0.8 to 6.4 from 192 or 256 all land within 1.5% of it; from 128 misses the target).
STOP_SLOPE = 3.2
STOP_SLOPE_FROM = 192


def _validation(workload: str, index: HNSWIndex, metric: str, k: int, n_val: int):
    q_val = prepare(graphs.workload_queries(workload, nq=n_val, seed=VALIDATION_SEED), metric)
    g = index.device_graph
    _, val_d = exact_search(g.vectors, torch.from_numpy(q_val).to(g.device), k, metric)
    return q_val, val_d.cpu().numpy()


def train(workload: str, n_train: int = 200_000, ef_cap: int = 192, k: int = 10,
          target: float = 0.95, epochs: int = 4, n_val: int = 10_000, device: str = "cuda",
          slope: float = STOP_SLOPE, slope_from: int = STOP_SLOPE_FROM) -> dict:
    t0 = time.time()
    meta, arrays = graphs.open_workload(workload)
    params = {kk: v for kk, v in meta["params"].items() if kk != "engine"}
    metric = params["metric"]
    index = HNSWIndex.from_arrays(arrays, int(meta["entry_point"]), int(meta["max_level"]),
                                  device=device, **params)
    g = index.device_graph
    gen_seed = synthetic.TRAIN_SEED if graphs.WORKLOADS[workload]["gen"] == "mixture" else synthetic.T_TRAIN_SEED
    q_train = prepare(graphs.workload_queries(workload, nq=n_train, seed=gen_seed), metric)
    log = {"workload": workload, "n_train": n_train, "ef_cap": ef_cap, "k": k, "target": target}

    tr = collect_traces(g, q_train, k, ef_cap)
    t_tr = time.time()
    _, true_d = exact_search(g.vectors, torch.from_numpy(q_train).to(g.device), k, metric)
    true_kth = true_d[:, k - 1].cpu().numpy()
    X, y, _ = label_traces(tr, true_kth)
    log.update(trace_seconds=t_tr - t0, samples=int(X.shape[0]),
               mean_checkpoints=float(tr.count.mean()), label_mean=float(y.mean()))

    net = StopNetwork(g.device)
    net.ef_cap = ef_cap
    net.slope, net.slope_from = slope, slope_from
    losses = net.fit(X, y, epochs=epochs)
    log["epoch_losses"] = losses

    q_val, val_d = _validation(workload, index, metric, k, n_val)
    thr, rec = tune_threshold(g, net, q_val, val_d, k, ef_cap, target)
    log.update(threshold=thr, slope=net.slope, slope_from=net.slope_from, validation_recall=rec,
               seconds=time.time() - t0)
    out = graphs.graph_dir(workload) / "stopnet"
    net.save(out)
    (out / "train_log.json").write_text(json.dumps(log, indent=2))
    return log


# Trained networks shipped with the package (the training is deterministic; these are its output
# for the standard workloads, kept so that a fresh checkout needs no training run).
SHIPPED = Path(__file__).resolve().parent / "stopnets"


def load_or_train(workload: str, device: str = "cuda") -> StopNetwork:
    """The workload's trained network: the one next to the graph, else the shipped one, else
    trained now (about 20 s on a B200)."""
    for path in (graphs.graph_dir(workload) / "stopnet", SHIPPED / workload):
        try:
            return StopNetwork.load(path, device)
        except (FileNotFoundError, ValueError, KeyError):
            continue
    train(workload, device=device)
    return StopNetwork.load(graphs.graph_dir(workload) / "stopnet", device)


def retune(workload: str, path: Path | None = None, k: int = 10, target: float = 0.95,
           n_val: int = 10_000, device: str = "cuda") -> dict:
    """Re-tune the stored network's threshold (its schedule unchanged) on the validation queries
    and write it back (to ``path``, default the shipped copy)."""
    path = SHIPPED / workload if path is None else Path(path)
    net = StopNetwork.load(path, device)
    meta, arrays = graphs.open_workload(workload)
    params = {kk: v for kk, v in meta["params"].items() if kk != "engine"}
    index = HNSWIndex.from_arrays(arrays, int(meta["entry_point"]), int(meta["max_level"]),
                                  device=device, **params)
    q_val, val_d = _validation(workload, index, params["metric"], k, n_val)
    thr, rec = tune_threshold(index.device_graph, net, q_val, val_d, k, net.ef_cap, target)
    net.save(path)
    return {"workload": workload, "threshold": thr, "slope": net.slope,
            "slope_from": net.slope_from, "validation_recall": rec}


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--workload", default="mix1m")
    p.add_argument("--n-train", type=int, default=200_000)
    p.add_argument("--ef-cap", type=int, default=192)
    p.add_argument("--epochs", type=int, default=4)
    p.add_argument("--slope", type=float, default=STOP_SLOPE,
                   help="threshold rise per 64 layer-0 expansions beyond --slope-from (0: constant)")
    p.add_argument("--slope-from", type=int, default=STOP_SLOPE_FROM)
    p.add_argument("--target", type=float, default=0.95,
                   help="recall@10 target of the threshold (a graph that cannot reach 0.95 at "
                        "the cap efSearch is tuned to what it can reach)")
    p.add_argument("--retune", action="store_true",
                   help="only re-tune the shipped network's threshold for the current schedule")
    args = p.parse_args()
    if args.retune:
        print(json.dumps(retune(args.workload)), flush=True)
        return
    print(json.dumps(train(args.workload, args.n_train, args.ef_cap, target=args.target,
                           epochs=args.epochs, slope=args.slope, slope_from=args.slope_from)),
          flush=True)


if __name__ == "__main__":
    main()
