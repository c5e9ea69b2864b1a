#!/usr/bin/env python
"""Benchmark of the batched HNSW search on one B200 (or N replicas under torchrun).

Workload: the 1M x 128 integer Gaussian-mixture graph (reference host build, M=16,
efConstruction=200, level seed 42; ``graphs/build_graphs.py``), 10,000 queries from the same
mixture (seed 1), k=10. A step is one batched search of all queries. Metric: QPS at recall@10 >=
0.95 (tie-aware recall against the exact oracle): the operating point is the smallest fixed efSearch
whose recall reaches 0.95 (plain fixed-ef), and, when a trained early-termination network is
available, the learned-stop search at the same recall target.

``value``: queries/s with queries and graph resident in HBM (device-timed with CUDA events on the
launching stream, max over ranks). ``e2e``: the same metric through the public API
(``HNSWIndex.batch_search`` with numpy queries: validation, host->device copy, search,
device->host copy of ids and distances). ``roofline``: algorithmic bytes per launch (from the
kernel's own per-query work counters) over the launch duration, against the measured HBM copy
bandwidth. ``cpu_baseline``: the CPU restatement of the reference search (oracle) on the host's
cores over a bounded sample of the same queries.

``--impl reference`` times the reference's CPU search path (the C restatement of the reference's
compiled search, on all host threads) on the same workload and prints the same JSON line.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "QPS at recall@10>=0.95, 1M x 128, 1 B200: learned-stop vs plain fixed-ef"
UNIT = "queries/s"
RECALL_TARGET = 0.95
EF_LADDER = (10, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256, 320, 384, 512)
L2_BYTES = 126 * 1024 * 1024


def parse() -> argparse.Namespace:
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("b200", "reference"), default="b200")
    p.add_argument("--workload", default="mix1m")
    p.add_argument("--nq", type=int, default=None)
    p.add_argument("--k", type=int, default=10)
    p.add_argument("--target", type=float, default=RECALL_TARGET,
                   help="recall@k target of both arms (graphs that cannot reach 0.95 at efSearch "
                        "<= 512, such as the Student-t cosine graph, are compared at what they reach)")
    p.add_argument("--cpu-sample-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-configs", action="store_true",
                   help="skip the other configurations (quantized, filtered, planner, exact k-NN)")
    return p.parse_args()


# ----------------------------------------------------------------------------------- helpers
from hnsw_engine_b200.replicas import job_throughput, max_over_ranks  # noqa: E402
from hnsw_engine_b200.replicas import rank_env as dist_env  # noqa: E402


def peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.is_file():
        d = json.loads(path.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples taken while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int) -> None:
        self.gpu = gpu_index
        self.samples: list[list[str]] = []
        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._run, daemon=True)

    def _run(self) -> None:
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                     "--format=csv,noheader,nounits"],
                    capture_output=True, text=True, timeout=5,
                ).stdout.strip()
                if out:
                    self.samples.append([s.strip() for s in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self) -> ClockSampler:
        self._thread.start()
        return self

    def __exit__(self, *exc) -> None:
        self._stop.set()
        self._thread.join(timeout=10)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 5 + i and s[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def algorithmic_bytes(counters: np.ndarray, arrays: dict, dim: int, k: int, row_bytes: int) -> float:
    """Per-launch algorithmic bytes: rows scored, link rows read, queries and results.

    distances x row bytes + hops x (count word + mean used link slots x 4) + nq x (query + k x 16).
    """
    dist = float(counters[:, 0].sum())
    hops = float(counters[:, 1].sum())
    mean_links = float(np.asarray(arrays["count0"]).mean())
    nq = counters.shape[0]
    return dist * row_bytes + hops * (4.0 + 4.0 * mean_links) + nq * (dim * 4.0 + k * 16.0)


def measured_traffic(workload: str) -> int | None:
    """DRAM bytes (read + write) of one learned-stop search launch of this workload, as an ncu
    capture of this same command recorded them (``profiles/search_kernel_bytes_<workload>.md``,
    line ``traffic_bytes_per_launch: N``); None when no capture of the workload is committed."""
    path = ROOT / "profiles" / f"search_kernel_bytes_{workload}.md"
    if not path.is_file():
        return None
    for line in path.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            return int(line.split(":", 1)[1])
    return None


def ground_truth(vectors_dev, queries: np.ndarray, k: int, metric: str):
    """Exact top-k (ids, float64 distances) from the tensor-core exact k-NN (untimed)."""
    import torch

    from hnsw_engine_b200.exact_knn import exact_search

    ids, dists = exact_search(vectors_dev, torch.from_numpy(queries).to(vectors_dev.device), k, metric)
    return ids.cpu().numpy(), dists.cpu().numpy()


def recall_of(ids: np.ndarray, dists: np.ndarray, gt_ids: np.ndarray, gt_d: np.ndarray, k: int) -> float:
    from hnsw_engine_b200.metrics import recall_at_k

    return recall_at_k(ids, dists, gt_ids, gt_d, k)["recall"]


# -------------------------------------------------------------------------------- CPU baselines
def cpu_sample(arrays, ep, ml, queries, k, ef, metric, seconds: float, threads: int) -> dict:
    """Time the oracle (C restatement of the reference search) on a bounded sample of queries."""
    from oracle import cpu

    cpu.build()
    probe = min(len(queries), max(64, threads * 8))
    t0 = time.perf_counter()
    cpu.search_batch(arrays, ep, ml, queries[:probe], k, ef, metric, threads=threads)
    per_q = (time.perf_counter() - t0) / probe
    # about `seconds` of work: the workload's queries, cycled when one pass takes less
    n = int(min(16 * len(queries), max(probe, seconds / max(per_q, 1e-9))))
    sample = queries[np.arange(n) % len(queries)]
    if not np.isscalar(ef):
        ef = np.asarray(ef)[np.arange(n) % len(queries)]
    t0 = time.perf_counter()
    cpu.search_batch(arrays, ep, ml, sample, k, ef, metric, threads=threads)
    el = time.perf_counter() - t0
    return {"value": n / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} queries ({len(queries)} workload queries"
                      f"{', cycled' if n > len(queries) else ''}) at "
                      f"ef={ef if np.isscalar(ef) else 'per-query'}, "
                      f"C restatement of the reference search (oracle/hnsw_oracle.c), "
                      f"{threads} threads, {el:.1f} s"}


def run_reference(args: argparse.Namespace) -> None:
    """The reference arm: the reference search path on the host cores, same workload and metric."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from hnsw_engine_b200 import graphs
    from hnsw_engine_b200.validation import prepare
    from oracle import cpu

    meta, arrays = graphs.open_workload(args.workload)
    ep, ml = int(meta["entry_point"]), int(meta["max_level"])
    metric = meta["params"]["metric"]
    queries = prepare(graphs.workload_queries(args.workload, nq=args.nq), metric)
    threads = cpu.default_threads()
    ef = int(os.environ.get("HNSW_BENCH_EF", "0")) or None
    if ef is None:
        # The GPU arm's plain operating point: measured live by that arm on the same box when it
        # has run, else the committed measurement of this workload (the search results, hence the
        # recall of each efSearch, are the reference's own).
        live = ROOT / "graphs" / args.workload / "operating_point.json"
        committed = json.loads((ROOT / "graphs" / "operating_points.json").read_text())
        ef = (json.loads(live.read_text())["ef"] if live.is_file()
              else int(committed[args.workload]["ef"]))
    per_step_s = max(2.0, min(20.0, 120.0 / max(1, args.steps + args.warmup)))
    values = []
    for step in range(args.warmup + args.steps):
        res = cpu_sample(arrays, ep, ml, queries, args.k, ef, metric, per_step_s, threads)
        if step >= args.warmup:
            values.append(res["value"])
    value = statistics.median(values)
    res["value"] = value
    res["cpu_model"] = cpu_model()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * len(queries) / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": f"{args.workload}: {arrays['vectors'].shape[0]} x {arrays['vectors'].shape[1]} "
                               f"{metric}, nq={len(queries)}, k={args.k}, ef={ef} (plain fixed-ef operating point)",
                   "parallelism": "host threads"},
        "cpu_baseline": res,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------ GPU arm
def timed_steps(step, steps: int, stream) -> list[float]:
    """Per-step device milliseconds of ``steps`` calls of ``step`` (CUDA events on ``stream``)."""
    import torch

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for i in range(steps):
        starts[i].record(stream)
        step()
        ends[i].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in zip(starts, ends, strict=True)]


def other_configs(index, workload: str, queries: np.ndarray, q_dev, gt_ids, gt_d, k: int, ef: int,
                  stream) -> dict:
    """The workload's other configurations on the same graph and queries, device-resident and timed
    with CUDA events (median of 3 launches; 1 for the slowest): int8 scalar-quantizer codes with the
    fused exact re-rank of the beam at the operating efSearch; Bernoulli and prefix filters at
    p = 0.5 / 0.1 / 0.01 at the same efSearch (recall against the exact neighbours among the
    allowed rows) and the selectivity planner at p = 0.01; the tensor-core exact k-NN at k = 100."""
    import torch

    from hnsw_engine_b200 import synthetic
    from hnsw_engine_b200.engine import pack_mask, to_device
    from hnsw_engine_b200.exact_knn import exact_search
    from hnsw_engine_b200.quantization import QuantizedIndex

    g = index.device_graph
    dev = q_dev.device
    nq = queries.shape[0]
    metric = index.metric
    out: dict = {}

    def med(fn, reps: int = 3) -> float:
        fn()
        torch.cuda.synchronize()
        return float(np.median(timed_steps(fn, reps, stream)))

    qi = QuantizedIndex(index)
    code_q = torch.from_numpy(qi.quantizer.transform_queries(queries, metric)).to(dev)
    held: dict = {}

    def run_codes():
        held["r"] = qi.batch_search_device(code_q, q_dev, k, ef, ef)

    ms = med(run_codes)
    ids, d = held["r"]
    out["int8_codes_fused_rerank"] = {
        "ef": ef, "rerank": ef, "step": float(qi.quantizer.step), "ms": ms, "qps": nq / ms * 1e3,
        "recall_at_10": recall_of(ids.cpu().numpy(), d.cpu().numpy(), gt_ids, gt_d, k)}

    n = g.n
    for kind in ("bernoulli", "prefix"):
        for p in (0.5, 0.1, 0.01):
            mask = synthetic.bernoulli_mask(n, p) if kind == "bernoulli" else synthetic.prefix_mask(n, p)
            sub = torch.from_numpy(np.flatnonzero(mask)).to(dev)
            t_ids, t_d = exact_search(g.vectors[sub].contiguous(), q_dev, k, metric)
            t_ids, t_d = sub[t_ids].cpu().numpy(), t_d.cpu().numpy()
            bitmap = to_device(pack_mask(g.internal_mask(mask)).view(np.int32), torch.int32, dev)
            frac = float(mask.mean())

            def run_filtered():
                held["r"] = g.search(q_dev, k, ef, allowed=bitmap, allowed_fraction=frac,
                                     counters=False)

            ms = med(run_filtered, reps=1 if p < 0.05 else 3)
            ids, d, _ = held["r"]
            entry = {"ef": ef, "ms": ms, "qps": nq / ms * 1e3,
                     "recall_at_10": recall_of(ids.cpu().numpy(), d.cpu().numpy(), t_ids, t_d, k)}
            if p < 0.05:
                def run_planner():
                    held["r"] = index.batch_search(q_dev, k=k, ef=ef, filter=mask, exact_below=0.05)

                ms = med(run_planner)
                ids, d = held["r"]
                entry["planner_exact_below_0.05"] = {
                    "ms": ms, "qps": nq / ms * 1e3,
                    "recall_at_10": recall_of(ids.cpu().numpy(), d.cpu().numpy(), t_ids, t_d, k)}
            out[f"filtered_{kind}_p{p}"] = entry

    kx = 100
    exact_search(g.vectors, q_dev, kx)  # scratch allocated outside the timing
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, _, st = exact_search(g.vectors, q_dev, kx, metric, return_stats=True)
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    flops = 2.0 * nq * n * g.dim
    out["exact_knn_k100"] = {
        "seconds": sec, "qps": nq / sec, "tflops": flops / sec / 1e12,
        "filter_max_error_measured": st.filter_max_error,
        "filter_error_bound": st.filter_error_bound,
        "candidates_per_query": st.candidates / nq, "launches": st.launches}
    return out


def autotune_report(g) -> dict:
    """The autotuner's choices in this run: per kind of batch (distance mode, codes, filter, efSearch
    cap bucket, learned stop, rerank), the chosen kernel configuration and every configuration's
    median milliseconds on the batch that tuned it."""
    out = {}
    for key, cfg in g.tuned.items():
        mode, codes, filt, bucket, stop, rerank = key
        name = f"mode{mode}{'-codes' if codes else ''}{'-filtered' if filt else ''}-ef<={bucket}" \
               f"{'-stop' if stop else ''}{'-rerank' if rerank else ''}"
        out[name] = {"choice": g.lib.hnsw_b200_kernel_config_name(mode, cfg).decode(),
                     "ms": [round(x, 4) for x in g.tune_log.get(key, [])]}
    return out


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def main() -> None:
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    from hnsw_engine_b200 import HNSWIndex, graphs, synthetic
    from hnsw_engine_b200.learned_stop import audited_search, stopped_search, tune_threshold
    from hnsw_engine_b200.train_stop import load_or_train
    from hnsw_engine_b200.validation import prepare

    meta, arrays = graphs.open_workload(args.workload)
    ep, ml = int(meta["entry_point"]), int(meta["max_level"])
    params = {k: v for k, v in meta["params"].items() if k != "engine"}
    metric = params["metric"]
    index = HNSWIndex.from_arrays(arrays, ep, ml, device=dev, **params)
    g = index.device_graph
    raw_q = graphs.workload_queries(args.workload, nq=args.nq)
    queries = prepare(raw_q, metric)
    nq, k = queries.shape[0], args.k
    dim = queries.shape[1]
    q_dev = torch.from_numpy(queries).to(dev)
    stream = torch.cuda.current_stream(dev)
    mode = g.choose_mode(queries, False)
    row_bytes = dim * (1 if mode == 2 else 4)

    # Held-out protocol: every operating point is fixed on the validation queries (seed 9), then
    # both arms are timed and scored on the benchmark queries (seed 1), which nothing was tuned on.
    from hnsw_engine_b200.train_stop import VALIDATION_SEED

    val_q = prepare(graphs.workload_queries(args.workload, nq=nq, seed=VALIDATION_SEED), metric)
    val_dev = torch.from_numpy(val_q).to(dev)
    gt_ids, gt_d = ground_truth(g.vectors, queries, k, metric)
    vgt_ids, vgt_d = ground_truth(g.vectors, val_q, k, metric)

    def val_recall(ef: int) -> float:
        ids, dists, _ = g.search(val_dev, k, ef, dist_mode=mode)
        return recall_of(ids.cpu().numpy(), dists.cpu().numpy(), vgt_ids, vgt_d, k)

    # Plain fixed-ef operating point: the smallest efSearch on the ladder reaching the target on
    # the validation queries, then the smallest integer efSearch between the rung below and it.
    sweep = {}
    ef_op = EF_LADDER[-1]
    for ef in EF_LADDER:
        sweep[ef] = val_recall(ef)
        if sweep[ef] >= args.target:
            ef_op = ef
            break
    i_op = EF_LADDER.index(ef_op)
    lo, hi = (EF_LADDER[i_op - 1] if i_op else k - 1), ef_op
    ef_fine = ef_op
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if val_recall(mid) >= args.target:
            hi = ef_fine = mid
        else:
            lo = mid
    if rank == 0:
        try:
            (ROOT / "graphs" / args.workload / "operating_point.json").write_text(
                json.dumps({"ef": ef_op, "validation_recall": sweep[ef_op]}))
        except OSError:
            pass

    # Learned stop: the trained network, its threshold tuned on the validation queries for the
    # recall target. The in-sample threshold (tuned on the benchmark queries themselves) is kept
    # only as a side figure.
    net = load_or_train(args.workload, device=str(dev))
    cap = net.ef_cap
    thr, val_rec_l = tune_threshold(g, net, val_dev, vgt_d, k, cap, args.target)
    thr_in, _ = tune_threshold(g, net, q_dev, gt_d, k, cap, args.target)
    net.threshold = thr
    packed = net.packed()

    ids_o = torch.empty((nq, k), dtype=torch.int64, device=dev)
    d_o = torch.empty((nq, k), dtype=torch.float64, device=dev)
    c_o = torch.empty((nq, 2), dtype=torch.int64, device=dev)
    ids_p = torch.empty_like(ids_o)
    d_p = torch.empty_like(d_o)
    c_p = torch.empty_like(c_o)
    ids_f = torch.empty_like(ids_o)
    d_f = torch.empty_like(d_o)
    c_f = torch.empty_like(c_o)
    ids_i = torch.empty_like(ids_o)
    d_i = torch.empty_like(d_o)
    c_i = torch.empty_like(c_o)

    def step_learned():
        g.search(q_dev, k, cap, out=(ids_o, d_o, c_o), dist_mode=mode,
                 stop=(packed, thr, net.slope, net.slope_from))

    def step_in_sample():
        g.search(q_dev, k, cap, out=(ids_i, d_i, c_i), dist_mode=mode,
                 stop=(packed, thr_in, net.slope, net.slope_from))

    def step_plain():
        g.search(q_dev, k, ef_op, out=(ids_p, d_p, c_p), dist_mode=mode)

    def step_fine():
        g.search(q_dev, k, ef_fine, out=(ids_f, d_f, c_f), dist_mode=mode)

    for _ in range(max(3, args.warmup)):
        step_learned()
        step_plain()
        step_fine()
        step_in_sample()
    torch.cuda.synchronize()
    launches_per_step = g.last_launches
    # Each arm's step recorded once as a CUDA graph (start order and search kernel, no host work
    # between them) and replayed: the synchronous call waits for its kernel to read the overflow
    # count, which leaves the GPU idle while the host issues the next step.
    from hnsw_engine_b200.engine import CapturedSearch

    stop_v = (packed, thr, net.slope, net.slope_from)
    cap_l = CapturedSearch(g, q_dev, k, cap, stop=stop_v)
    cap_i = CapturedSearch(g, q_dev, k, cap, stop=(packed, thr_in, net.slope, net.slope_from))
    cap_p = CapturedSearch(g, q_dev, k, ef_op)
    cap_f = CapturedSearch(g, q_dev, k, ef_fine)
    for _ in range(max(3, args.warmup)):
        for c in (cap_l, cap_i, cap_p, cap_f):
            c.replay()
    torch.cuda.synchronize()
    alg_bytes = algorithmic_bytes(c_o.cpu().numpy(), arrays, dim, k, row_bytes)
    alg_bytes_plain = algorithmic_bytes(c_p.cpu().numpy(), arrays, dim, k, row_bytes)

    # Timed regions (device-resident inputs; graph and rows exceed L2, no flush needed).
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        # NVTX range "timed_learned": lets a profiler list exactly the value's launches
        torch.cuda.nvtx.range_push("timed_learned")
        ms_learned = timed_steps(cap_l.replay, args.steps, stream)
        torch.cuda.nvtx.range_pop()
        ms_fine = timed_steps(cap_f.replay, args.steps, stream)
        ms_plain = timed_steps(cap_p.replay, args.steps, stream)
        ms_in = timed_steps(cap_i.replay, max(3, args.steps // 4), stream)
        ms_sync = timed_steps(step_learned, max(3, args.steps // 4), stream)
    # The replays' results are the synchronous calls' (overflow checked once, after the loops).
    for c, ref in ((cap_l, (ids_o, d_o, c_o)), (cap_i, (ids_i, d_i, c_i)), (cap_p, (ids_p, d_p, c_p)),
                   (cap_f, (ids_f, d_f, c_f))):
        for x, y in zip(c.results(), ref, strict=True):
            assert torch.equal(x, y), "graph replay results differ from the synchronous search"
    total_l = max_over_ranks(pg, float(sum(ms_learned)), dev)
    total_p = max_over_ranks(pg, float(sum(ms_plain)), dev)
    fine_qps = job_throughput(world, nq, args.steps, max_over_ranks(pg, float(sum(ms_fine)), dev))
    in_qps = job_throughput(world, nq, len(ms_in), max_over_ranks(pg, float(sum(ms_in)), dev))
    value = job_throughput(world, nq, args.steps, total_l)
    plain_qps = job_throughput(world, nq, args.steps, total_p)
    mean_ms = total_l / args.steps
    rec_l = recall_of(ids_o.cpu().numpy(), d_o.cpu().numpy(), gt_ids, gt_d, k)
    rec_p = recall_of(ids_p.cpu().numpy(), d_p.cpu().numpy(), gt_ids, gt_d, k)
    rec_f = recall_of(ids_f.cpu().numpy(), d_f.cpu().numpy(), gt_ids, gt_d, k)
    rec_i = recall_of(ids_i.cpu().numpy(), d_i.cpu().numpy(), gt_ids, gt_d, k)
    hops_l = float(c_o[:, 1].float().mean())
    hops_p = float(c_p[:, 1].float().mean())
    hops_f = float(c_f[:, 1].float().mean())

    # End to end through the public API with host buffers (numpy in, numpy out): each step copies
    # the float32 queries to the GPU and the ids and distances back. Mean over the steps.
    for _ in range(3):  # results held as in the timed loop, so its page-locked buffers exist
        e_ids, e_d = index.batch_search(raw_q, k=k, ef=cap, stop=net)
    torch.cuda.synchronize()
    e_steps = max(5, min(args.steps, 30))
    t0 = time.perf_counter()
    for _ in range(e_steps):
        e_ids, e_d = index.batch_search(raw_q, k=k, ef=cap, stop=net)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(pg, (time.perf_counter() - t0) * 1000.0 / e_steps, dev)
    e2e_value = job_throughput(world, nq, 1, e2e_ms)
    assert np.array_equal(e_ids, ids_o.cpu().numpy()), "e2e results differ from device results"

    # The per-batch audit (2% of each batch against the exact k-NN; plain fixed ef on a miss),
    # over ten batches of a tenth of the queries.
    audits = []
    for part_i, part in enumerate(np.array_split(np.arange(nq), 10)):
        _, _, fell, arec = audited_search(g, q_dev[torch.from_numpy(part).to(dev)], k, cap, net,
                                          ef_op, args.target, seed=part_i)
        audits.append((bool(fell), float(arec)))

    # Per-query efSearch uniform on 32..512 (the batched-at-scale configuration).
    pq = synthetic.per_query_ef(nq, seed=11, low=32, high=512)
    pq_dev = torch.from_numpy(pq).to(dev)
    g.search(q_dev, k, pq_dev, dist_mode=mode)
    pq_ms = timed_steps(lambda: g.search(q_dev, k, pq_dev, dist_mode=mode), 3, stream)
    pq_ids, pq_d, pq_c = g.search(q_dev, k, pq_dev, dist_mode=mode)
    pq_rec = recall_of(pq_ids.cpu().numpy(), pq_d.cpu().numpy(), gt_ids, gt_d, k)
    pq_bytes = algorithmic_bytes(pq_c.cpu().numpy(), arrays, dim, k, row_bytes)
    pq_mean = max_over_ranks(pg, float(np.median(pq_ms)), dev)
    more = other_configs(index, args.workload, queries, q_dev, gt_ids, gt_d, k, ef_op, stream) \
        if world == 1 and not args.no_configs else None

    pk = peaks()
    achieved = alg_bytes / (mean_ms / 1000.0) / 1e9
    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import cpu

        cpu_base = cpu_sample(arrays, ep, ml, queries, k, ef_op, metric, args.cpu_sample_seconds,
                              cpu.default_threads())
        one = cpu_sample(arrays, ep, ml, queries, k, ef_op, metric, 5.0, 1)
        cpu_base["single_thread"] = {"value": one["value"], "sample": one["sample"]}
        cpu_base["cpu_model"] = cpu_model()
        cpu_base["host_threads"] = os.cpu_count()
    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": max(3, args.warmup),
            "ms_per_step": mean_ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": {2: "u8 (exact int32 dp4a)", 1: "f32 (exact integer)", 0: "f64"}[mode],
            "data": "synthetic",
            "config": {
                "workload": f"{args.workload}: {arrays['vectors'].shape[0]} x {dim} "
                            f"{graphs.WORKLOADS[args.workload]['gen']} data, {metric}, "
                            f"M={params['M']}, efC={params['ef_construction']}, nq={nq}, k={k}",
                "method": "learned stop (value) vs plain fixed-ef, equal recall target "
                          f"{args.target}",
                "protocol": "held out: plain efSearch and the stop threshold fixed on "
                            f"{nq} validation queries (seed {VALIDATION_SEED}); both arms timed "
                            "and scored on the benchmark queries (seed 1)",
                "learned_stop": {"ef_cap": cap, "threshold": thr, "recall_at_10": rec_l,
                                 "validation_recall_at_10": val_rec_l,
                                 "threshold_slope": net.slope, "slope_from_hops": net.slope_from,
                                 "qps": value, "mean_hops": hops_l,
                                 "audit_batches": len(audits),
                                 "audit_fallbacks": sum(f for f, _ in audits),
                                 "audit_sample_recalls": [r for _, r in audits],
                                 "in_sample": {"threshold": thr_in, "recall_at_10": rec_i,
                                               "qps": in_qps,
                                               "note": "threshold tuned on the benchmark queries "
                                                       "themselves; not the value"}},
                "plain_fixed_ef": {"ef": ef_op, "recall_at_10": rec_p, "qps": plain_qps,
                                   "mean_hops": hops_p,
                                   "achieved_gbs": alg_bytes_plain / (total_p / args.steps / 1000.0) / 1e9},
                "learned_over_plain": value / plain_qps,
                "plain_fixed_ef_fine": {"ef": ef_fine, "recall_at_10": rec_f, "qps": fine_qps,
                                        "mean_hops": hops_f},
                "learned_over_plain_fine": value / fine_qps,
                "validation_ef_sweep": {str(e): r for e, r in sweep.items()},
                "l2_policy": "inputs larger than L2 (vectors %d MB + links %d MB > 126 MB)"
                             % (arrays["vectors"].nbytes >> 20, np.asarray(arrays["links0"]).nbytes >> 20),
                "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                "start_order": ("longest predicted first (per-cell expansions learned from the "
                                "earlier batches of this run)" if g._schedule is not None and g.schedule
                                else "row order"),
                "per_query_ef_32_512": {"qps": job_throughput(world, nq, 1, pq_mean), "recall_at_10": pq_rec,
                                        "achieved_gbs": pq_bytes / (pq_mean / 1000.0) / 1e9},
                "step": "each arm's batch search recorded once as a CUDA graph (start order launches "
                        "and search kernel) and replayed; results checked equal to the synchronous "
                        "call's",
                "synchronous_call": {"ms": float(np.median(ms_sync)),
                                     "qps": nq / float(np.median(ms_sync)) * 1e3,
                                     "note": "the learned-stop step through hnsw_b200_search, which "
                                             "waits for its kernel to read the overflow count"},
                "configs": more,
                "autotune": autotune_report(g),
            },
            "roofline": {
                "bound": "hbm",
                "achieved": achieved,
                "peak": pk["hbm_gbs"],
                "unit": "GB/s",
                "frac": achieved / pk["hbm_gbs"],
                "traffic": measured_traffic(args.workload),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one learned-stop "
                                  "launch of this command (profiles/search_kernel_bytes_%s.md)" % args.workload,
                "peak_source": pk["source"],
                "algorithmic_bytes_per_launch": alg_bytes,
                "row_bytes": row_bytes,
            },
            "cpu_baseline": cpu_base,
            "e2e": {
                "value": e2e_value,
                "unit": UNIT,
                "h2d_bytes_per_step": int(raw_q.astype(np.float32).nbytes),
                "d2h_bytes_per_step": int(e_ids.nbytes + e_d.nbytes),
                "steps": e_steps,
            },
            "gpu_launches": int(launches_per_step * args.steps),
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
