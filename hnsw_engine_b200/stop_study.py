"""How much a learned stop can gain on a workload: oracle bounds and the signal in the stop features.

    python -m hnsw_engine_b200.stop_study --workload mix1m

Searches the workload's queries with the plain GPU kernel at a cap efSearch (512) with the trace
on (the stop features and the first 16 result distances every 16 layer-0 expansions), labels
every checkpoint with its tie-aware recall@10 hits against the tensor-core exact k-NN, and prints
one JSON object:

* ``plain``: recall and mean layer-0 expansions of plain fixed efSearch on a ladder (from the
  cap search's own trajectory: a search at a smaller efSearch follows the same expansions and
  stops once its efSearch-th result is expanded; the kernel's counters give the exact figures);
* ``oracle_complete_stop``: stop each query at the first checkpoint holding all the hits its
  search at the cap will reach -- what a perfect detector of "the top 10 are found" would spend;
* ``oracle_budget``: per-query stop checkpoints chosen with hindsight to minimise mean expansions
  at mean recall >= target (a Lagrangian over each query's hits curve);
* ``completion_auc``: at fixed checkpoints, the ROC AUC of a gradient-boosted classifier on the
  12 stop features (trained on the training queries, scored on the held-out ones) for "this
  query already has its final hits"; 0.5 is no signal;
* ``query_level_spearman``: rank correlation of each query's completion expansions with the
  query-level features the kernel can see before searching (nearest-pivot distance, layer-0 entry
  distance).

There is no reference counterpart; it is a study of this engine's learned stop.
"""

from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from . import graphs, synthetic
from .exact_knn import exact_search
from .index import HNSWIndex
from .learned_stop import STOP_EVERY, checkpoint_hits, collect_traces
from .metrics import RELATIVE_TIE_TOLERANCE
from .validation import prepare


def _auc(score: np.ndarray, label: np.ndarray) -> float:
    order = np.argsort(score, kind="stable")
    ranks = np.empty(len(score))
    ranks[order] = np.arange(1, len(score) + 1)
    pos = label.astype(bool)
    n_pos, n_neg = int(pos.sum()), int((~pos).sum())
    if n_pos == 0 or n_neg == 0:
        return float("nan")
    return float((ranks[pos].sum() - n_pos * (n_pos + 1) / 2) / (n_pos * n_neg))


def _spearman(a: np.ndarray, b: np.ndarray) -> float:
    ra = np.argsort(np.argsort(a)).astype(np.float64)
    rb = np.argsort(np.argsort(b)).astype(np.float64)
    return float(np.corrcoef(ra, rb)[0, 1])


def study(workload: str = "mix1m", cap: int = 512, n_train: int = 20_000, n_test: int = 10_000,
          k: int = 10, target: float = 0.95, device: str = "cuda") -> dict:
    meta, arrays = graphs.open_workload(workload)
    params = {kk: v for kk, v in meta["params"].items() if kk != "engine"}
    metric = params["metric"]
    index = HNSWIndex.from_arrays(arrays, int(meta["entry_point"]), int(meta["max_level"]),
                                  device=device, **params)
    g = index.device_graph
    train_seed = synthetic.TRAIN_SEED if graphs.WORKLOADS[workload]["gen"] == "mixture" else synthetic.T_TRAIN_SEED
    out: dict = {"workload": workload, "cap_ef": cap, "target": target, "checkpoint_every": STOP_EVERY}
    sets = {}
    for name, nq, seed in (("train", n_train, train_seed), ("test", n_test, None)):
        q = prepare(graphs.workload_queries(workload, nq=nq, seed=seed), metric)
        qd = torch.from_numpy(q).to(g.device)
        tr = collect_traces(g, q, k, cap, trace_cap=cap // STOP_EVERY + 8)
        _, true_d = exact_search(g.vectors, qd, k, metric)
        kth = true_d[:, k - 1].cpu().numpy()
        hits, final = checkpoint_hits(tr, kth)
        sets[name] = (q, qd, tr, hits, final, kth)

    q, qd, tr, hits, final, kth = sets["test"]
    nq, ncp = hits.shape
    cps = (np.arange(ncp) + 1) * STOP_EVERY
    valid = np.arange(ncp)[None, :] < tr.count[:, None]
    # plain fixed ef, measured by the kernel itself (expansions from its counters)
    plain = {}
    for ef in (64, 128, 160, 176, 184, 192, 224, 256, 320, 384, 512):
        if ef > cap:
            continue
        ids, d, c = g.search(qd, k, ef)
        thr = kth + RELATIVE_TIE_TOLERANCE * np.maximum(1.0, np.abs(kth))
        h = (d.cpu().numpy()[:, :k] <= thr[:, None]).sum(1)
        plain[str(ef)] = {"recall": float(h.mean() / k), "mean_hops": float(c[:, 1].float().mean())}
    out["plain"] = plain
    # oracle: first checkpoint with the final hits (or the end of the search)
    done = valid & (hits >= final[:, None])
    first = np.where(done.any(1), done.argmax(1), -1)
    stop_at = np.where(first >= 0, cps[np.maximum(first, 0)], tr.hops)
    stop_at = np.minimum(stop_at, tr.hops)
    out["oracle_complete_stop"] = {"recall": float(final.mean() / k),
                                   "mean_layer0_expansions": float(stop_at.mean()),
                                   "cap_search_mean_layer0_expansions": float(tr.hops.mean())}
    # Lagrangian budget oracle over (checkpoint, hits) options, plus the full search
    opt_t = np.concatenate([np.where(valid, cps[None, :], np.inf), tr.hops[:, None].astype(float)], 1)
    opt_h = np.concatenate([np.where(valid, hits, -1), final[:, None]], 1).astype(float)

    def alloc(lam: float):
        v = opt_h - lam * opt_t
        j = np.argmax(v, 1)
        return opt_t[np.arange(nq), j].mean(), opt_h[np.arange(nq), j].mean() / k

    lo, hi = 0.0, 1.0
    for _ in range(50):
        mid = 0.5 * (lo + hi)
        if alloc(mid)[1] >= target:
            lo = mid
        else:
            hi = mid
    t_b, r_b = alloc(lo)
    out["oracle_budget"] = {"recall": float(r_b), "mean_layer0_expansions": float(t_b)}
    # completion detection signal of the 12 features
    from sklearn.ensemble import HistGradientBoostingClassifier

    _, _, tr_tr, hits_tr, final_tr, _ = sets["train"]
    auc = {}
    for cp in (3, 5, 7, 9, 11):
        if cp >= ncp:
            continue
        m_tr = cp < tr_tr.count
        m_te = cp < tr.count
        y_tr = hits_tr[m_tr, cp] >= final_tr[m_tr]
        y_te = hits[m_te, cp] >= final[m_te]
        clf = HistGradientBoostingClassifier(max_iter=200, random_state=0)
        clf.fit(tr_tr.feat[m_tr, cp], y_tr)
        auc[str(int(cps[cp]))] = {"share_complete": float(y_te.mean()),
                                  "auc": _auc(clf.predict_proba(tr.feat[m_te, cp])[:, 1], y_te)}
    out["completion_auc"] = auc
    # query-level signals
    sched = g._schedule
    t_complete = stop_at.astype(np.float64)
    qlev = {}
    if sched is not None:
        piv = sched.pivots
        dq = torch.cdist(qd.double(), piv.double()).min(1).values.cpu().numpy()
        qlev["nearest_pivot_distance"] = _spearman(dq, t_complete)
    qlev["layer0_entry_distance"] = _spearman(tr.feat[:, 0, 6], t_complete)
    out["query_level_spearman"] = qlev
    return out


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--workload", default="mix1m")
    p.add_argument("--cap", type=int, default=512)
    p.add_argument("--n-train", type=int, default=20_000)
    args = p.parse_args()
    print(json.dumps(study(args.workload, args.cap, args.n_train)), flush=True)


if __name__ == "__main__":
    main()
