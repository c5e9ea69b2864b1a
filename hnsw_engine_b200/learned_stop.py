"""Learned early termination of the layer-0 search (no reference counterpart).

Every 16 layer-0 expansions the search kernel computes 12 search-progress features (best and k-th
result distances, the k-th distance's change over the last one and two checkpoints, expansions and
distance computations so far, the layer-0 entry distance, the share of the first k results not yet
expanded, the k-th distance relative to the entry distance, checkpoints since the first k last
changed, how many admissions entered the first k since the last checkpoint, and the frontier
distance relative to the k-th). A 12 -> 64 -> 64 -> 1 ReLU network with BF16 weights predicts the
recall@k hits (tie-aware, as ``recall_at_k``) that the query would still gain by searching on to the
cap efSearch; the kernel stops a query once the predicted gain falls below a threshold tuned for the
recall target.

Pipeline (all GPU work in ``libhnsw_b200``):

1. :func:`collect_traces` -- plain search at the cap efSearch with the trace buffers on;
2. :func:`label_traces` -- the exact k-th distances (tensor-core exact k-NN) give, per checkpoint,
   the hits the search would still gain;
3. :class:`StopNetwork.fit` -- hand-written CUDA forward/backward/Adam (``hnsw_b200_mlp_*``);
4. :func:`tune_threshold` -- bisection on a validation set for the recall target;
5. search with ``stop_mlp`` / ``stop_threshold`` (``StopNetwork.packed``); the plain fixed-ef search
   is the fallback (:func:`audited_search`).
"""

from __future__ import annotations

import ctypes
import json
from dataclasses import dataclass
from pathlib import Path
from typing import Any

import numpy as np
import torch
from numpy.typing import NDArray

from . import _lib
from .engine import DeviceGraph
from .metrics import RELATIVE_TIE_TOLERANCE

FEATURES = 12
HIDDEN = 64
STOP_EVERY = 16
FEATURE_NAMES = (
    "log1p_d1", "log1p_dk", "dk_change_1", "dk_change_2", "hops_div64", "dists_div1024",
    "log1p_d_entry", "unexpanded_in_topk", "dk_minus_entry", "stale_checkpoints_div4",
    "topk_churn", "frontier_minus_dk",
)


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else int(t.data_ptr())


def _stream(dev: torch.device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


# ------------------------------------------------------------------------------------- traces
@dataclass
class Traces:
    feat: NDArray[np.float32]     # (nq, cap, 12)
    dk: NDArray[np.float64]       # (nq, cap, kt) first results' distances at each checkpoint
    count: NDArray[np.int32]      # (nq,) checkpoints recorded
    hops: NDArray[np.int32]       # (nq,) layer-0 expansions of the whole search
    final_d: NDArray[np.float64]  # (nq, k) distances returned by the full search


def collect_traces(graph: DeviceGraph, queries: Any, k: int, ef: int, trace_cap: int = 64,
                   chunk: int = 20000) -> Traces:
    """Plain search at ``ef`` recording the stop features every 16 layer-0 expansions."""
    dev = graph.device
    nq = int(queries.shape[0])
    feat = np.empty((nq, trace_cap, FEATURES), np.float32)
    kt = 16  # the kernel records the first 16 result distances per checkpoint
    dk = np.empty((nq, trace_cap, kt), np.float64)
    count = np.empty(nq, np.int32)
    hops = np.empty(nq, np.int32)
    final = np.empty((nq, k), np.float64)
    for s in range(0, nq, chunk):
        e = min(nq, s + chunk)
        m = e - s
        tf = torch.empty((m, trace_cap, FEATURES), dtype=torch.float32, device=dev)
        td = torch.empty((m, trace_cap, kt), dtype=torch.float64, device=dev)
        tc = torch.zeros(m, dtype=torch.int32, device=dev)
        th = torch.zeros(m, dtype=torch.int32, device=dev)
        _, dists, _ = graph.search(queries[s:e], k, ef, trace=(tf, td, tc, th))
        feat[s:e] = tf.cpu().numpy()
        dk[s:e] = td.cpu().numpy()
        count[s:e] = tc.cpu().numpy()
        hops[s:e] = th.cpu().numpy()
        final[s:e] = dists[:, :k].cpu().numpy()
    return Traces(feat, dk, count, hops, final)


def checkpoint_hits(tr: Traces, true_kth: NDArray[np.float64]) -> tuple[NDArray, NDArray]:
    """Tie-aware hits of the first k results at every checkpoint, and of the final result.

    Results are unique and sorted, so a result counts exactly when its distance is within the
    tie-aware threshold of the exact k-th distance (``recall_at_k``'s rule).
    """
    thr = true_kth + RELATIVE_TIE_TOLERANCE * np.maximum(1.0, np.abs(true_kth))
    k = tr.final_d.shape[1]
    hits = (tr.dk[:, :, :k] <= thr[:, None, None]).sum(axis=2)
    final = (tr.final_d <= thr[:, None]).sum(axis=1)
    return hits, final


def label_traces(tr: Traces, true_kth: NDArray[np.float64], target: str = "gain"
                 ) -> tuple[NDArray, NDArray, NDArray]:
    """Samples ``(X, y, qid)`` from every recorded checkpoint.

    ``target="gain"`` (default): y = the recall@k hits the search would still add by running to its
    end (the full search's tie-aware hits minus the checkpoint's); stopping where the predicted
    gain is small trades the fewest hits for the most saved work, which is what an average recall
    target rewards. ``target="remaining"``: y = log1p(checkpoints remaining until the result
    reaches its final hits).
    """
    nq, cap = tr.dk.shape[:2]
    cps = np.arange(cap)[None, :]
    valid = cps < tr.count[:, None]
    hits, final = checkpoint_hits(tr, true_kth)
    if target == "gain":
        y = np.maximum(0, final[:, None] - hits).astype(np.float32)
    else:
        ok = valid & (hits >= final[:, None])
        first = np.where(ok.any(axis=1), ok.argmax(axis=1), -1)
        end_cp = tr.hops / STOP_EVERY  # the search ends after this many checkpoints
        last = np.where(first >= 0, first, np.maximum(end_cp, tr.count))
        y = np.log1p(np.maximum(0.0, last[:, None] - cps)).astype(np.float32)
    X = tr.feat[valid]
    return X, y[valid], np.broadcast_to(np.arange(nq)[:, None], (nq, cap))[valid]


# ------------------------------------------------------------------------------------ network
def init_params(seed: int = 0) -> NDArray[np.float32]:
    """He-style initialisation of W1[64][12], b1, W2[64][64], b2, W3[64], b3."""
    rng = np.random.default_rng(seed)
    return np.concatenate([
        rng.standard_normal(HIDDEN * FEATURES) * np.sqrt(2.0 / FEATURES), np.zeros(HIDDEN),
        rng.standard_normal(HIDDEN * HIDDEN) * np.sqrt(2.0 / HIDDEN), np.zeros(HIDDEN),
        rng.standard_normal(HIDDEN) * np.sqrt(1.0 / HIDDEN), np.zeros(1),
    ]).astype(np.float32)


class StopNetwork:
    """The early-termination network, trained and evaluated by the library's CUDA kernels."""

    def __init__(self, device: str | torch.device = "cuda", seed: int = 0) -> None:
        self.lib = _lib.load()
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        n = int(self.lib.hnsw_b200_mlp_param_count())
        self.params = torch.from_numpy(init_params(seed)).to(self.device)
        assert self.params.numel() == n
        self.m = torch.zeros(n, dtype=torch.float32, device=self.device)
        self.v = torch.zeros(n, dtype=torch.float32, device=self.device)
        self.step = 0
        self.mean = np.zeros(FEATURES, np.float32)
        self.std = np.ones(FEATURES, np.float32)
        self.threshold = 0.0
        # threshold schedule: + slope per 64 layer-0 expansions beyond slope_from (0: constant)
        self.slope = 0.0
        self.slope_from = 0
        self.ef_cap = 256
        self.history: list[float] = []

    def _norm(self, X: NDArray) -> NDArray[np.float32]:
        return ((X.astype(np.float32) - self.mean) * (1.0 / self.std).astype(np.float32)).astype(np.float32)

    def fit(self, X: NDArray, y: NDArray, *, epochs: int = 4, batch: int = 4096, lr: float = 2e-3,
            seed: int = 0) -> list[float]:
        """Adam on mean squared error over shuffled mini-batches (standardised features)."""
        self.mean = X.mean(axis=0).astype(np.float32)
        self.std = np.maximum(X.std(axis=0), 1e-6).astype(np.float32)
        Xd = torch.from_numpy(self._norm(X)).to(self.device)
        yd = torch.from_numpy(np.ascontiguousarray(y, dtype=np.float32)).to(self.device)
        n = Xd.shape[0]
        scratch = torch.empty(int(self.lib.hnsw_b200_mlp_scratch_bytes(batch)) // 4 + 1,
                              dtype=torch.float32, device=self.device)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        g = torch.Generator(device="cpu").manual_seed(seed)
        losses = []
        with torch.cuda.device(self.device):
            for ep in range(epochs):
                order = torch.randperm(n, generator=g).to(self.device)
                ep_loss, nb = 0.0, 0
                rate = lr * (0.5 ** ep)
                for s in range(0, n - batch + 1, batch):
                    idx = order[s : s + batch]
                    xb, yb = Xd[idx].contiguous(), yd[idx].contiguous()
                    self.step += 1
                    _lib.check(self.lib.hnsw_b200_mlp_train_step(
                        _ptr(self.params), _ptr(self.m), _ptr(self.v), self.step, rate, _ptr(xb),
                        _ptr(yb), batch, _ptr(scratch), _ptr(loss), _stream(self.device)))
                    if nb % 50 == 0:
                        ep_loss += float(loss.item())
                    nb += 1
                losses.append(ep_loss / max(1, (nb + 49) // 50))
        self.history += losses
        return losses

    def gradients(self, X: NDArray, y: NDArray) -> tuple[NDArray, float]:
        """CUDA gradients of the batch loss at the current parameters (features used as given)."""
        B = X.shape[0]
        Xd = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(self.device)
        yd = torch.from_numpy(np.ascontiguousarray(y, dtype=np.float32)).to(self.device)
        scratch = torch.empty(int(self.lib.hnsw_b200_mlp_scratch_bytes(B)) // 4 + 1,
                              dtype=torch.float32, device=self.device)
        grads = torch.empty_like(self.params)
        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.hnsw_b200_mlp_gradients(_ptr(self.params), _ptr(Xd), _ptr(yd), B,
                                                        _ptr(scratch), _ptr(grads), _ptr(loss),
                                                        _stream(self.device)))
        return grads.cpu().numpy(), float(loss.item())

    def predict(self, X: NDArray, normalize: bool = True) -> NDArray[np.float32]:
        Xn = self._norm(X) if normalize else np.ascontiguousarray(X, dtype=np.float32)
        Xd = torch.from_numpy(Xn).to(self.device)
        out = torch.empty(Xd.shape[0], dtype=torch.float32, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.hnsw_b200_mlp_predict(_ptr(self.params), _ptr(Xd), Xd.shape[0],
                                                      _ptr(out), _stream(self.device)))
        return out.cpu().numpy()

    def packed(self) -> torch.Tensor:
        """The network in the search kernel's layout (BF16 weights, standardisation included)."""
        nbytes = int(self.lib.hnsw_b200_mlp_packed_bytes())
        out = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        mu = torch.from_numpy(self.mean).to(self.device)
        inv = torch.from_numpy((1.0 / self.std).astype(np.float32)).to(self.device)
        with torch.cuda.device(self.device):
            _lib.check(self.lib.hnsw_b200_mlp_pack(_ptr(self.params), _ptr(mu), _ptr(inv), _ptr(out),
                                                   _stream(self.device)))
        return out

    def save(self, path: str | Path) -> None:
        root = Path(path)
        root.mkdir(parents=True, exist_ok=True)
        np.save(root / "params.npy", self.params.cpu().numpy())
        np.save(root / "adam_m.npy", self.m.cpu().numpy())
        np.save(root / "adam_v.npy", self.v.cpu().numpy())
        np.save(root / "mean.npy", self.mean)
        np.save(root / "std.npy", self.std)
        (root / "meta.json").write_text(json.dumps({
            "step": self.step, "threshold": self.threshold, "ef_cap": self.ef_cap,
            "slope": self.slope, "slope_from": self.slope_from,
            "history": self.history, "features": FEATURE_NAMES, "stop_every": STOP_EVERY,
        }, indent=2))

    @classmethod
    def load(cls, path: str | Path, device: str | torch.device = "cuda") -> StopNetwork:
        root = Path(path)
        net = cls(device)
        net.params = torch.from_numpy(np.load(root / "params.npy")).to(net.device)
        net.m = torch.from_numpy(np.load(root / "adam_m.npy")).to(net.device)
        net.v = torch.from_numpy(np.load(root / "adam_v.npy")).to(net.device)
        net.mean = np.load(root / "mean.npy")
        net.std = np.load(root / "std.npy")
        meta = json.loads((root / "meta.json").read_text())
        if tuple(meta.get("features", ())) != FEATURE_NAMES:
            raise ValueError(f"{root}: network trained on different stop features")
        net.step, net.threshold, net.history = meta["step"], meta["threshold"], meta["history"]
        net.ef_cap = int(meta.get("ef_cap", 256))
        net.slope = float(meta.get("slope", 0.0))
        net.slope_from = int(meta.get("slope_from", 0))
        return net

    def stop_args(self, threshold: float | None = None) -> tuple[torch.Tensor, float, float, int]:
        """The ``stop=`` argument of :meth:`DeviceGraph.search` for this network."""
        return (self.packed(), self.threshold if threshold is None else float(threshold),
                self.slope, self.slope_from)


# ------------------------------------------------------------------------- threshold and search
def stopped_search(graph: DeviceGraph, queries: Any, k: int, ef: int, packed: torch.Tensor,
                   threshold: float, slope: float = 0.0, slope_from: int = 0, **kw: Any):
    """One batched search with the learned stop; returns device ``(ids, dists, counters)``."""
    return graph.search(queries, k, ef, stop=(packed, threshold, slope, slope_from), **kw)


def recall_of(ids: NDArray, dists: NDArray, true_dist: NDArray, k: int) -> float:
    from .metrics import per_query_hits

    return float(per_query_hits(ids, dists, true_dist, k).mean() / k)


def tune_threshold(graph: DeviceGraph, net: StopNetwork, queries: Any, true_dist: NDArray, k: int,
                   ef: int, target: float, iters: int = 14) -> tuple[float, float]:
    """Largest threshold (earliest stops) whose measured recall@k on ``queries`` meets ``target``."""
    packed = net.packed()
    lo, hi = -1.0, 4.0  # predictions are expected further hits (0 .. k)
    best = (lo, 0.0)
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        ids, d, _ = stopped_search(graph, queries, k, ef, packed, mid, net.slope, net.slope_from)
        rec = recall_of(ids.cpu().numpy(), d.cpu().numpy(), true_dist, k)
        if rec >= target:
            best = (mid, rec)
            lo = mid
        else:
            hi = mid
    if best[1] == 0.0:
        ids, d, _ = stopped_search(graph, queries, k, ef, packed, lo, net.slope, net.slope_from)
        best = (lo, recall_of(ids.cpu().numpy(), d.cpu().numpy(), true_dist, k))
    net.threshold = best[0]
    return best


def audited_search(graph: DeviceGraph, queries: Any, k: int, ef_cap: int, net: StopNetwork,
                   fallback_ef: int, target: float, audit_fraction: float = 0.02, seed: int = 0):
    """Learned-stop search with a per-batch recall audit; plain fixed-ef search is the fallback.

    A random ``audit_fraction`` of the batch is checked against the exact k-NN; if its recall is
    below ``target`` the whole batch is searched again with plain fixed ``fallback_ef``. Returns
    ``(ids, dists, fell_back, audit_recall)`` (device tensors).
    """
    from .exact_knn import exact_search

    ids, dists, _ = stopped_search(graph, queries, k, ef_cap, net.packed(), net.threshold,
                                   net.slope, net.slope_from, counters=False)
    nq = int(queries.shape[0])
    rng = np.random.default_rng(seed)
    sample = np.sort(rng.choice(nq, size=max(1, int(round(audit_fraction * nq))), replace=False))
    q_host = queries.cpu().numpy() if isinstance(queries, torch.Tensor) else np.asarray(queries)
    _, true_d = exact_search(graph.vectors, torch.from_numpy(q_host[sample]).to(graph.device), k,
                             graph.metric)
    rec = recall_of(ids[sample].cpu().numpy(), dists[sample].cpu().numpy(), true_d.cpu().numpy(), k)
    if rec >= target:
        return ids, dists, False, rec
    ids, dists, _ = graph.search(queries, k, fallback_ef, counters=False)
    return ids, dists, True, rec
