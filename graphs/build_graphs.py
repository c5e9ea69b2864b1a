"""Build the benchmark graphs with the reference's own host build and save them in its native layout.

Graph construction stays on the reference's insertion code (``HNSWIndex.add``,
``src/hnsw_engine/index.py:219-223`` -> ``numba_engine._insert_batch``), because its sequential
insertion order defines the graph the GPU engine must search. This script needs the reference
importable (``--reference-src``), so it runs where the reference is checked out; its output
directories (``graphs/<name>/``, git-ignored) are what the engine, the tests and ``bench.py`` read.

``save_native`` writes ``header.json`` plus seven ``.npy`` arrays
(``src/hnsw_engine/persistence.py:192-213``). ``--drop-vectors`` removes ``vectors.npy``
afterwards and records its SHA-256 in ``vectors.sha256``: the vectors are a pure function of the
generator seed, so loaders regenerate them (:func:`hnsw_engine_b200.graphs.open_workload`) and
check the digest, which keeps the directories small enough to ship.

Usage::

    NUMBA_CACHE_DIR=/tmp/numba python graphs/build_graphs.py --reference-src <ref>/src mix10k
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))

from hnsw_engine_b200.graphs import WORKLOADS, workload_vectors  # noqa: E402


def build(name: str, reference_src: str, drop_vectors: bool) -> None:
    sys.path.insert(0, reference_src)
    from hnsw_engine import HNSWIndex  # the reference package

    spec = WORKLOADS[name]
    out = HERE / name
    t0 = time.time()
    data = workload_vectors(name)
    index = HNSWIndex(
        spec["dim"],
        metric=spec["metric"],
        M=spec["M"],
        ef_construction=spec["ef_construction"],
        seed=spec["level_seed"],
        engine="numba",
    )
    index.add(data)
    build_s = time.time() - t0
    index.save_native(out)
    vec = out / "vectors.npy"
    import numpy as np

    stored = np.load(vec, mmap_mode="r")
    digest = hashlib.sha256(np.ascontiguousarray(stored).tobytes()).hexdigest()
    (out / "vectors.sha256").write_text(digest + "\n")
    if drop_vectors:
        os.remove(vec)
    (out / "build.json").write_text(
        json.dumps({"workload": name, "build_seconds": build_s, **spec}, indent=2)
    )
    print(f"{name}: built in {build_s:.1f} s -> {out}", flush=True)


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("names", nargs="+", choices=sorted(WORKLOADS))
    parser.add_argument("--reference-src", required=True)
    parser.add_argument("--drop-vectors", action="store_true")
    args = parser.parse_args()
    for name in args.names:
        build(name, args.reference_src, args.drop_vectors)


if __name__ == "__main__":
    main()
