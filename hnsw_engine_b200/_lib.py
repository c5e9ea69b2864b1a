"""ctypes binding of ``libhnsw_b200.so`` (the C ABI declared in ``include/hnsw_b200.h``).

The library is built in-tree by :func:`hnsw_engine_b200.build.build`. Importing this module never
falls back to anything else: a missing or stale library raises, so the CUDA path is the only path.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libhnsw_b200.so"

OK = 0
EINVAL = -1
ECUDA = -2
ENOMEM = -3
ERETRY = -4

L2, IP, COSINE = 0, 1, 2
METRIC_CODES = {"l2": L2, "ip": IP, "cosine": COSINE}
DIST_F64 = 0
DIST_EXACT_F32 = 1
DIST_BYTES = 2


class Graph(ctypes.Structure):
    _fields_ = [
        ("vectors", ctypes.c_void_p),
        ("codes", ctypes.c_void_p),
        ("links0", ctypes.c_void_p),
        ("count0", ctypes.c_void_p),
        ("upper_offset", ctypes.c_void_p),
        ("links_up", ctypes.c_void_p),
        ("count_up", ctypes.c_void_p),
        ("n", ctypes.c_int64),
        ("rows", ctypes.c_int64),
        ("dim", ctypes.c_int32),
        ("links0_stride", ctypes.c_int32),
        ("links_up_stride", ctypes.c_int32),
        ("metric", ctypes.c_int32),
        ("entry_point", ctypes.c_int64),
        ("max_level", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("vector_bytes", ctypes.c_void_p),
        ("node_ids", ctypes.c_void_p),
    ]


class SearchArgs(ctypes.Structure):
    _fields_ = [
        ("queries", ctypes.c_void_p),
        ("queries_f64", ctypes.c_int32),
        ("use_codes", ctypes.c_int32),
        ("nq", ctypes.c_int64),
        ("k", ctypes.c_int32),
        ("k_search", ctypes.c_int32),
        ("ef", ctypes.c_void_p),
        ("ef_max", ctypes.c_int32),
        ("dist_mode", ctypes.c_int32),
        ("allowed", ctypes.c_void_p),
        ("allowed_fraction", ctypes.c_float),
        ("rerank_queries", ctypes.c_void_p),
        ("out_ids", ctypes.c_void_p),
        ("out_dists", ctypes.c_void_p),
        ("out_counters", ctypes.c_void_p),
        ("stop_mlp", ctypes.c_void_p),
        ("stop_threshold", ctypes.c_float),
        ("trace_cap", ctypes.c_int32),
        ("trace_feat", ctypes.c_void_p),
        ("trace_dk", ctypes.c_void_p),
        ("trace_count", ctypes.c_void_p),
        ("trace_hops", ctypes.c_void_p),
        ("stop_slope", ctypes.c_float),
        ("stop_slope_from", ctypes.c_int32),
        ("priority", ctypes.c_void_p),
        ("cells", ctypes.c_void_p),
        ("cell_cost", ctypes.c_void_p),
        ("n_cells", ctypes.c_int32),
        ("kernel_config", ctypes.c_int32),
    ]


class ExactArgs(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("queries", ctypes.c_void_p),
        ("dtype", ctypes.c_int32),
        ("dim", ctypes.c_int32),
        ("n", ctypes.c_int64),
        ("nq", ctypes.c_int64),
        ("k", ctypes.c_int32),
        ("metric", ctypes.c_int32),
        ("integer_valued", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("out_ids", ctypes.c_void_p),
        ("out_dists", ctypes.c_void_p),
        ("out_filter_max_error", ctypes.c_void_p),
        ("out_candidates", ctypes.c_void_p),
        ("out_launches", ctypes.c_void_p),
        ("out_filter_error_bound", ctypes.c_void_p),
    ]


class ValueStats(ctypes.Structure):
    """``hnsw_b200_value_stats_t``."""

    _fields_ = [
        ("finite", ctypes.c_int32),
        ("integer", ctypes.c_int32),
        ("min", ctypes.c_double),
        ("max", ctypes.c_double),
    ]


# Every symbol include/hnsw_b200.h declares, with its ctypes signature.
SIGNATURES: dict[str, tuple[object, list[object]]] = {
    "hnsw_b200_open": (ctypes.c_int, [ctypes.POINTER(Graph), ctypes.POINTER(ctypes.c_void_p)]),
    "hnsw_b200_close": (None, [ctypes.c_void_p]),
    "hnsw_b200_search": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SearchArgs), ctypes.c_void_p]),
    "hnsw_b200_exact_knn": (ctypes.c_int, [ctypes.POINTER(ExactArgs), ctypes.c_void_p]),
    "hnsw_b200_mlp_param_count": (ctypes.c_int64, []),
    "hnsw_b200_mlp_packed_bytes": (ctypes.c_int64, []),
    "hnsw_b200_mlp_scratch_bytes": (ctypes.c_int64, [ctypes.c_int32]),
    "hnsw_b200_mlp_train_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_int64, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "hnsw_b200_mlp_gradients": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.c_void_p]),
    "hnsw_b200_mlp_predict": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                               ctypes.c_void_p, ctypes.c_void_p]),
    "hnsw_b200_mlp_pack": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_void_p, ctypes.c_void_p]),
    "hnsw_b200_search_noalloc": (ctypes.c_int, [ctypes.POINTER(Graph), ctypes.POINTER(SearchArgs),
                                  ctypes.c_void_p]),
    "hnsw_b200_last_launches": (ctypes.c_int64, [ctypes.c_void_p]),
    "hnsw_b200_last_error": (ctypes.c_char_p, []),
    "hnsw_b200_validate_scratch_bytes": (ctypes.c_int64, [ctypes.c_int64]),
    "hnsw_b200_quant_scratch_bytes": (ctypes.c_int64, [ctypes.c_int32]),
    "hnsw_b200_quant_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.c_void_p,
                                             ctypes.c_void_p]),
    "hnsw_b200_quant_encode": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p,
                                              ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]),
    "hnsw_b200_validate_graph": (ctypes.c_int, [ctypes.POINTER(Graph), ctypes.c_void_p, ctypes.c_int32,
                                                ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32),
                                                ctypes.c_void_p]),
    "hnsw_b200_upload_queries": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                                ctypes.c_int32, ctypes.POINTER(ValueStats),
                                                ctypes.c_void_p, ctypes.c_void_p]),
    "hnsw_b200_start_priority": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                                                ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_void_p]),
    "hnsw_b200_version": (ctypes.c_char_p, []),
    "hnsw_b200_kernel_configs": (ctypes.c_int32, [ctypes.c_int32]),
    "hnsw_b200_search_async": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(SearchArgs),
                                              ctypes.c_void_p]),
    "hnsw_b200_search_failed": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                               ctypes.c_void_p]),
    "hnsw_b200_kernel_config_name": (ctypes.c_char_p, [ctypes.c_int32, ctypes.c_int32]),
}

_lib: ctypes.CDLL | None = None


class HnswB200Error(RuntimeError):
    """A C-ABI call failed; ``code`` is the negative status it returned."""

    def __init__(self, code: int, message: str) -> None:
        super().__init__(f"hnsw_b200 error {code}: {message}")
        self.code = code


def load() -> ctypes.CDLL:
    """The loaded library with argument types set; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.is_file():
            raise ImportError(
                f"{LIB_PATH} is missing: build the CUDA extension first "
                "(python -c 'import hnsw_engine_b200.build as b; b.build()')"
            )
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib


def check(code: int) -> None:
    """Raise :class:`HnswB200Error` for a nonzero status."""
    if code != OK:
        msg = load().hnsw_b200_last_error()
        raise HnswB200Error(code, msg.decode() if msg else "")
