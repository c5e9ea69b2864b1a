"""The C ABI without a GPU: the library loads, exports every entry point the header declares, and
its host-side argument checks answer before any device work."""

from __future__ import annotations

import ctypes
import re

import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "hnsw_b200.h"


def declared_functions() -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    return sorted(set(re.findall(r"\b(hnsw_b200_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from hnsw_engine_b200 import _lib, build

    build.build()  # no-op when up to date
    return _lib.load()


def test_header_declares_the_entry_points() -> None:
    names = declared_functions()
    for expected in ("hnsw_b200_open", "hnsw_b200_search", "hnsw_b200_close", "hnsw_b200_exact_knn",
                     "hnsw_b200_mlp_train_step", "hnsw_b200_search_noalloc", "hnsw_b200_last_error"):
        assert expected in names


def test_library_exports_every_declared_symbol(lib) -> None:
    from hnsw_engine_b200._lib import SIGNATURES

    names = declared_functions()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python bindings type every declared function, and nothing undeclared
    assert sorted(SIGNATURES) == names


def test_pure_host_queries(lib) -> None:
    assert lib.hnsw_b200_version().decode()
    # 12*64 + 64 + 64*64 + 64 + 64 + 1 parameters of the stop network
    assert lib.hnsw_b200_mlp_param_count() == 5057
    # bf16 W1^T, W2^T, W3 then f32 b1, b2, b3, feature mean and 1/std
    assert lib.hnsw_b200_mlp_packed_bytes() == 2 * (768 + 4096 + 64) + 4 * (64 + 64 + 1 + 24)
    assert 0 < lib.hnsw_b200_mlp_scratch_bytes(256) < lib.hnsw_b200_mlp_scratch_bytes(4096)


def test_open_rejects_bad_graphs_before_device_work(lib) -> None:
    from hnsw_engine_b200._lib import Graph

    h = ctypes.c_void_p()
    assert lib.hnsw_b200_open(None, ctypes.byref(h)) == -1
    assert "null" in lib.hnsw_b200_last_error().decode()
    g = Graph(n=0, dim=4, metric=0)
    assert lib.hnsw_b200_open(ctypes.byref(g), ctypes.byref(h)) == -1
    assert "n must be" in lib.hnsw_b200_last_error().decode()
    fake = 4096  # never dereferenced: the checks below fail first
    g = Graph(vectors=fake, links0=fake, count0=fake, upper_offset=fake, n=10, dim=4, metric=7,
              links0_stride=33, links_up_stride=17)
    assert lib.hnsw_b200_open(ctypes.byref(g), ctypes.byref(h)) == -1
    assert "metric" in lib.hnsw_b200_last_error().decode()
    g.metric = 0
    g.entry_point = 10
    assert lib.hnsw_b200_open(ctypes.byref(g), ctypes.byref(h)) == -1
    assert "entry point" in lib.hnsw_b200_last_error().decode()
    assert not h.value


def test_search_rejects_a_null_handle(lib) -> None:
    from hnsw_engine_b200._lib import SearchArgs

    a = SearchArgs(nq=1, k=1, k_search=1)
    assert lib.hnsw_b200_search(None, ctypes.byref(a), None) == -1


def test_missing_library_fails_loudly(monkeypatch, tmp_path) -> None:
    from hnsw_engine_b200 import _lib

    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "absent.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError, match="missing"):
        _lib.load()
