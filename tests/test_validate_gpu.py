"""On-device graph validation raises exactly what the host validator (the reference's
``_validate_native`` checks, numba_engine.py:878-915) raises, for every kind of corruption."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import mix10k_arrays

pytestmark = pytest.mark.gpu

M = 16


def _copy(arrays):
    return {k: np.array(v, copy=True) for k, v in arrays.items()}


def _upper_nodes(a):
    return np.flatnonzero(a["levels"] > 0)


def neg_level(a, ep, ml):
    lv = a["levels"]
    zero = np.flatnonzero(lv == 0)
    lv[zero[0]] = -1
    lv[zero[1]] = 1  # keeps the level sum equal to the upper rows
    return ep, ml


def entry_not_top(a, ep, ml):
    other = int(np.flatnonzero(a["levels"] == 0)[0])
    return other, ml


def max_level_wrong(a, ep, ml):
    return ep, ml + 1


def count0_high(a, ep, ml):
    a["count0"][5] = 2 * M + 1
    return ep, ml


def count0_negative(a, ep, ml):
    a["count0"][7] = -2
    return ep, ml


def link0_outside(a, ep, ml):
    node = int(np.flatnonzero(a["count0"] > 3)[0])
    a["links0"][node, 2] = a["levels"].shape[0]
    return ep, ml


def link0_negative(a, ep, ml):
    node = int(np.flatnonzero(a["count0"] > 3)[1])
    a["links0"][node, 0] = -1
    return ep, ml


def rows_overlap(a, ep, ml):
    up = _upper_nodes(a)
    a["upper_offset"][up[1]] = a["upper_offset"][up[0]]
    return ep, ml


def rows_out_of_range(a, ep, ml):
    up = _upper_nodes(a)
    a["upper_offset"][up[2]] = a["links_up"].shape[0]
    return ep, ml


def count_up_high(a, ep, ml):
    a["count_up"][3] = M + 1
    return ep, ml


def link_up_outside(a, ep, ml):
    row = int(np.flatnonzero(a["count_up"] > 1)[0])
    a["links_up"][row, 1] = -5
    return ep, ml


def link_up_absent_from_layer(a, ep, ml):
    # a layer-2 row (second row of a node with level >= 2) pointing to a level-1 node
    lv, off = a["levels"], a["upper_offset"]
    node = int(np.flatnonzero(lv >= 2)[0])
    row = int(off[node]) + 1
    level1 = int(np.flatnonzero(lv == 1)[0])
    if a["count_up"][row] == 0:
        a["count_up"][row] = 1
    a["links_up"][row, 0] = level1
    return ep, ml


CORRUPTIONS = [neg_level, entry_not_top, max_level_wrong, count0_high, count0_negative,
               link0_outside, link0_negative, rows_overlap, rows_out_of_range, count_up_high,
               link_up_outside, link_up_absent_from_layer]


@pytest.mark.parametrize("corrupt", CORRUPTIONS, ids=[c.__name__ for c in CORRUPTIONS])
def test_device_validation_raises_the_host_message(corrupt) -> None:
    from hnsw_engine_b200 import HNSWIndex
    from hnsw_engine_b200.validation import validate_native

    arrays, ep, ml = mix10k_arrays()
    a = _copy(arrays)
    ep2, ml2 = corrupt(a, ep, ml)
    with pytest.raises(ValueError) as host:
        validate_native(a, ep2, ml2, M)
    with pytest.raises(ValueError) as dev:
        HNSWIndex.from_arrays(a, ep2, ml2, dim=128, metric="l2", M=M)
    assert str(dev.value) == str(host.value)


def test_valid_graph_passes_and_searches() -> None:
    from hnsw_engine_b200 import HNSWIndex

    arrays, ep, ml = mix10k_arrays()
    index = HNSWIndex.from_arrays(arrays, ep, ml, dim=128, metric="l2", M=M)
    ids, dists = index.batch_search(np.asarray(arrays["vectors"])[:4], k=1, ef=16)
    assert (dists[:, 0] == 0).all() and (ids[:, 0] >= 0).all()
