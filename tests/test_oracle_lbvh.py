"""Known-answer tests of the oracle's LBVH and SAH builders, restated from
crates/core/src/lbvh.rs:624-773, crates/core/tests/lbvh_build.rs and
crates/gpu/tests/radix_sort.rs. CPU only."""
import numpy as np
import pytest

import oracle as O


def _lib():
    return O.lib()


def test_expand_bits_known_answers():  # lbvh.rs:628-647
    L = _lib()
    assert L.orc_expand_bits(0x3FF) == 0x09249249
    assert L.orc_expand_bits(0) == 0
    for k in range(10):
        assert L.orc_expand_bits(1 << k) == 1 << (3 * k)
    assert L.orc_expand_bits(0xFFFFFC00) == 0  # bits above 10 are discarded


def test_morton_lanes_and_monotonicity():  # lbvh.rs:650-682
    L = _lib()
    assert L.orc_morton3d(1.0, 0.0, 0.0) == 0x09249249 << 2
    assert L.orc_morton3d(0.0, 1.0, 0.0) == 0x09249249 << 1
    assert L.orc_morton3d(0.0, 0.0, 1.0) == 0x09249249
    assert L.orc_morton3d(1.0, 1.0, 1.0) == 0x3FFFFFFF
    assert L.orc_morton3d(0.0, 0.0, 0.0) == 0
    # clamped: out of range and NaN quantise to the ends / zero
    assert L.orc_morton3d(2.0, -1.0, float("nan")) == 0x09249249 << 2
    prev = -1
    for i in range(1024):
        c = L.orc_morton3d(i / 1023.0, 0.0, 0.0)
        assert c > prev
        prev = c


def test_longest_common_prefix():  # lbvh.rs:740-772
    codes = np.array([0b000, 0b001, 0b011, 0b011, 0b100], np.uint32)
    L = _lib()
    p = codes.ctypes.data_as(O.C.c_void_p)
    n = len(codes)
    assert L.orc_lcp(p, n, 0, 1) == 31
    assert L.orc_lcp(p, n, 1, 2) == 30
    assert L.orc_lcp(p, n, 0, 4) == 29
    assert L.orc_lcp(p, n, 0, -1) == -1 and L.orc_lcp(p, n, 4, 5) == -1
    # duplicates fall back to the index: 32 + clz(2 ^ 3)
    assert L.orc_lcp(p, n, 2, 3) == 32 + 31


def _random_mesh(n, seed):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-10, 10, (n, 3)).astype(np.float32)
    pos = np.zeros((3 * n, 4), np.float32)
    for k in range(3):
        pos[k::3, :3] = centres + rng.uniform(-0.3, 0.3, (n, 3)).astype(np.float32)
    tris = np.zeros(n, O.TRIANGLE)
    tris["i0"], tris["i1"], tris["i2"] = np.arange(n) * 3, np.arange(n) * 3 + 1, np.arange(n) * 3 + 2
    return tris, pos


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 100, 1000])
def test_lbvh_invariants(n):  # crates/core/tests/lbvh_build.rs
    tris, pos = _random_mesh(n, n)
    lb = O.Lbvh(tris, pos)
    assert sorted(lb.prim_indices.tolist()) == list(range(n))  # a permutation
    assert np.all(np.diff(lb.sorted_codes.astype(np.int64)) >= 0)  # sorted
    leaves = lb.nodes[lb.nodes["count"] > 0]
    assert leaves["count"].max() <= 4
    assert leaves["count"].sum() == n
    if n > 1:
        assert lb.subtree_size[0] == n  # lbvh_gpu.rs:264-279
        # root box = union of every triangle box
        np.testing.assert_array_equal(lb.node_bounds[0, :3], lb.tri_bounds[:, :3].min(0))
        np.testing.assert_array_equal(lb.node_bounds[0, 3:], lb.tri_bounds[:, 3:].max(0))


def test_lbvh_duplicate_codes_and_quality():
    # Every triangle at the same place: all codes equal, the index tiebreak
    # still yields a valid tree (lbvh.rs:140-148).
    n = 64
    pos = np.zeros((3 * n, 4), np.float32)
    pos[1::3, 0] = 1.0
    pos[2::3, 1] = 1.0
    tris = np.zeros(n, O.TRIANGLE)
    tris["i0"], tris["i1"], tris["i2"] = np.arange(n) * 3, np.arange(n) * 3 + 1, np.arange(n) * 3 + 2
    lb = O.Lbvh(tris, pos)
    assert np.all(lb.codes == lb.codes[0])
    assert sorted(lb.prim_indices.tolist()) == list(range(n))
    assert np.array_equal(lb.order, np.arange(n))  # stable: equal keys keep input order


def test_lbvh_quality_vs_sah():  # lbvh_build.rs: quality ratio < 3x SAH
    tris, pos = _random_mesh(2000, 7)
    lb = O.Lbvh(tris, pos)
    nodes, prims, sah, problems = O.sah_build(tris, pos)
    assert problems == 0
    assert lb.sah_cost < 3.0 * sah


@pytest.mark.parametrize("n", [0, 1, 255, 256, 257, 5000])
def test_sort_pairs_is_stable(n):  # crates/gpu/tests/radix_sort.rs:35-122
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 16, n, dtype=np.uint32)  # many duplicates
    vals = np.arange(n, dtype=np.uint32)
    ko, vo = O.sort_pairs(keys, vals)
    order = np.lexsort((vals, keys))
    assert np.array_equal(ko, keys[order]) and np.array_equal(vo, vals[order])
