"""Compressed 8-wide BVH (wide.cu) collapsed on the device from the binary
tree, and its traversal (wide_trace in scene_dev.cuh).

Structure, decoded here from the device's own arrays: every triangle of the
leaf-order soup appears exactly once in the wide soup, with the same
(p0, p1 - p0, p2 - p0) values and its leaf-order index; every slot's
quantized box contains everything below it; nodes are reached once. Cases:
the device LBVH of a displaced-spheres scene, a caller-supplied SAH tree
with a 120-triangle leaf (coincident centroids), so leaf chunks chain, and a
one-triangle scene whose root is a leaf.

Traversal: renders through the wide tree equal renders through the binary
tree (LUC_BINARY_BVH=1) pixel for pixel, up to exactly tied triangle
distances, which the two traversals may break differently.
"""
import dataclasses
import os

import numpy as np
import pytest

import lucida_b200 as lb
from lucida_b200 import layout as L, scenes
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = lb.Gpu(0)
    yield g
    g.close()


@pytest.fixture(scope="module")
def gpu_binary():
    os.environ["LUC_BINARY_BVH"] = "1"
    try:
        g = lb.Gpu(0)
    finally:
        del os.environ["LUC_BINARY_BVH"]
    yield g
    g.close()


def _soup(tris, pos):
    p = pos[:, :3].astype(np.float32)
    p0, p1, p2 = p[tris["i0"]], p[tris["i1"]], p[tris["i2"]]
    return p0, p1 - p0, p2 - p0


def _decode(w):
    p = w[:, 0:3].view(np.float32).astype(np.float64)
    e = np.stack([(w[:, 3] >> (8 * a)) & 0xFF for a in range(3)], 1).astype(np.int64) - 127
    scale = np.ldexp(1.0, e)
    imask = w[:, 3] >> 24

    def bytes8(lo_word):
        b = w[:, lo_word:lo_word + 2].copy().view(np.uint8).reshape(-1, 8)
        return b.astype(np.float64)
    qlo = np.stack([bytes8(8), bytes8(10), bytes8(12)], 1)   # (n, 3, 8)
    qhi = np.stack([bytes8(14), bytes8(16), bytes8(18)], 1)
    lo = p[:, :, None] + qlo * scale[:, :, None]
    hi = p[:, :, None] + qhi * scale[:, :, None]
    return dict(cbase=w[:, 4], tbase=w[:, 5], imask=imask, cntmask=w[:, 6], lo=lo, hi=hi)


def _check_structure(g, tris_leaf_order, pos):
    wn = g.read_scene("wide_nodes")
    ws = g.read_scene("wide_soup")
    n = len(tris_leaf_order)
    assert len(wn) > 0 and len(ws) == n
    # The soup: a permutation of the leaf-order soup, values bit-identical.
    idx = ws[:, 3].view(np.uint32)
    assert np.array_equal(np.sort(idx), np.arange(n, dtype=np.uint32))
    p0, e1, e2 = _soup(tris_leaf_order, pos)
    assert np.array_equal(ws[:, 0:3], p0[idx]) and np.array_equal(ws[:, 4:7], e1[idx])
    assert np.array_equal(ws[:, 8:11], e2[idx])
    # Triangle bounds (float64) in wide-soup order.
    v0 = p0[idx].astype(np.float64)
    v1 = v0 + e1[idx].astype(np.float64)
    v2 = v0 + e2[idx].astype(np.float64)
    tlo = np.minimum(np.minimum(v0, v1), v2)
    thi = np.maximum(np.maximum(v0, v1), v2)
    d = _decode(wn)
    seen_nodes = np.zeros(len(wn), np.int32)
    seen_tris = np.zeros(n, np.int32)
    bad = []

    def visit(k):  # returns (lo, hi) of everything below wide node k
        seen_nodes[k] += 1
        lo_all = np.full(3, np.inf)
        hi_all = np.full(3, -np.inf)
        rank = 0
        for s in range(8):
            if d["imask"][k] >> s & 1:
                clo, chi = visit(int(d["cbase"][k]) + rank)
                rank += 1
            else:
                cm = int(d["cntmask"][k])
                nib = (cm >> (4 * s)) & 0xF
                cnt, off = bin(nib).count("1"), bin(cm & ((1 << (4 * s)) - 1)).count("1")
                if cnt == 0:
                    continue
                assert nib == (1 << cnt) - 1  # a slot's triangles are its nibble's low bits
                first = int(d["tbase"][k]) + off
                seen_tris[first:first + cnt] += 1
                clo = tlo[first:first + cnt].min(0)
                chi = thi[first:first + cnt].max(0)
            if not (np.all(d["lo"][k, :, s] <= clo) and np.all(d["hi"][k, :, s] >= chi)):
                bad.append((k, s))
            lo_all = np.minimum(lo_all, clo)
            hi_all = np.maximum(hi_all, chi)
        return lo_all, hi_all

    import sys
    sys.setrecursionlimit(10000)
    visit(0)
    assert not bad, bad[:5]
    assert np.all(seen_nodes == 1) and np.all(seen_tris == 1)
    return len(wn)


def test_device_lbvh_collapses(gpu):
    s = scenes.displaced_spheres(count=24, level=3, env_size=(64, 32))
    gpu.upload(s, force=True)
    tris = gpu.read_scene("triangles")
    nw = _check_structure(gpu, tris, s.positions)
    nb = len(gpu.read_scene("nodes"))
    print("binary nodes", nb, "wide nodes", nw)
    assert nw < nb // 3


def _sah_scene_with_big_leaf():
    s = scenes.displaced_spheres(count=6, level=2, env_size=(64, 32))
    tris = np.concatenate([s.triangles, np.repeat(s.triangles[:1], 120)])
    nodes, prims, _, problems = O.sah_build(tris.view(O.TRIANGLE), s.positions)
    assert problems == 0
    counts = nodes["count"]
    assert counts.max() >= 120  # the coincident copies share one leaf
    return dataclasses.replace(s, triangles=tris[prims], bvh_nodes=nodes.view(L.BVH_NODE))


def test_caller_tree_with_big_leaf_collapses(gpu):
    s = _sah_scene_with_big_leaf()
    gpu.upload(s, force=True)
    _check_structure(gpu, s.triangles, s.positions)


def test_single_triangle_root_leaf(gpu):
    s = scenes.displaced_spheres(count=1, level=0, env_size=(64, 32))
    s = dataclasses.replace(s, triangles=s.triangles[:1].copy())
    gpu.upload(s, force=True)
    _check_structure(gpu, gpu.read_scene("triangles"), s.positions)


def _case(case):
    if case == "lbvh":
        return scenes.displaced_spheres(count=24, level=3, env_size=(64, 32))
    if case == "sah_big_leaf":
        return _sah_scene_with_big_leaf()
    from tests.bridge import scene_from_oracle
    return scene_from_oracle(O.Scene.builtin("cornell-mesh"))  # SAH tree with leaves under the root


CASES = ["lbvh", "sah_big_leaf", "cornell_mesh"]


def _rays(s, n, seed):
    """Incoherent rays: origins uniform in the geometry's bounds, directions
    uniform on the sphere."""
    rng = np.random.default_rng(seed)
    p = s.positions[:, :3]
    lo, hi = p.min(0), p.max(0)
    o = (lo + (hi - lo) * rng.random((n, 3))).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    return o, d


@pytest.mark.parametrize("case", CASES)
def test_ray_queries_match_binary_traversal(gpu, gpu_binary, case):
    """Closest-hit distances bit-identical to the binary traversal's, the same
    triangle wherever the distance is not an exact tie, the same occlusion."""
    s = _case(case)
    gpu.upload(s)
    gpu_binary.upload(s)
    assert len(gpu.read_scene("wide_nodes")) > 0
    o, d = _rays(s, 200_000, 5)
    tw, uw, vw, iw = gpu.intersect(o, d)
    tb, ub, vb, ib = gpu_binary.intersect(o, d)
    hit = iw != 0xFFFFFFFF
    print(case, "hit fraction", hit.mean(), "id differs", (iw != ib).sum())
    assert 0.2 < hit.mean() and np.array_equal(iw == 0xFFFFFFFF, ib == 0xFFFFFFFF)
    assert np.array_equal(tw.view(np.uint32), tb.view(np.uint32))
    same = iw == ib
    assert same.mean() >= 0.9999
    assert np.array_equal(uw[same].view(np.uint32), ub[same].view(np.uint32))
    rng = np.random.default_rng(6)
    tmax = np.where(hit, tw * rng.uniform(0.5, 1.5, len(tw)), 1e4).astype(np.float32)
    assert np.array_equal(gpu.intersect(o, d, tmax), gpu_binary.intersect(o, d, tmax))


def test_ray_queries_match_oracle():
    """The caller's SAH tree through the wide traversal against the oracle's
    restatement of Scene::intersect on the same scene."""
    from tests.bridge import scene_from_oracle
    osc = O.Scene.builtin("cornell-mesh")
    s = scene_from_oracle(osc)
    g = lb.Gpu(0)
    try:
        g.upload(s)
        o, d = _rays(s, 50_000, 9)
        t, _, _, ids = g.intersect(o, d)
        ref = osc.intersect(np.concatenate([o, d], 1))
        t_ref = np.where(ref[:, 0] < 0, np.float32(1e30), ref[:, 0]).astype(np.float32)
        t_dev = np.where(ids == 0xFFFFFFFF, np.float32(1e30), t)
        assert np.mean(t_dev.view(np.uint32) == t_ref.view(np.uint32)) >= 0.9999
    finally:
        g.close()


@pytest.mark.parametrize("case", CASES)
def test_wide_and_binary_render_alike(gpu, gpu_binary, case):
    s = _case(case)
    p = lb.RenderParams(width=96, height=64, samples=4, max_depth=6, sampler="sobol")
    a = lb.render_accum(gpu, s, p).reshape(-1)
    sw = gpu.stats()
    b = lb.render_accum(gpu_binary, s, p).reshape(-1)
    sb = gpu_binary.stats()
    assert len(gpu.read_scene("wide_nodes")) > 0 and len(gpu_binary.read_scene("wide_nodes")) == 0
    same = np.all(a["radiance"] == b["radiance"], axis=-1)
    print(case, "identical pixels", same.mean(), "nodes/ray wide", sw.nodes_extend / max(1, sw.rays_extend),
          "binary", sb.nodes_extend / max(1, sb.rays_extend), "tris/ray wide", sw.tris_extend / max(1, sw.rays_extend),
          "binary", sb.tris_extend / max(1, sb.rays_extend))
    assert same.mean() >= 0.999
    assert abs(int(sw.rays_extend) - int(sb.rays_extend)) <= 0.001 * sb.rays_extend
