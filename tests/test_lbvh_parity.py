"""The device LBVH builder and radix sort against the oracle, stage by stage
and bit for bit (crates/gpu/tests/lbvh_gpu.rs, radix_sort.rs). On CUDA with
IEEE division and no contraction the Morton codes are exact, so the sort
order, the Karras topology, the fitted boxes and the relaid-out tree must be
identical to the CPU builder's."""
import numpy as np
import pytest

import oracle as O
import lucida_b200 as lb
from lucida_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = lb.Gpu(0)
    yield g
    g.close()


def _mesh(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-50, 50, (n, 3)).astype(np.float32)
    pos = np.zeros((3 * n, 4), np.float32)
    for k in range(3):
        pos[k::3, :3] = c + rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    t = np.zeros(n, O.TRIANGLE)
    t["i0"], t["i1"], t["i2"] = np.arange(n) * 3, np.arange(n) * 3 + 1, np.arange(n) * 3 + 2
    return t, pos


def _compare(gpu_out, ref, n):
    assert np.array_equal(gpu_out.codes, ref.codes), "morton codes"
    assert np.array_equal(gpu_out.order, ref.order), "sort order"
    if n > 1:
        assert np.array_equal(gpu_out.karras, ref.karras), "karras topology"
        assert np.array_equal(gpu_out.parent, ref.parent), "parents"
        assert np.array_equal(gpu_out.subtree_size, ref.subtree_size), "subtree sizes"
        assert np.array_equal(gpu_out.node_bounds, ref.node_bounds), "fitted bounds"
    assert np.array_equal(gpu_out.scene_bounds, ref.centroid_bounds.reshape(-1)), "centroid bounds"
    assert len(gpu_out.nodes) == len(ref.nodes), "node count"
    assert gpu_out.nodes.tobytes() == ref.nodes.tobytes(), "relaid-out tree"
    assert np.array_equal(gpu_out.prim_indices, ref.prim_indices), "leaf primitive order"


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 17, 255, 256, 257, 4095, 4096, 4097, 10000, 100000])
def test_lbvh_random_meshes(gpu, n):
    t, p = _mesh(n, n)
    _compare(lb.LbvhBuilder(gpu).build_parts(t, p), O.Lbvh(t, p), n)


def test_lbvh_duplicate_codes(gpu):
    n = 3000
    t, p = _mesh(n, 1)
    p[:, :3] = np.round(p[:, :3] / 20.0) * 20.0  # heavy code collisions
    _compare(lb.LbvhBuilder(gpu).build_parts(t, p), O.Lbvh(t, p), n)


def test_lbvh_reference_scene_and_config_mesh(gpu):
    osc = O.Scene.builtin("cornell-mesh")
    t, p = osc.array(O.W_TRIANGLES), osc.array(O.W_POSITIONS)
    _compare(lb.LbvhBuilder(gpu).build_parts(t, p), O.Lbvh(t, p), len(t))
    s = scenes.displaced_spheres(count=16, level=3)
    _compare(lb.LbvhBuilder(gpu).build_parts(s.triangles, s.positions), O.Lbvh(s.triangles, s.positions),
             len(s.triangles))


def test_lbvh_over_boxes_tlas(gpu):
    rng = np.random.default_rng(3)
    lo = rng.uniform(-100, 100, (4096, 3)).astype(np.float32)
    boxes = np.concatenate([lo, lo + rng.uniform(0.5, 4, (4096, 3)).astype(np.float32)], 1)
    _compare(lb.LbvhBuilder(gpu).build_boxes(boxes), O.Lbvh(boxes=boxes), 4096)


@pytest.mark.parametrize("n,hi", [(0, 16), (1, 16), (255, 16), (256, 2**32), (257, 2**32), (4097, 7),
                                  (100000, 2**32), (1 << 20, 2**32)])
def test_radix_sort_matches_stable_sort(gpu, n, hi):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, hi, n, dtype=np.uint64).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    ko, vo = lb.LbvhBuilder(gpu).sort(keys, vals)
    rk, rv = O.sort_pairs(keys, vals)
    assert np.array_equal(ko, rk) and np.array_equal(vo, rv)


def test_radix_sort_adversarial(gpu):
    n = 50000
    for keys in (np.full(n, 0xFFFFFFFF, np.uint32), np.arange(n, dtype=np.uint32)[::-1].copy(),
                 (np.arange(n, dtype=np.uint32) << 24)):
        vals = np.arange(n, dtype=np.uint32)
        ko, vo = lb.LbvhBuilder(gpu).sort(keys, vals)
        rk, rv = O.sort_pairs(keys, vals)
        assert np.array_equal(ko, rk) and np.array_equal(vo, rv)


def test_lbvh_render_matches_sah_render(gpu):
    """An acceleration structure changes speed, not the picture: the device
    LBVH (triangles compacted into its leaf order) renders the same image as
    the oracle's SAH tree (scene.rs BvhBuilder note)."""
    from tests.bridge import oracle_from_scene, parity
    s = scenes.displaced_spheres(count=24, level=3, env_size=(256, 128))
    osc = oracle_from_scene(s)
    u = osc.uniforms(64, 48, 4, 5, sampler=1)
    acc = lb.render_accum(gpu, s, lb.RenderParams(width=64, height=48, samples=4, max_depth=5),
                          uniforms=lb.layout.uniforms_from_bytes(bytes(u))).reshape(-1)
    parity(acc["radiance"], osc, u, "lbvh vs sah")
