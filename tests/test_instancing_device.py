"""Device-built instancing (luc_upload_meshes + luc_set_instances) against
the oracle's restatement of the same build (Scene::build_instances_lbvh):
one LBVH per mesh, a TLAS by LBVH over the instances' world bounds, rebuilt
whenever the placements change.

Bit-exact: every BLAS and TLAS node, the triangles in leaf order, and the
instance rows (the adjugate inverse of each transform and the world bounds
are evaluated in the same operation order on both sides). Then renders of
the scene match the oracle's at the usual thresholds, before and after the
instances move.
"""
import numpy as np
import pytest

import lucida_b200 as lb
from lucida_b200 import scenes
from tests.bridge import oracle_from_scene, parity
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = lb.Gpu(0)
    yield g
    g.close()


def _small():
    return scenes.instanced_field(num_meshes=3, tri_range=(1000, 4000), num_instances=40, extent=(20.0, 4.0, 20.0),
                                  level=2, env_size=(64, 32))


def _words(a, k):
    return np.ascontiguousarray(a).view(np.uint32).reshape(-1, k)


def _same_arrays(gpu, osc):
    np.testing.assert_array_equal(_words(gpu.read_scene("nodes"), 8), _words(osc.array(O.W_BVH_NODES), 8))
    np.testing.assert_array_equal(_words(gpu.read_scene("triangles"), 4), _words(osc.array(O.W_TRIANGLES), 4))
    np.testing.assert_array_equal(_words(gpu.read_scene("primitives"), 16), _words(osc.array(O.W_PRIMITIVES), 16))


def _render_check(gpu, s, osc, label, ref_shadows=False):
    osc.set_reference_shadows(ref_shadows)
    u = osc.uniforms(64, 48, 8, 6, frame_seed=0x5EED1234, sampling=2, sampler=1)
    params = lb.RenderParams(width=64, height=48, samples=8, max_depth=6, sampling="mis", sampler="sobol")
    acc = lb.render_accum(gpu, s, params, uniforms=lb.layout.uniforms_from_bytes(bytes(u)),
                          reference_shadows=ref_shadows).reshape(-1)
    parity(acc["radiance"], osc, u, label)


def test_device_build_is_bit_exact_and_renders_match(gpu):
    s = _small()
    gpu.set_tlas_leaf(4)  # the reference's LBVH_MAX_LEAF: its node layout bit for bit
    gpu.upload(s, force=True)
    osc = oracle_from_scene(s)
    _same_arrays(gpu, osc)
    _render_check(gpu, s, osc, "instanced-field")
    _render_check(gpu, s, osc, "instanced-field/reference-shadows", ref_shadows=True)


@pytest.mark.parametrize("leaf", [1, 4, 8])
def test_ray_queries_match_the_oracle(gpu, leaf):
    """Closest hits of single rays (luc_intersect: the integrator's
    two-level walk, whole) against the oracle's Scene::intersect on its
    leaf-4 build: the same distance bit for bit, whichever TLAS the device
    walks (leaf 1 and 4: the 8-wide TLAS; leaf 8: the binary child pairs);
    and occlusion queries consistent with those distances."""
    s = _small()
    gpu.set_tlas_leaf(leaf)
    gpu.upload(s, force=True)
    osc = oracle_from_scene(s)
    rng = np.random.default_rng(31 + leaf)
    n = 20_000
    o = np.stack([rng.uniform(-12, 12, n), rng.uniform(0.2, 6, n), rng.uniform(-12, 12, n)], 1).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    t, _, _, ids = gpu.intersect(o, d)
    ref = osc.intersect(np.concatenate([o, d], 1))
    hit_ref = ref[:, 0] >= 0
    hit_dev = ids != 0xFFFFFFFF
    assert hit_ref.sum() > n // 4 and (~hit_ref).sum() > n // 20  # both kinds of ray occur
    same = (hit_ref == hit_dev) & (~hit_ref | (t.view(np.uint32) == ref[:, 0].view(np.uint32)))
    assert same.mean() >= 0.9999, same.mean()
    # Occluded within (1e-4, tmax) exactly when the nearest hit lies inside.
    tmax = np.where(hit_ref, ref[:, 0], 10.0).astype(np.float32)
    half = (0.5 * tmax).astype(np.float32)
    occ_half = gpu.intersect(o, d, half)
    occ_far = gpu.intersect(o, d, (tmax * 1.01 + 1e-3).astype(np.float32))
    clear = half > 1e-3
    assert np.mean(occ_half[clear] == False) >= 0.9999  # noqa: E712 — nothing nearer than the nearest hit
    assert np.mean(occ_far[hit_ref] == True) >= 0.9999  # noqa: E712 — the nearest hit itself occludes
    gpu.set_tlas_leaf(1)


@pytest.mark.parametrize("leaf", [1, 8])
def test_other_tlas_leaf_sizes_render_the_same(gpu, leaf):
    """TLASes other than the reference's (leaf size 4) differ in node layout
    but not in what a ray hits: the renders meet the same bar against the
    oracle's leaf-4 build. Leaf size 1 (the default) is walked through its
    8-wide collapse, leaf size 8 (too large for a wide leaf slot) through the
    binary child pairs."""
    s = _small()
    gpu.set_tlas_leaf(leaf)
    gpu.upload(s, force=True)
    osc = oracle_from_scene(s)
    if leaf == 1:
        tlas = gpu.read_scene("nodes")[-(2 * 40 - 1):]
        counts = tlas.view(np.uint32).reshape(-1, 8)[:, 7]
        assert counts.max() == 1  # every leaf holds one instance
    _render_check(gpu, s, osc, f"instanced-field/leaf-{leaf}")
    _render_check(gpu, s, osc, f"instanced-field/leaf-{leaf}/reference-shadows", ref_shadows=True)
    gpu.set_tlas_leaf(1)


def test_tlas_rebuild_after_the_instances_move(gpu):
    s = _small()
    gpu.set_tlas_leaf(4)
    gpu.upload(s, force=True)
    o2w, mesh, material = s.placements
    rng = np.random.default_rng(7)
    for step in range(3):
        moved = o2w.copy()
        moved[:, :, 3] += rng.uniform(-1.5, 1.5, (len(moved), 3)).astype(np.float32)
        keep = len(moved) - 7 * step  # fewer instances on later frames: the buffers keep their size
        s2 = lb.SceneDef(**{**s.__dict__, "placements": (moved[:keep], mesh[:keep], material[:keep])})
        gpu.set_instances(moved[:keep], mesh[:keep], material[:keep])
        gpu._scene = s2  # the resident scene is now s2; render_accum must not re-upload
        osc = oracle_from_scene(s2)
        _same_arrays(gpu, osc)
        _render_check(gpu, s2, osc, f"instanced-field/moved-{step}")


def test_set_instances_validation(gpu):
    s = _small()
    gpu.upload(s, force=True)
    o2w, mesh, material = s.placements
    with pytest.raises(lb.GpuError):
        gpu.set_instances(o2w[:2], np.array([0, 9], np.uint32))  # no such mesh
    bad = o2w[:1].copy()
    bad[0, :, :3] = 0.0  # singular
    with pytest.raises(lb.GpuError):
        gpu.set_instances(bad, mesh[:1])
    bad = o2w[:1].copy()
    bad[0, 0, 0] = np.nan
    with pytest.raises(lb.GpuError):
        gpu.set_instances(bad, mesh[:1])
    gpu.set_instances(o2w, mesh, material)  # still usable
