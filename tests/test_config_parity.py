"""Parity at the benchmark configurations' own sizes.

* Analytic Cornell box exactly as configured: 512 x 512, 64 spp, 8 bounces,
  independent PCG streams, NEE + MIS, through both architectures
  (wavefront and megakernel) — 16.8M paths per render, every pixel held to
  the per-pixel bar of tests.bridge.parity.
* The full 1,310,720-triangle displaced-spheres scene (256 level-4 icospheres
  under the 1024 x 512 sky) and the full guided-room geometry, each with its
  tree built by the device LBVH, against the oracle on the reference's own
  binned-SAH tree (scene.rs:227-239), at 128 x 128 x 2 spp, 8 bounces.
* The instanced field (16 meshes, 3.03M triangles, 4096 instances; BLASes
  and TLAS built on the device by LBVH) against the oracle's restatement of
  that build, 12 bounces.
* The LBVH stage by stage, bit for bit, at the sizes the renders build: the
  1,310,720-triangle scene and the instanced field's largest mesh.
"""
import numpy as np
import pytest

import oracle as O
import lucida_b200 as lb
from lucida_b200 import scenes
from tests.bridge import oracle_from_scene, parity
from tests.test_lbvh_parity import _compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = lb.Gpu(0)
    yield g
    g.close()


@pytest.fixture(scope="module")
def cornell_c1():
    """The oracle's two renders of the analytic Cornell box as configured,
    shared by both architectures' tests."""
    s = scenes.cornell_analytic()
    osc = oracle_from_scene(s)
    u = osc.uniforms(512, 512, 64, 8, frame_seed=0x5EED1234, sampling=lb.layout.SAMPLING["mis"],
                     sampler=lb.layout.SAMPLER["independent"])
    return s, osc, u, osc.render_sums(u), osc.render_sums(u, libm="double")


@pytest.mark.parametrize("arch", ["wavefront", "megakernel"])
def test_cornell_box_full_config(gpu, cornell_c1, arch):
    s, osc, u, ref_g, ref_d = cornell_c1
    params = lb.RenderParams(width=512, height=512, samples=64, max_depth=8, sampler="independent")
    acc = lb.render_accum(gpu, s, params, uniforms=lb.layout.uniforms_from_bytes(bytes(u)),
                          architecture=arch).reshape(-1)
    assert np.all(acc["samples"] == 64)
    parity(acc["radiance"], osc, u, f"cornell-box 512x512x64 d8 {arch}", ref_glibc=ref_g, ref_double=ref_d)


@pytest.mark.parametrize("which", ["displaced-spheres", "guided-room"])
def test_full_triangle_scenes(gpu, which):
    s = scenes.displaced_spheres() if which == "displaced-spheres" else scenes.guided_room()
    assert len(s.triangles) == 1_310_720 or which == "guided-room"
    osc = oracle_from_scene(s)  # the reference's binned-SAH tree
    u = osc.uniforms(128, 128, 2, 8, frame_seed=0x5EED1234, sampling=lb.layout.SAMPLING["mis"],
                     sampler=lb.layout.SAMPLER["sobol"])
    params = lb.RenderParams(width=128, height=128, samples=2, max_depth=8)
    acc = lb.render_accum(gpu, s, params, uniforms=lb.layout.uniforms_from_bytes(bytes(u))).reshape(-1)
    parity(acc["radiance"], osc, u, f"{which} full geometry ({len(s.triangles)} triangles), device LBVH")


def test_instanced_field_full_geometry(gpu):
    s = scenes.instanced_field()
    osc = oracle_from_scene(s)  # restated device build: per-mesh LBVH BLASes, LBVH TLAS
    u = osc.uniforms(96, 54, 1, 12, frame_seed=0x5EED1234, sampling=lb.layout.SAMPLING["mis"],
                     sampler=lb.layout.SAMPLER["sobol"])
    params = lb.RenderParams(width=96, height=54, samples=1, max_depth=12)
    acc = lb.render_accum(gpu, s, params, uniforms=lb.layout.uniforms_from_bytes(bytes(u))).reshape(-1)
    parity(acc["radiance"], osc, u, f"instanced field ({len(s.triangles)} triangles, 4096 instances)")


def test_lbvh_bit_exact_at_benchmark_sizes(gpu):
    s = scenes.displaced_spheres(env_size=(0, 0))
    n = len(s.triangles)
    assert n == 1_310_720
    _compare(lb.LbvhBuilder(gpu).build_parts(s.triangles, s.positions), O.Lbvh(s.triangles, s.positions), n)
    field = scenes.instanced_field(env_size=(0, 0))
    first, count = max(((int(f), int(c)) for f, c in field.meshes), key=lambda m: m[1])
    assert count > 400_000
    tris = field.triangles[first:first + count]
    _compare(lb.LbvhBuilder(gpu).build_parts(tris, field.positions), O.Lbvh(tris, field.positions), count)
