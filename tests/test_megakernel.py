"""Megakernel architecture (luc_render with LUC_ARCH_MEGAKERNEL) against the
wavefront (crates/gpu/tests/wavefront_agreement.rs:43-84 checks the two to
8e-9; here they share one shade_vertex and the wavefront's accumulation
order, so the accumulators must be identical bit for bit), and against the
oracle (cpu_gpu_agreement.rs:39-80, megakernel_matches_the_cpu_reference).
"""
import numpy as np
import pytest

import lucida_b200 as lb
from lucida_b200 import scenes
import oracle as O
from tests.bridge import parity, scene_from_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = lb.Gpu(0)
    yield g
    g.close()


def _both(gpu, s, p, **kw):
    w = lb.render_accum(gpu, s, p, architecture="wavefront", **kw).reshape(-1)
    sw = gpu.stats()
    m = lb.render_accum(gpu, s, p, architecture="megakernel", **kw).reshape(-1)
    sm = gpu.stats()
    return w, m, sw, sm


@pytest.mark.parametrize("name", ["cornell-box", "glass-box", "sunset", "metal-sweep", "cornell-mesh", "mis-scene",
                                  "furnace-test"])
@pytest.mark.parametrize("mode", ["mis", "nee", "bsdf"])
def test_megakernel_equals_wavefront(gpu, name, mode):
    s = scene_from_oracle(O.Scene.builtin(name))
    for sampler in ("sobol", "independent"):
        p = lb.RenderParams(width=64, height=48, samples=6, max_depth=7, sampler=sampler, sampling=mode,
                            frame_seed=0x5EED1234, sample_offset=3)
        w, m, sw, sm = _both(gpu, s, p)
        assert w.tobytes() == m.tobytes(), (name, mode, sampler)
        assert (sw.rays_extend, sw.rays_shadow, sw.nodes_extend, sw.tris_extend, sw.nodes_shadow) == \
               (sm.rays_extend, sm.rays_shadow, sm.nodes_extend, sm.tris_extend, sm.nodes_shadow)
        assert sm.paths == sw.paths == 64 * 48 * 6 and sm.launches == 2  # one walk + RESOLVE


def test_megakernel_on_triangle_workload_and_instances(gpu):
    s = scenes.displaced_spheres(count=24, level=3, env_size=(128, 64))
    p = lb.RenderParams(width=80, height=60, samples=4, max_depth=8)
    w, m, _, _ = _both(gpu, s, p)
    assert w.tobytes() == m.tobytes()
    inst = scenes.instanced_field(num_meshes=3, tri_range=(1000, 4000), num_instances=40,
                                  extent=(20.0, 4.0, 20.0), level=2, env_size=(64, 32))
    for ref_shadows in (False, True):
        w, m, _, _ = _both(gpu, inst, p, reference_shadows=ref_shadows)
        assert w.tobytes() == m.tobytes(), ref_shadows


def test_megakernel_matches_the_oracle(gpu):
    osc = O.Scene.builtin("cornell-box")
    s = scene_from_oracle(osc)
    u = osc.uniforms(64, 48, 16, 8, frame_seed=0x5EED1234, sampling=2, sampler=0)
    acc = lb.render_accum(gpu, s, lb.RenderParams(width=64, height=48, samples=16, max_depth=8),
                          uniforms=lb.layout.uniforms_from_bytes(bytes(u)), architecture="megakernel").reshape(-1)
    parity(acc["radiance"], osc, u, "megakernel/cornell-box")


def test_megakernel_rejects_the_guide(gpu):
    s = scene_from_oracle(O.Scene.builtin("cornell-box"))
    with pytest.raises(lb.GpuError):
        lb.render_accum(gpu, s, lb.RenderParams(width=8, height=8, samples=1, max_depth=2), guided=True,
                        architecture="megakernel")
