"""The CUDA wavefront integrator against the oracle, per pixel.

Both sides trace the same scene with the same uniforms (camera, seed,
sampler) and the same counter-seeded streams, so they agree to float
rounding rather than to Monte Carlo noise (crates/gpu/tests/
cpu_gpu_agreement.rs pattern). The accumulators are compared directly
(radiance sums in sample order, no 1/spp).

Tolerance (tests.bridge.parity): per-pixel relative error <= 1e-3 on every
pixel against the oracle whose transcendentals round like the device's
(double evaluation, one rounding); against the oracle with glibc's f32
functions (the reference's), the reference's metrics (mean relative error
< 1e-4 where cpu_gpu_agreement.rs:83-87 asserts < 2e-3, energy within
1e-4, >= 99.9% of pixels within 1e-3), every pixel beyond 1e-3 explained by
the libm rounding alone and classified as a path flip or an amplified
rounding from the oracle's per-sample path signatures.
"""
import numpy as np
import pytest

import oracle as O
import lucida_b200 as lb
from lucida_b200 import scenes
from tests.bridge import oracle_from_scene, parity, scene_from_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = lb.Gpu(0)
    yield g
    g.close()


def _render_both(gpu, osc, width, height, spp, depth, sampling="mis", sampler="sobol", seed=0x5EED1234,
                 scene=None, offset=0):
    s = scene if scene is not None else scene_from_oracle(osc)
    u = osc.uniforms(width, height, spp, depth, frame_seed=seed, sample_offset=offset,
                     sampling=lb.layout.SAMPLING[sampling], sampler=lb.layout.SAMPLER[sampler])
    params = lb.RenderParams(width=width, height=height, samples=spp, max_depth=depth, frame_seed=seed,
                             sample_offset=offset, sampling=sampling, sampler=sampler)
    acc = lb.render_accum(gpu, s, params, uniforms=lb.layout.uniforms_from_bytes(bytes(u)))
    return acc.reshape(-1), u


def _check(acc, osc, u, label, ref=None):
    return parity(acc["radiance"], osc, u, label, ref_glibc=ref)


@pytest.mark.parametrize("sampler", ["independent", "sobol"])
def test_cornell_analytic_config(gpu, sampler):
    s = scenes.cornell_analytic()
    osc = oracle_from_scene(s)
    acc, u = _render_both(gpu, osc, 96, 96, 16, 8, sampler=sampler, scene=s)
    ref = osc.render_sums(u)
    _check(acc, osc, u, f"cornell-analytic/{sampler}", ref)
    # The guide channels (first-hit albedo/normal/depth sums) follow the same streams.
    np.testing.assert_allclose(acc["albedo"].reshape(-1, 3), ref[:, 6:9], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(acc["depth"].reshape(-1), ref[:, 12], rtol=1e-5, atol=1e-5)
    assert np.all(acc["samples"] == 16)


@pytest.mark.parametrize("name", ["cornell-box", "furnace-test", "glass-box", "mis-scene", "metal-sweep",
                                  "sunset", "cornell-mesh"])
@pytest.mark.parametrize("mode", ["bsdf", "nee", "mis"])
def test_reference_scenes(gpu, name, mode):
    osc = O.Scene.builtin(name)
    acc, u = _render_both(gpu, osc, 64, 48, 8, 6, sampling=mode)
    _check(acc, osc, u, f"{name}/{mode}")


@pytest.mark.parametrize("which", ["displaced-spheres", "guided-room"])
def test_triangle_workload_scenes(gpu, which):
    """The throughput and path-guiding workloads at reduced size (24 meshes,
    subdivision 3): the device's own LBVH against the oracle's SAH tree,
    plain MIS render with the Sobol sampler."""
    if which == "displaced-spheres":
        s = scenes.displaced_spheres(count=24, level=3, env_size=(256, 128))
    else:
        s = scenes.guided_room(count=24, level=3)
    osc = oracle_from_scene(s)
    acc, u = _render_both(gpu, osc, 64, 48, 8, 8, scene=s)
    _check(acc, osc, u, which)


@pytest.mark.parametrize("mode", ["bsdf", "nee", "mis"])
@pytest.mark.parametrize("shadows", ["two-level", "reference"])
def test_instanced_scene(gpu, mode, shadows):
    """The reference's instance-forest (one BLAS, 49 rotated and non-uniformly
    scaled instances under a TLAS, material overrides): two-level closest hit
    and shading, and shadow rays either through the two levels (the default)
    or as the reference casts them (LUC_FLAG_REFERENCE_SHADOWS)."""
    osc = O.Scene.builtin("instance-forest")
    ref_shadows = shadows == "reference"
    osc.set_reference_shadows(ref_shadows)
    s = scene_from_oracle(osc)
    u = osc.uniforms(64, 48, 8, 6, frame_seed=0x5EED1234, sampling=lb.layout.SAMPLING[mode],
                     sampler=lb.layout.SAMPLER["sobol"])
    params = lb.RenderParams(width=64, height=48, samples=8, max_depth=6, sampling=mode, sampler="sobol")
    acc = lb.render_accum(gpu, s, params, uniforms=lb.layout.uniforms_from_bytes(bytes(u)),
                          reference_shadows=ref_shadows).reshape(-1)
    _check(acc, osc, u, f"instance-forest/{mode}/{shadows}")


def test_instanced_shadow_modes_differ(gpu):
    """The two shadow-ray behaviours are really different on this scene (the
    reference's untransformed mesh sits at the origin, the instances cast real
    shadows), so the mode test above compares two distinct images."""
    osc = O.Scene.builtin("instance-forest")
    s = scene_from_oracle(osc)
    params = lb.RenderParams(width=64, height=48, samples=16, max_depth=4, sampling="nee", sampler="sobol")
    a = lb.render_accum(gpu, s, params)["radiance"]
    b = lb.render_accum(gpu, s, params, reference_shadows=True)["radiance"]
    assert np.mean(np.any(a != b, axis=-1)) > 0.05
    assert b.sum() > a.sum()  # fewer blockers in the reference's shadow rays


def test_progressive_equals_one_shot(gpu):
    """Accumulating 4 + 4 samples into one device accumulator equals one 8-sample
    render bit for bit (cpu_gpu_agreement.rs:119-168 asks < 1e-5)."""
    import torch
    s = scenes.cornell_analytic()
    gpu.upload(s)
    p = lb.RenderParams(width=64, height=64, samples=8, max_depth=6, sampler="sobol")
    one = lb.render_accum(gpu, s, p)
    dev = torch.zeros(64 * 64 * 16, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    from lucida_b200.native import lib, check
    import ctypes as C
    for off in (0, 4):
        u = lb.build_uniforms(s, lb.RenderParams(width=64, height=64, samples=4, max_depth=6, sampler="sobol",
                                                 sample_offset=off))
        check(gpu.handle, lib().luc_render(gpu.handle, C.byref(u), 4, 6, 0, None, C.c_void_p(dev.data_ptr())))
    prog = dev.cpu().numpy().view(lb.layout.ACCUM).reshape(64, 64)
    assert np.array_equal(prog["radiance"], one["radiance"])
    assert np.all(prog["samples"] == 8)


@pytest.mark.parametrize("depth", [1, 2, 4, 8, 16])
def test_agreement_across_path_lengths(gpu, depth):
    """cpu_gpu_agreement.rs:93-117: cornell-box at max_depth 1, 2, 4, 8, 16."""
    osc = O.Scene.builtin("cornell-box")
    acc, u = _render_both(gpu, osc, 48, 48, 8, depth)
    _check(acc, osc, u, f"depth {depth}")


def test_deep_dielectric_paths(gpu):
    """cpu_gpu_agreement.rs:521-569: glass-box at max_depth 24."""
    osc = O.Scene.builtin("glass-box")
    acc, u = _render_both(gpu, osc, 64, 48, 8, 24)
    _check(acc, osc, u, "glass-box d24")


def test_empty_primitive_arrays(gpu):
    """cpu_gpu_agreement.rs:174-198: cornell-box without its analytic
    primitives (lights and all) renders and agrees with the oracle."""
    osc = O.Scene.builtin("cornell-box")
    s = scene_from_oracle(osc)
    empty = lb.SceneDef(materials=s.materials, primitives=s.primitives[:0], lights=s.lights[:0],
                        positions=s.positions, vertex_attrs=s.vertex_attrs, triangles=s.triangles,
                        camera=s.camera, background=s.background)
    bare = O.Scene.from_arrays(s.materials.view(O.MATERIAL), s.primitives[:0].view(O.PRIMITIVE), s.positions,
                               s.vertex_attrs.view(O.VERTEX_ATTR), s.triangles.view(O.TRIANGLE),
                               lights=s.lights[:0].view(O.LIGHT), background=s.background,
                               camera=dict(eye=s.camera.eye, look_at=s.camera.look_at, vfov_deg=s.camera.vfov_deg,
                                           up=s.camera.up, aperture=s.camera.aperture,
                                           focus_distance=s.camera.focus_distance), bvh="sah")
    acc, u = _render_both(gpu, bare, 48, 48, 8, 3, scene=empty)
    ref = bare.render_sums(u)
    assert np.array_equal(acc["radiance"], ref[:, 0:3].reshape(acc["radiance"].shape))


def test_furnace_spheres_invisible(gpu):
    """cpu_gpu_agreement.rs:347-375: in the white furnace the energy-
    conserving metal spheres vanish: mean radiance 1 within 3e-3 at 24
    bounces (the reference's 160x80, 512 spp)."""
    s = scene_from_oracle(O.Scene.builtin("furnace-test"))
    f = lb.render_with(gpu, s, lb.RenderParams(width=160, height=80, samples=512, max_depth=24))
    assert np.all(np.isfinite(f.data))
    mean = float(f.data[..., 0].astype(np.float64).mean())
    print("furnace mean", mean, "worst", float(np.abs(f.data[..., 0] - 1.0).max()))
    assert abs(mean - 1.0) < 3e-3


def test_depth_sweep_energy_monotone(gpu):
    """integrator.rs:803-833: raising the bounce limit only adds energy."""
    s = scenes.cornell_analytic()
    means = []
    for d in range(1, 7):
        f = lb.render_with(gpu, s, lb.RenderParams(width=48, height=48, samples=16, max_depth=d))
        means.append(float(f.data.mean()))
    assert all(b >= a - 1e-5 for a, b in zip(means, means[1:])), means


def test_profiled_renders_time_every_stage(gpu):
    """LUC_FLAG_PROFILE on the captured-graph path (event-record nodes) and on
    the batched path: stage times are filled in and the image is unchanged."""
    s = scenes.cornell_analytic()
    params = lb.RenderParams(width=64, height=64, samples=4, max_depth=4, sampler="independent")
    plain = lb.render_accum(gpu, s, params)
    for _ in range(2):  # capture, then replay
        prof = lb.render_accum(gpu, s, params, profile=True)
        st = gpu.stats()
        assert np.array_equal(prof["radiance"], plain["radiance"])
        assert st.ms_generate > 0 and st.ms_extend > 0 and st.ms_shade > 0 and st.ms_resolve > 0
        assert st.ms_total >= st.ms_extend + st.ms_shade
    from lucida_b200 import Guide
    guide = Guide(gpu, seed=1)
    guide.configure(train=True, records_per_step=4096)
    for _ in range(2):
        lb.render_accum(gpu, s, params, profile=True, guided=True)
        st = gpu.stats()
        assert st.ms_guide > 0 and st.ms_train > 0 and st.ms_shade > 0
    assert guide.stats().steps == 2
