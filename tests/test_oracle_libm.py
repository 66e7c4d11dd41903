"""The oracle's two transcendental roundings and its per-sample path traces
(CPU only).

The parity bar (tests.bridge.parity) compares a device render with the
oracle run two ways: glibc's f32 functions (the reference's) and double
evaluation rounded once (the device's). These tests pin what that relies on:
the two roundings are one algorithm (renders agree far inside 1e-3), a
per-sample trace sums to the render exactly, and a path signature changes
when, and only when, the path's branches change.
"""
import numpy as np

import oracle as O
import lucida_b200 as lb
from lucida_b200 import scenes
from tests.bridge import compare, oracle_from_scene


def _uniforms(osc, w, h, spp, depth, sampler="independent"):
    return osc.uniforms(w, h, spp, depth, frame_seed=0x5EED1234, sampling=lb.layout.SAMPLING["mis"],
                        sampler=lb.layout.SAMPLER[sampler])


def test_libm_modes_are_one_algorithm():
    osc = oracle_from_scene(scenes.cornell_analytic())
    u = _uniforms(osc, 64, 64, 8, 8)
    g = osc.render_sums(u)
    d = osc.render_sums(u, libm="double")
    st = compare(g[:, 0:3], d[:, 0:3])
    assert 0.5 < st["bit_exact"] < 1.0, st  # the roundings differ, on a minority of pixels
    assert st["max_rel"] < 1e-4 and st["mean_rel"] < 1e-7, st
    assert np.array_equal(g[:, 6:13], d[:, 6:13])  # first-hit guides take no transcendental
    # The mode is restored after each call.
    assert np.array_equal(osc.render_sums(u), g)


def test_traces_sum_to_the_render():
    for name, sampler in (("cornell-box", "sobol"), ("sunset", "sobol"), ("glass-box", "independent")):
        osc = O.Scene.builtin(name)
        u = _uniforms(osc, 32, 24, 6, 6, sampler)
        sums = osc.render_sums(u)
        pixels = np.arange(0, 32 * 24, 7)
        for libm in ("glibc", "double"):
            rad, sig = osc.sample_traces(u, pixels, libm=libm)
            acc = np.zeros((len(pixels), 3), np.float32)
            for k in range(u.samples_per_launch):  # sample order, f32, as the render adds them
                acc += rad[:, k]
            ref = sums if libm == "glibc" else osc.render_sums(u, libm="double")
            assert np.array_equal(acc, ref[pixels, 0:3]), (name, libm)
            assert np.all(sig != 0)
            _, again = osc.sample_traces(u, pixels, libm=libm)
            assert np.array_equal(again, sig)  # deterministic


def test_signature_tracks_branches():
    """Signatures of one sample agree between the two roundings on nearly
    every sample (same branches), and a planted change to the scene's
    geometry (one sphere moved by 1e-3) changes the signatures of some
    samples, but far from all."""
    s = scenes.cornell_analytic()
    osc = oracle_from_scene(s)
    u = _uniforms(osc, 48, 48, 4, 8)
    pixels = np.arange(48 * 48)
    rg, sg = osc.sample_traces(u, pixels)
    rd, sd = osc.sample_traces(u, pixels, libm="double")
    same = sg == sd
    assert same.mean() > 0.999
    # Where the branches agree the radiance agrees to rounding.
    a, b = rg[same].astype(np.float64), rd[same].astype(np.float64)
    assert np.max(np.abs(a - b) / (np.abs(a) + np.abs(b) + 1e-4)) < 1e-3
    moved = s.primitives.copy()
    k = int(np.nonzero(moved["kind"] == lb.layout.PRIM_KIND_SPHERE)[0][0])
    moved["position"][k, 0] += 1e-3
    s2 = lb.SceneDef(materials=s.materials, primitives=moved, lights=s.lights, positions=s.positions,
                     vertex_attrs=s.vertex_attrs, triangles=s.triangles, camera=s.camera,
                     background=s.background)
    r2, s2sig = oracle_from_scene(s2).sample_traces(u, pixels)
    changed = s2sig != sg
    assert 0 < changed.mean() < 0.5
