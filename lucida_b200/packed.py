"""Packed scene assets: the reference's pre-packed binary scene format.

The reference ships its scenes to the browser as one blob per scene
(`web/public/scenes/<name>.bin`) plus a generated manifest entry
(`web/src/generated/scenes.ts`) giving each section's byte offset and
element count, the camera, the background, the environment size and the
instancing counts (crates/cli/src/bin/codegen.rs:433-487, 536-640). The
blob is the SceneBlob arrays in a fixed order, each section starting on a
16-byte boundary (zero padding):

    materials (80 B), primitives (64 B; instance rows appended), lights
    (64 B), positions (16 B), vertexAttrs (32 B), triangles (16 B, SAH-leaf
    order), bvhNodes (32 B), envRadiance (16 B), envCdf (4 B; rows 0..h-1 the
    conditionals, row h the marginal, width max(w + 1, h + 1))

    scene = load(blob_bytes, entry)              # -> SceneDef, caller's SAH tree kept
    blob, entry = pack(scene)                    # the same format back
    entries = parse_manifest(open(".../scenes.ts").read())

`load` hands the reference's own SAH tree to the library (luc_upload_scene
traverses it as given, collapsed to the wide tree on the device).
"""
from __future__ import annotations

import re

import numpy as np

from . import layout as L
from .gpu import Camera, SceneDef

ALIGN = 16
SECTIONS = [("materials", L.MATERIAL), ("primitives", L.PRIMITIVE), ("lights", L.LIGHT),
            ("positions", np.dtype((np.float32, 4))), ("vertexAttrs", L.VERTEX_ATTR), ("triangles", L.TRIANGLE),
            ("bvhNodes", L.BVH_NODE), ("envRadiance", np.dtype((np.float32, 4))), ("envCdf", np.dtype(np.float32))]


def parse_manifest(text: str) -> dict:
    """The generated TypeScript manifest (codegen.rs:536-640) -> {name: entry}.
    An entry holds asset, byteLength, remote, sections {name: (byteOffset,
    count)}, instancing (count, analyticPrimitives, tlasRoot), env (width,
    height, totalWeight), background and camera."""
    scenes = {}
    for block in re.split(r"\n  \{\n", text)[1:]:
        name = re.search(r'name: "([^"]+)"', block).group(1)
        rec = {"asset": re.search(r'asset: "([^"]+)"', block).group(1),
               "byteLength": int(re.search(r"byteLength: (\d+)", block).group(1)),
               "remote": "remote: null" not in block, "sections": {}}
        for s, _ in SECTIONS:
            m = re.search(r"%s: \{ byteOffset: (\d+), count: (\d+) \}" % s, block)
            rec["sections"][s] = (int(m.group(1)), int(m.group(2)))
        inst = re.search(r"instancing: \{ count: (\d+), analyticPrimitives: (\d+), tlasRoot: (\d+) \}", block)
        rec["instancing"] = [int(inst.group(i)) for i in (1, 2, 3)]
        env = re.search(r"env: \{ width: (\d+), height: (\d+), totalWeight: ([-0-9.e+]+) \}", block)
        rec["env"] = [int(env.group(1)), int(env.group(2)), float(env.group(3))]
        bg = re.search(r"background: \[([^\]]*)\]", block).group(1)
        rec["background"] = [float(x) for x in bg.split(",")]
        cam = re.search(r"camera: \{ eye: \[([^\]]*)\], lookAt: \[([^\]]*)\], up: \[([^\]]*)\], "
                        r"vfovDeg: ([-0-9.e]+), aperture: ([-0-9.e]+), focusDistance: ([-0-9.e]+) \}", block)
        rec["camera"] = {"eye": [float(x) for x in cam.group(1).split(",")],
                         "look_at": [float(x) for x in cam.group(2).split(",")],
                         "up": [float(x) for x in cam.group(3).split(",")],
                         "vfov_deg": float(cam.group(4)), "aperture": float(cam.group(5)),
                         "focus_distance": float(cam.group(6))}
        scenes[name] = rec
    return scenes


def _arrays(scene: SceneDef) -> dict:
    w, h = scene.env_size
    cdf = np.zeros(0, np.float32)
    if w:
        cw = max(w + 1, h + 1)
        cdf = np.zeros((h + 1, cw), np.float32)
        cdf[:, :scene.env_cdf.shape[1]] = scene.env_cdf[:h + 1, :cw]
    return {"materials": scene.materials, "primitives": scene.primitives, "lights": scene.lights,
            "positions": np.asarray(scene.positions, np.float32).reshape(-1, 4),
            "vertexAttrs": scene.vertex_attrs, "triangles": scene.triangles,
            "bvhNodes": scene.bvh_nodes if scene.bvh_nodes is not None else np.zeros(0, L.BVH_NODE),
            "envRadiance": (np.asarray(scene.env_pixels, np.float32).reshape(-1, 4) if w
                            else np.zeros((0, 4), np.float32)),
            "envCdf": cdf.reshape(-1)}


def pack(scene: SceneDef) -> tuple[bytes, dict]:
    """SceneDef -> (blob, manifest entry) in codegen.rs's layout (pack_scene)."""
    arrays = _arrays(scene)
    out = bytearray()
    sections = {}
    for name, dt in SECTIONS:
        a = np.ascontiguousarray(arrays[name])
        data = a.tobytes()
        assert len(data) % dt.itemsize == 0, name
        while len(out) % ALIGN:
            out.append(0)
        sections[name] = (len(out), len(data) // dt.itemsize)
        out += data
    w, h = scene.env_size
    cam = scene.camera
    num_prims = len(scene.primitives) - scene.num_instances
    entry = {"byteLength": len(out), "sections": sections,
             "instancing": [scene.num_instances, num_prims, scene.tlas_root],
             "env": [w, h, float(scene.env_total_weight) if w else 0.0],
             "background": [float(x) for x in scene.background],
             "camera": {"eye": list(cam.eye), "look_at": list(cam.look_at), "up": list(cam.up),
                        "vfov_deg": cam.vfov_deg, "aperture": cam.aperture, "focus_distance": cam.focus_distance}}
    return bytes(out), entry


def load(blob: bytes, entry: dict) -> SceneDef:
    """(blob, manifest entry) -> SceneDef, the reference's SAH tree kept as
    the scene's BVH. Validates sizes and the 16-byte alignment."""
    if entry.get("byteLength", len(blob)) != len(blob):
        raise ValueError(f"blob is {len(blob)} bytes, manifest says {entry['byteLength']}")
    arr = {}
    for name, dt in SECTIONS:
        off, count = entry["sections"][name]
        if off % ALIGN:
            raise ValueError(f"section {name} at {off} is not {ALIGN}-byte aligned")
        end = off + count * dt.itemsize
        if end > len(blob):
            raise ValueError(f"section {name} runs past the blob ({end} > {len(blob)})")
        arr[name] = np.frombuffer(blob, dt, count, off).copy()
    w, h, total = entry["env"]
    ni, num_prims, tlas_root = entry["instancing"]
    if num_prims + ni != len(arr["primitives"]):
        raise ValueError("instancing counts do not add up to the primitive section")
    env_px = env_cdf = None
    if w:
        cw = max(w + 1, h + 1)
        if len(arr["envRadiance"]) != w * h or len(arr["envCdf"]) != cw * (h + 1):
            raise ValueError("environment sections do not match the manifest's size")
        env_px = arr["envRadiance"].reshape(h, w, 4)
        env_cdf = arr["envCdf"].reshape(h + 1, cw)
    cam = entry["camera"]
    return SceneDef(materials=arr["materials"], primitives=arr["primitives"], lights=arr["lights"],
                    positions=arr["positions"], vertex_attrs=arr["vertexAttrs"], triangles=arr["triangles"],
                    bvh_nodes=arr["bvhNodes"] if len(arr["bvhNodes"]) else None,
                    num_instances=ni, tlas_root=tlas_root,
                    camera=Camera(eye=tuple(cam["eye"]), look_at=tuple(cam["look_at"]), vfov_deg=cam["vfov_deg"],
                                  up=tuple(cam["up"]), aperture=cam["aperture"],
                                  focus_distance=cam["focus_distance"]),
                    background=tuple(entry["background"]), env_pixels=env_px, env_cdf=env_cdf,
                    env_total_weight=float(total))


def load_file(blob_path: str, manifest_path: str, name: str) -> SceneDef:
    """One scene of the reference's web assets (a .bin and scenes.ts)."""
    entry = parse_manifest(open(manifest_path).read())[name]
    return load(open(blob_path, "rb").read(), entry)
