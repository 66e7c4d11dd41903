"""Generate tests/golden/scene_fixtures.json from Lucida's packed scene assets.

Reads the reference's Rust-generated scene blobs (web/public/scenes/*.bin)
and their section manifest (web/src/generated/scenes.ts) from a Lucida
checkout and records, per scene and per section, the element count and a
SHA-256 of the section bytes; sections of at most 4 KiB are also stored raw
(base64) so a mismatch can be diffed field by field. The camera, background
and environment metadata are recorded too.

These digests pin the oracle's scene construction (materials, primitives,
SAH BVH nodes and triangle compaction order, light lists, procedural sky and
its CDF) bit for bit, without the reference being present at test time.

Usage:  python tests/golden/make_scene_digests.py /path/to/Lucida
"""
import base64
import hashlib
import json
import os
import re
import sys

SECTIONS = ["materials", "primitives", "lights", "positions", "vertexAttrs", "triangles", "bvhNodes",
            "envRadiance", "envCdf"]
ELEM = {"materials": 80, "primitives": 64, "lights": 64, "positions": 16, "vertexAttrs": 32,
        "triangles": 16, "bvhNodes": 32, "envRadiance": 16, "envCdf": 4}


def parse_manifest(text):
    scenes = {}
    for block in re.split(r"\n  \{\n", text)[1:]:
        name = re.search(r'name: "([^"]+)"', block).group(1)
        rec = {"asset": re.search(r'asset: "([^"]+)"', block).group(1),
               "byteLength": int(re.search(r"byteLength: (\d+)", block).group(1)),
               "remote": "remote: null" not in block}
        rec["sections"] = {}
        for s in SECTIONS:
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


def main(root):
    manifest = parse_manifest(open(os.path.join(root, "web/src/generated/scenes.ts")).read())
    out = {}
    for name, rec in manifest.items():
        path = os.path.join(root, "web/public", rec["asset"])
        if rec["remote"] or not os.path.exists(path):
            continue
        blob = open(path, "rb").read()
        secs = {}
        for s, (off, count) in rec["sections"].items():
            data = blob[off:off + count * ELEM[s]]
            entry = {"count": count, "sha256": hashlib.sha256(data).hexdigest()}
            if len(data) <= 4096:
                entry["raw"] = base64.b64encode(data).decode()
            if s == "vertexAttrs" and count:
                # Normal + pad lanes only (first 16 bytes of each 32-byte record):
                # the uv lanes carry the generating platform's libm rounding.
                lanes = b"".join(data[i * 32:i * 32 + 16] for i in range(count))
                entry["normal_lanes_sha256"] = hashlib.sha256(lanes).hexdigest()
            if s == "bvhNodes" and rec["instancing"][0]:
                # Instanced scene: the BLAS part (before the TLAS root) by
                # digest, the TLAS nodes raw, so the two can be checked apart.
                tlas_root = rec["instancing"][2]
                entry["blas_sha256"] = hashlib.sha256(data[:tlas_root * 32]).hexdigest()
                entry["tlas_raw"] = base64.b64encode(data[tlas_root * 32:]).decode()
            secs[s] = entry
        out[name] = {"sections": secs, "instancing": rec["instancing"], "env": rec["env"],
                     "background": rec["background"], "camera": rec["camera"]}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "scene_fixtures.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", dst, "scenes:", sorted(out))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
