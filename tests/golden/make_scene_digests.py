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
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", ".."))
from lucida_b200.packed import parse_manifest  # noqa: E402

SECTIONS = ["materials", "primitives", "lights", "positions", "vertexAttrs", "triangles", "bvhNodes",
            "envRadiance", "envCdf"]
ELEM = {"materials": 80, "primitives": 64, "lights": 64, "positions": 16, "vertexAttrs": 32,
        "triangles": 16, "bvhNodes": 32, "envRadiance": 16, "envCdf": 4}


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
    if len(sys.argv) != 2:
        sys.exit("usage: make_scene_digests.py <path of the Lucida checkout>")
    main(sys.argv[1])
