"""Animated instanced frames with the learned guide and the denoiser.

    python -m lucida_b200.frame_bench [--frames 32] [--spp 8] [--depth 12]
        [--width 1920 --height 1080] [--meshes 16] [--instances 4096]
        [--no-guide] [--no-denoise] [--fp32-guides] [--out JSON]

Workload: scenes.instanced_field — 16 base meshes of 50k-500k triangles (the
displaced-icosphere recipe), 4096 instances (uniform random rotation, scale
U[0.5, 2], positions in a 100 x 10 x 100 box), device-built BLASes. Every
frame the instances turn a little about their own vertical axis and move, the
TLAS is rebuilt on the device by LBVH (luc_set_instances), the frame renders
--spp samples per pixel at --depth bounces with the guide (one Adam step per
batch), and the à-trous denoiser runs 5 iterations (sigma_n 128, sigma_d 1,
sigma_l 4) with FP16 guides. Stage times are CUDA events on the context's
stream; one JSON line (Mpaths/s over the whole frame loop, per-stage ms).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
import time

import numpy as np

from . import scenes
from .gpu import Gpu, RenderParams, build_uniforms
from .guide import Guide
from .native import (LUC_DENOISE_HALF_GUIDES, LUC_FLAG_GUIDED, LUC_FLAG_PROFILE, DenoiseParams, check, lib)


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--frames", type=int, default=32)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--spp", type=int, default=8)
    ap.add_argument("--depth", type=int, default=12)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--meshes", type=int, default=16)
    ap.add_argument("--instances", type=int, default=4096)
    ap.add_argument("--min-tris", type=int, default=50_000)
    ap.add_argument("--max-tris", type=int, default=500_000)
    ap.add_argument("--no-guide", action="store_true")
    ap.add_argument("--no-denoise", action="store_true")
    ap.add_argument("--fp32-guides", action="store_true")
    ap.add_argument("--out", default=None)
    return ap.parse_args(argv)


def _animate(o2w0, frame, rng_dir):
    """Turn each instance by 0.02 rad per frame about world y through its own
    position and drift it along a fixed random direction."""
    a = 0.02 * frame
    c, s = np.cos(a), np.sin(a)
    ry = np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]], np.float32)
    out = o2w0.copy()
    out[:, :, :3] = np.einsum("ij,njk->nik", ry, o2w0[:, :, :3])
    out[:, :, 3] = o2w0[:, :, 3] + 0.05 * frame * rng_dir
    return out


def main(argv=None):
    import torch
    args = parse(argv)
    t0 = time.time()
    scene = scenes.instanced_field(num_meshes=args.meshes, tri_range=(args.min_tris, args.max_tris),
                                   num_instances=args.instances)
    build_s = time.time() - t0
    torch.cuda.init()
    stream = torch.cuda.current_stream()
    gpu = Gpu(0)
    gpu.set_stream(stream.cuda_stream)
    t0 = time.time()
    gpu.upload(scene)
    torch.cuda.synchronize()
    upload_s = time.time() - t0
    o2w0, mesh, material = scene.placements
    rng_dir = np.random.default_rng(99).normal(size=(len(o2w0), 3)).astype(np.float32)
    guided = not args.no_guide
    if guided:
        guide = Guide(gpu, seed=1)
        guide.configure(train=True, records_per_step=1 << 18, lr=1e-2)
    params = RenderParams(width=args.width, height=args.height, samples=args.spp, max_depth=args.depth,
                          sampler="sobol")
    u = build_uniforms(scene, params)
    P = args.width * args.height
    acc = torch.zeros(P * 16, dtype=torch.float32, device="cuda")
    den = torch.zeros(P * 16, dtype=torch.float32, device="cuda")
    dp = DenoiseParams(5, 128.0, 1.0, 4.0, 0.1)
    dflags = 0 if args.fp32_guides else LUC_DENOISE_HALF_GUIDES
    flags = (LUC_FLAG_GUIDED if guided else 0) | LUC_FLAG_PROFILE
    rows = []
    for f in range(args.warmup + args.frames):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        gpu.set_instances(_animate(o2w0, f, rng_dir), mesh, material)
        ev[1].record(stream)
        acc.zero_()
        u.sample_offset = f * args.spp
        u.frame_seed = 0x5EED1234
        check(gpu.handle, lib().luc_render(gpu.handle, C.byref(u), args.spp, args.depth, flags, None,
                                           C.c_void_p(acc.data_ptr())))
        st = gpu.stats()
        ev[2].record(stream)
        if not args.no_denoise:
            check(gpu.handle, lib().luc_denoise_dev(gpu.handle, C.c_void_p(acc.data_ptr()), args.width, args.height,
                                                    C.byref(dp), dflags, C.c_void_p(den.data_ptr())))
        ev[3].record(stream)
        torch.cuda.synchronize()
        if f >= args.warmup:
            rows.append({"tlas_ms": ev[0].elapsed_time(ev[1]), "render_ms": ev[1].elapsed_time(ev[2]),
                         "denoise_ms": ev[2].elapsed_time(ev[3]), "frame_ms": ev[0].elapsed_time(ev[3]),
                         "extend_ms": st.ms_extend, "shade_ms": st.ms_shade, "connect_ms": st.ms_connect,
                         "guide_ms": st.ms_guide, "train_ms": st.ms_train, "rays": st.rays_extend})
    med = {k: float(np.median([r[k] for r in rows])) for k in rows[0]}
    total_ms = float(np.sum([r["frame_ms"] for r in rows]))
    paths = P * args.spp * len(rows)
    out = {"metric": "Mpaths/s", "value": paths / total_ms / 1e3, "unit": "Mpaths/s",
           "workload": f"instanced field {args.meshes} meshes ({len(scene.triangles)} triangles) x "
                       f"{args.instances} instances, {args.width}x{args.height}, {args.spp} spp x {args.frames} "
                       f"frames, {args.depth} bounces",
           "guided": guided, "denoise": not args.no_denoise, "fp16_guides": not args.fp32_guides,
           "median_ms": med, "scene_build_s": round(build_s, 2), "upload_and_blas_s": round(upload_s, 2)}
    if guided:
        gi = guide.stats()
        out["guide"] = {"steps": gi.steps, "last_loss": gi.last_loss}
    line = json.dumps(out)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")
    gpu.close()


if __name__ == "__main__":
    main(sys.argv[1:])
