"""Animated instanced frames with the learned guide and the denoiser.

    python -m lucida_b200.frame_bench [--frames 32] [--spp 8] [--depth 12]
        [--width 1920 --height 1080] [--meshes 16] [--instances 4096]
        [--no-guide] [--no-denoise] [--fp32-guides] [--profile-frames 3]
        [--reference-spp 256] [--out JSON]

Workload: scenes.instanced_field — 16 base meshes of 50k-500k triangles (the
displaced-icosphere recipe), 4096 instances (uniform random rotation, scale
U[0.5, 2], positions in a 100 x 10 x 100 box), device-built BLASes. Every
frame the instances turn a little about their own vertical axis and move, the
TLAS is rebuilt on the device by LBVH (luc_set_instances), the frame renders
--spp samples per pixel at --depth bounces with the guide (one Adam step per
batch), and the à-trous denoiser runs 5 iterations (sigma_n 128, sigma_d 1,
sigma_l 4) with FP16 guides. The timed loop runs the frames as they would
run in an application (no per-stage events, each CONNECT beside the next
EXTEND): CUDA events bracket each frame's TLAS build, render and denoise on
the context's stream. The per-stage split comes from --profile-frames
repeats of the last frame with stage events (LUC_FLAG_PROFILE serialises the
stages), after the timed loop.

Image error (--reference-spp > 0): the last frame's placement rendered plain
with --reference-spp samples (its own scrambling seed) is the converged
image; against it the loop's last frame (guided, denoised), the same frame
undenoised, and a plain render of the same --spp undenoised and denoised are
compared by MSE, relative MSE ((x - r)^2 / (r^2 + 1e-2)) and the median
per-pixel distance (the denoiser's own metric,
crates/core/tests/denoise_render.rs:43-88).

One JSON line: Mpaths/s over the whole frame loop, per-frame and per-stage
medians, the error table.
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
    ap.add_argument("--profile-frames", type=int, default=3)
    ap.add_argument("--reference-spp", type=int, default=256)
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
    flags = LUC_FLAG_GUIDED if guided else 0

    def render(f, fl, spp=args.spp, seed=0x5EED1234, into=acc):
        into.zero_()
        u.sample_offset = f * args.spp
        u.frame_seed = seed
        check(gpu.handle, lib().luc_render(gpu.handle, C.byref(u), spp, args.depth, fl, None,
                                           C.c_void_p(into.data_ptr())))

    def denoise(src, dst):
        check(gpu.handle, lib().luc_denoise_dev(gpu.handle, C.c_void_p(src.data_ptr()), args.width, args.height,
                                                C.byref(dp), dflags, C.c_void_p(dst.data_ptr())))

    rows = []
    for f in range(args.warmup + args.frames):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        gpu.set_instances(_animate(o2w0, f, rng_dir), mesh, material)
        ev[1].record(stream)
        render(f, flags)
        ev[2].record(stream)
        if not args.no_denoise:
            denoise(acc, den)
        ev[3].record(stream)
        torch.cuda.synchronize()
        if f >= args.warmup:
            rows.append({"tlas_ms": ev[0].elapsed_time(ev[1]), "render_ms": ev[1].elapsed_time(ev[2]),
                         "denoise_ms": ev[2].elapsed_time(ev[3]), "frame_ms": ev[0].elapsed_time(ev[3]),
                         "rays": gpu.stats().rays_extend})
    last = args.warmup + args.frames - 1
    med = {k: float(np.median([r[k] for r in rows])) for k in rows[0]}
    total_ms = float(np.sum([r["frame_ms"] for r in rows]))
    paths = P * args.spp * len(rows)
    images = {}
    if args.reference_spp > 0 or args.profile_frames > 0:
        images["guided"] = acc.view(P, 16)[:, 0:4].cpu().numpy().copy() if guided else None
        images["guided_denoised"] = den.view(P, 16)[:, 0:4].cpu().numpy().copy() if (guided and not args.no_denoise) else None
    # Stage split: repeats of the last frame with stage events (not timed above).
    stages = []
    for k in range(args.profile_frames):
        render(last, flags | LUC_FLAG_PROFILE)
        torch.cuda.synchronize()
        st = gpu.stats()
        stages.append({"extend_ms": st.ms_extend, "shade_ms": st.ms_shade, "connect_ms": st.ms_connect,
                       "guide_ms": st.ms_guide, "train_ms": st.ms_train, "total_ms": st.ms_total,
                       "nodes_per_ray": st.nodes_extend / max(st.rays_extend, 1),
                       "tris_per_ray": st.tris_extend / max(st.rays_extend, 1),
                       "nodes_per_shadow_ray": st.nodes_shadow / max(st.rays_shadow, 1),
                       "tris_per_shadow_ray": st.tris_shadow / max(st.rays_shadow, 1),
                       "blas_per_ray": st.blas_extend / max(st.rays_extend, 1),
                       "blas_per_shadow_ray": st.blas_shadow / max(st.rays_shadow, 1),
                       "shadow_rays": st.rays_shadow})
    stage_med = {k: float(np.median([r[k] for r in stages])) for k in stages[0]} if stages else {}
    out = {"metric": "Mpaths/s", "value": paths / total_ms / 1e3, "unit": "Mpaths/s",
           "workload": f"instanced field {args.meshes} meshes ({len(scene.triangles)} triangles) x "
                       f"{args.instances} instances, {args.width}x{args.height}, {args.spp} spp x {args.frames} "
                       f"frames, {args.depth} bounces",
           "guided": guided, "denoise": not args.no_denoise, "fp16_guides": not args.fp32_guides,
           "median_ms": med, "stage_ms_profiled": stage_med,
           "stage_source": f"median of {args.profile_frames} repeats of the last frame with LUC_FLAG_PROFILE "
                           "(stages in sequence), after the timed loop",
           "scene_build_s": round(build_s, 2), "upload_and_blas_s": round(upload_s, 2)}
    if guided:
        gi = guide.stats()
        out["guide"] = {"steps": gi.steps, "last_loss": gi.last_loss}
    if args.reference_spp > 0:
        ref = torch.zeros(P * 16, dtype=torch.float32, device="cuda")
        tmp = torch.zeros(P * 16, dtype=torch.float32, device="cuda")
        done = 0
        while done < args.reference_spp:  # plain, its own seed, in batches
            n = min(64, args.reference_spp - done)
            u.sample_offset = done
            u.frame_seed = 0xA5A5F00D
            check(gpu.handle, lib().luc_render(gpu.handle, C.byref(u), n, args.depth, 0, None,
                                               C.c_void_p(ref.data_ptr())))
            done += n
        r = ref.view(P, 16)[:, 0:4].cpu().numpy()
        r = r[:, 0:3].astype(np.float64) / np.maximum(r[:, 3:4], 1.0)
        render(last, 0, into=tmp)  # plain, the loop's spp and seed
        images["plain"] = tmp.view(P, 16)[:, 0:4].cpu().numpy().copy()
        if not args.no_denoise:
            denoise(tmp, den)
            images["plain_denoised"] = den.view(P, 16)[:, 0:4].cpu().numpy().copy()
        errs = {}
        for k, a in images.items():
            if a is None:
                continue
            x = a[:, 0:3].astype(np.float64) / np.maximum(a[:, 3:4], 1.0)
            d2 = (x - r) ** 2
            dist = np.sort(np.sqrt(d2.sum(1)))
            errs[k] = {"mse": float(d2.mean()), "relmse": float((d2 / (r * r + 1e-2)).mean()),
                       "median_distance": float(dist[len(dist) // 2]),
                       "p99_distance": float(dist[len(dist) * 99 // 100])}
        out["error_vs_reference"] = {"reference_spp": args.reference_spp, **errs}
        if "plain" in errs and "guided_denoised" in errs:
            out["denoised_guided_vs_undenoised_plain"] = {
                k: errs["plain"][k] / max(errs["guided_denoised"][k], 1e-300)
                for k in ("mse", "relmse", "median_distance")}
    line = json.dumps(out)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")
    gpu.close()


if __name__ == "__main__":
    main(sys.argv[1:])
