"""Throughput benchmark: Mpaths/s at 8 bounces on the displaced-sphere scene.

Workload (the benchmark's 1-GPU configuration): 256 icospheres of subdivision
level 4 (1,310,720 triangles) radially displaced by 3-octave value noise,
over a ground quad, per-mesh Lambertian / GGX conductor / rough dielectric
materials, lit by a procedural 1024 x 512 sky with a 0.5-degree sun of peak
1e4 (2-D CDF importance sampling); LBVH built on the device; 1024 x 1024, 16
spp, 8 bounces, Owen-scrambled Sobol, NEE + MIS. Synthetic, seeded inputs.

One step = one full frame (1024*1024*16 = 16.8M paths) through the wavefront
integrator into a device accumulator. `value` is device-timed (CUDA events on
the library's stream, which is torch's current stream), L2 flushed with a
256 MiB write before every timed step. `e2e` is the same metric through the
public API with host buffers: every step uploads the scene from pinned host
memory (and rebuilds the LBVH), renders, and reads the 64 MiB accumulator
back into pinned host memory, exactly what pt_gpu::render_with does per call.
The roofline's per-stage times come from profiled repeats of the timed frames
(stage events, stages in sequence), run after the timed region.

Multi-GPU (--gpus N under torchrun): each rank renders the same frame with a
disjoint sample range (sample_offset = rank * spp) — independent replicas, no
collective on the data path; value = all ranks' paths / max-over-ranks time.

--impl reference times the reference's CPU tracer — here the oracle's C++
restatement of crates/core's integrator, banded over every host core — on a
bounded band of image rows of the same scene and reports the same metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Mpaths/s at 8 bounces"
# Algorithmic bytes per node visit / triangle test / ray of EXTEND: a wide
# node record (80 B) and a wide-soup triangle (48 B); the binary tree's
# child-pair record (64 B for two children, 32 B per child tested) and soup
# triangle (48 B). A ray reads its origin and direction (32 B) and queue
# index (4 B) and writes its hit (16 B).
WIDE_BYTES = (80, 48)
BINARY_BYTES = (32, 48)
RAY_IO_BYTES = 52
# DRAM bytes (read + write) per EXTEND ray on the wide tree, from an ncu
# capture of every EXTEND launch of a 512x512x4-spp frame of the same scene
# (514.4 MB over 2,862,333 rays); scaled by the rays of a launch.
EXTEND_DRAM_BYTES_PER_RAY = 179.7


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--width", type=int, default=1024)
    ap.add_argument("--spp", type=int, default=16)
    ap.add_argument("--depth", type=int, default=8)
    ap.add_argument("--level", type=int, default=4)
    ap.add_argument("--spheres", type=int, default=256)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def build_scene(args):
    from lucida_b200 import scenes
    return scenes.displaced_spheres(count=args.spheres, level=args.level)


def cpu_baseline(scene, args, target_s: float):
    """Time the oracle (C++ restatement of the reference's CPU tracer) on a band
    of rows of the same frame, banded over every host core. Returns a dict."""
    import numpy as np
    from tests.bridge import oracle_from_scene
    t0 = time.time()
    osc = oracle_from_scene(scene, bvh="sah")  # Scene::finalize builds the binned-SAH tree
    prep = time.time() - t0
    w = args.width
    threads = os.cpu_count() or 1
    # Calibrate on a small band of rows (one row per worker), then size the
    # sample for ~target_s seconds. Rows go to workers one at a time so every
    # core stays busy on a bounded sample (the reference hands out 32-row
    # bands over a full frame; band height changes load balance, not work).
    u = osc.uniforms(w, w, args.spp, args.depth, sampler=1)
    y0 = w // 4
    rows = min(threads, w - y0)
    osc.render_sums(u, threads=threads, rows=(y0, y0 + 1), band=1)  # warms the energy table
    t0 = time.time()
    osc.render_sums(u, threads=threads, rows=(y0, y0 + rows), band=1)
    dt = max(time.time() - t0, 1e-3)
    rows = int(max(rows, min(w - y0, 0.5 * rows * target_s / dt)))
    t0 = time.time()
    osc.render_sums(u, threads=threads, rows=(y0, y0 + rows), band=1)
    dt = time.time() - t0
    paths = rows * w * args.spp
    return {"value": paths / dt / 1e6, "unit": "Mpaths/s", "cores": threads, "kind": "port",
            "sample": f"rows {y0}..{y0 + rows} of the {w}x{w} frame ({paths} paths, {args.spp} spp, "
                      f"depth {args.depth}), C++ restatement of the reference's banded CPU tracer, "
                      f"{threads} threads, 1-row bands, SAH BVH (build {prep:.1f}s untimed)", "seconds": dt}


def config_block(args, n_tris, world):
    return {"workload": f"displaced-spheres: {args.spheres} icospheres level {args.level} ({n_tris} triangles), "
                        f"sky 1024x512 + sun, LBVH on device, {args.width}x{args.width}, {args.spp} spp, "
                        f"{args.depth} bounces, Sobol, NEE+MIS",
            "width": args.width, "height": args.width, "spp": args.spp, "max_depth": args.depth,
            "triangles": n_tris, "parallelism": f"replicas x{world} (disjoint sample ranges)",
            "l2": "flushed (256 MiB write) before every timed step; path pool of 3.5 GB streamed per bounce"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    scene = build_scene(args)
    n_tris = len(scene.triangles)
    # Each step: a bounded band sized so the whole run stays within minutes.
    per_step = max(2.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_baseline(scene, args, per_step / 4)
    vals, secs = [], []
    cb = None
    for _ in range(args.steps):
        cb = cpu_baseline(scene, args, per_step)
        vals.append(cb["value"])
        secs.append(cb["seconds"])
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mpaths/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * args.width * args.width * args.spp / (v * 1e6),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": config_block(args, n_tris, 1),
            "cpu_baseline": {"value": v, "unit": "Mpaths/s", "cores": cb["cores"], "kind": "port",
                             "sample": cb["sample"]},
            "e2e": {"value": v, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's Rust tracer cannot be built here (no cargo); timed is the oracle's C++ "
                    "restatement of crates/core/src/integrator.rs with its 32-row band scheduler"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import ctypes as C

    import numpy as np
    import torch

    import lucida_b200 as lb
    from lucida_b200 import layout as L
    from lucida_b200.native import LUC_FLAG_NO_GUIDES, LUC_FLAG_PROFILE, check, lib

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    scene = build_scene(args)
    n_tris = len(scene.triangles)
    W = H = args.width
    P = W * H
    params = lb.RenderParams(width=W, height=H, samples=args.spp, max_depth=args.depth, sampler="sobol",
                             sampling="mis", sample_offset=rank * args.spp)
    u = lb.build_uniforms(scene, params)

    gpu = lb.Gpu(local)
    stream = torch.cuda.current_stream()
    gpu.set_stream(stream.cuda_stream)
    t0 = time.time()
    gpu.upload(scene)  # LBVH built on the device
    wide = len(gpu.read_scene("wide_nodes")) > 0  # collapsed to the 8-wide tree unless LUC_BINARY_BVH=1
    torch.cuda.synchronize()
    upload_s = time.time() - t0
    acc = torch.zeros(P * 16, dtype=torch.float32, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2
    h = gpu.handle

    def render_dev(flags=0):
        check(h, lib().luc_render(h, C.byref(u), args.spp, args.depth, flags, None, C.c_void_p(acc.data_ptr())))

    for _ in range(args.warmup):
        render_dev()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    stage = {"extend": 0.0, "shade": 0.0, "connect": 0.0, "generate": 0.0, "resolve": 0.0}
    counts = {"rays_extend": 0, "nodes_extend": 0, "tris_extend": 0, "rays_shadow": 0, "nodes_shadow": 0,
              "tris_shadow": 0, "launches": 0}
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            render_dev()
            ev[k][1].record(stream)
            s = gpu.stats()
            for key in counts:
                counts[key] += getattr(s, key)
        torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    # Stage split for the roofline: the same frames again with stage events
    # (LUC_FLAG_PROFILE runs the stages in sequence; the timed frames above
    # run each CONNECT beside the next EXTEND). Not part of the timed region.
    render_dev(LUC_FLAG_PROFILE)
    for k in range(args.steps):
        flush.fill_(float(k))
        render_dev(LUC_FLAG_PROFILE)
        s = gpu.stats()
        for key in stage:
            stage[key] += getattr(s, "ms_" + key)
    torch.cuda.synchronize()
    ms = max_over_ranks(sum(step_ms) / args.steps, world)
    value = world * P * args.spp / (ms / 1e3) / 1e6

    # --- end to end through the public API, host buffers in pinned memory
    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1)).pin_memory()
        return t.numpy().view(a.dtype).reshape(a.shape)

    pscene = lb.SceneDef(materials=pinned(scene.materials), primitives=pinned(scene.primitives),
                         lights=pinned(scene.lights), positions=pinned(scene.positions),
                         vertex_attrs=pinned(scene.vertex_attrs), triangles=pinned(scene.triangles),
                         camera=scene.camera, env_pixels=pinned(scene.env_pixels), env_cdf=pinned(scene.env_cdf),
                         env_total_weight=scene.env_total_weight)
    out_host = pinned(np.zeros(P, L.ACCUM))
    h2d = sum(a.nbytes for a in (pscene.materials, pscene.primitives, pscene.lights, pscene.positions,
                                 pscene.vertex_attrs, pscene.triangles, pscene.env_pixels, pscene.env_cdf))
    d2h = out_host.nbytes
    e2e_ms = []
    for k in range(args.e2e_steps + 1):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        gpu.upload(pscene, force=True)
        check(h, lib().luc_render(h, C.byref(u), args.spp, args.depth, 0, out_host.ctypes.data_as(C.c_void_p), None))
        b.record(stream)
        torch.cuda.synchronize()
        if k > 0:  # the first call warms the pinned-path allocations
            e2e_ms.append(a.elapsed_time(b))
    e2e_step = max_over_ranks(statistics.median(e2e_ms), world)
    e2e_value = world * P * args.spp / (e2e_step / 1e3) / 1e6

    # --- roofline of the dominant kernel (EXTEND: closest-hit traversal)
    hbm, peak_kind = peaks()
    launches_extend = args.depth * args.steps
    ext_ms = stage["extend"] / launches_extend
    node_b, tri_b = WIDE_BYTES if wide else BINARY_BYTES
    bytes_per_launch = (counts["nodes_extend"] * node_b + counts["tris_extend"] * tri_b +
                        counts["rays_extend"] * RAY_IO_BYTES) / launches_extend
    achieved = bytes_per_launch / (ext_ms / 1e3) / 1e9
    roofline = {"kernel": "k_extend (closest-hit BVH traversal)", "bound": "hbm", "achieved": achieved,
                "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_source": peak_kind,
                "traffic": EXTEND_DRAM_BYTES_PER_RAY * counts["rays_extend"] / launches_extend if wide else None,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per EXTEND ray on a 512x512x4-spp "
                                  "frame of this scene, scaled by this launch size's rays",
                "model": f"{'wide' if wide else 'binary'} tree: node visits x {node_b} B + triangle tests x "
                         f"{tri_b} B + rays x {RAY_IO_BYTES} B per launch (measured counters); most node bytes "
                         "are L2 hits",
                "ms_per_launch": ext_ms, "stage_ms_per_step": {k: v / args.steps for k, v in stage.items()},
                "stage_source": "CUDA events between stages on profiled repeats of the timed frames (stages in "
                                "sequence; the timed frames overlap each CONNECT with the next EXTEND)",
                "per_ray": {"nodes": counts["nodes_extend"] / max(1, counts["rays_extend"]),
                            "tris": counts["tris_extend"] / max(1, counts["rays_extend"]),
                            "rays_per_path": counts["rays_extend"] / (args.steps * P * args.spp)}}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(scene, args, args.cpu_seconds)
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene, random materials)",
                "config": config_block(args, n_tris, world),
                "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_step,
                        "includes": "scene upload from pinned host memory + device LBVH rebuild + render + "
                                    "accumulator readback (pt_gpu::render_with per call)"},
                "gpu_launches": int(counts["launches"]),
                "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks.summary(),
                "scene_upload_s": upload_s}
        print(json.dumps(line), flush=True)
    gpu.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
