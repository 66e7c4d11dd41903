"""Throughput benchmark: Mpaths/s at 8 bounces on the displaced-sphere scene.

Workload (the benchmark's 1-GPU configuration): 256 icospheres of subdivision
level 4 (1,310,720 triangles) radially displaced by 3-octave value noise,
over a ground quad, per-mesh Lambertian / GGX conductor / rough dielectric
materials, lit by a procedural 1024 x 512 sky with a 0.5-degree sun of peak
1e4 (2-D CDF importance sampling); LBVH built on the device; 1024 x 1024, 16
spp, 8 bounces, Owen-scrambled Sobol, NEE + MIS. Synthetic, seeded inputs.

One step = one full frame (1024*1024*16 = 16.8M paths per GPU) through the
wavefront integrator into a cleared device accumulator. `value` is device-timed (CUDA events on
the library's stream, which is torch's current stream), L2 flushed with a
256 MiB write before every timed step. `e2e` is the same metric through the
public API with host buffers: every step uploads the scene from pinned host
memory (and rebuilds the LBVH), renders, and reads the 64 MiB accumulator
back into pinned host memory, exactly what pt_gpu::render_with does per call.
The roofline's per-stage times come from profiled repeats of the timed frames
(stage events, stages in sequence), run after the timed region.

Multi-GPU (--gpus N under torchrun): each rank renders its own sample range
of the frame (lucida_b200.shards.shard_params: samples [rank*spp,
(rank+1)*spp) of every pixel) and every frame the ranks' accumulators are
merged into the frame's (merge_accumulators: an all-to-all of pixel slices
over NCCL, a rank-order sum of each slice, an all-gather of the sums) inside
the timed region; value = all ranks' paths /
max-over-ranks time.

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


class CpuBaseline:
    """The oracle (C++ restatement of the reference's CPU tracer) on a
    bounded sample of the same frame: image rows spaced evenly over the whole
    height, each row one work item for a pool of every host core (the
    reference hands 32-row bands of a full frame to its threads through an
    atomic counter, integrator.rs:635-699; on a sample of a few dozen rows,
    one-row items keep every core busy). The binned-SAH tree is built once,
    untimed (Scene::finalize)."""

    def __init__(self, scene, args):
        from tests.bridge import oracle_from_scene
        t0 = time.time()
        self.osc = oracle_from_scene(scene, bvh="sah")
        self.prep = time.time() - t0
        self.args = args
        self.threads = os.cpu_count() or 1
        w = args.width
        self.u = self.osc.uniforms(w, w, args.spp, args.depth, sampler=1)
        self.osc.render_rows(self.u, [w // 2], threads=1)  # warms the energy table
        t0 = time.time()
        self.osc.render_rows(self.u, self.rows(self.threads), threads=self.threads)
        self.row_s = max(time.time() - t0, 1e-3) / self.threads  # wall seconds per row on the pool

    def rows(self, n):
        import numpy as np
        h = self.args.width
        n = max(1, min(h, int(n)))
        return np.unique(np.round(np.linspace(0, h - 1, n)).astype(np.uint32))

    def run(self, target_s: float):
        rows = self.rows(target_s / self.row_s)
        t0 = time.time()
        self.osc.render_rows(self.u, rows, threads=self.threads)
        dt = time.time() - t0
        a, w = self.args, self.args.width
        paths = len(rows) * w * a.spp
        return {"value": paths / dt / 1e6, "unit": "Mpaths/s", "cores": self.threads, "kind": "port",
                "sample": f"{len(rows)} rows spaced evenly over the {w}x{w} frame ({paths} paths, {a.spp} spp, "
                          f"depth {a.depth}), C++ restatement of the reference's CPU tracer on {self.threads} "
                          f"threads, one row per work item, binned-SAH BVH (build {self.prep:.1f}s untimed)",
                "seconds": dt}


def config_block(args, n_tris, world):
    return {"workload": f"displaced-spheres: {args.spheres} icospheres level {args.level} ({n_tris} triangles), "
                        f"sky 1024x512 + sun, LBVH on device, {args.width}x{args.width}, {args.spp} spp, "
                        f"{args.depth} bounces, Sobol, NEE+MIS",
            "width": args.width, "height": args.width, "spp": args.spp, "max_depth": args.depth,
            "triangles": n_tris,
            "parallelism": f"sample-range shards x{world}" + (", accumulators merged every frame (all-to-all of "
                                                             "pixel slices, rank-order sums, all-gather)"
                                                             if world > 1 else ""),
            "l2": "flushed (256 MiB write) before every timed step; path pool of 3.5 GB streamed per bounce"}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    scene = build_scene(args)
    n_tris = len(scene.triangles)
    # Each step: a bounded sample sized so the whole run stays within minutes.
    per_step = max(2.0, min(12.0, 90.0 / max(1, args.steps)))
    base = CpuBaseline(scene, args)
    for _ in range(args.warmup):
        base.run(per_step / 4)
    vals, secs = [], []
    cb = None
    for _ in range(args.steps):
        cb = base.run(per_step)
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
                    "restatement of crates/core/src/integrator.rs over every host core, on rows spaced evenly "
                    "over the frame, one row per work item"}
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
    from lucida_b200.native import LUC_FLAG_PROFILE, check, lib
    from lucida_b200.shards import merge_accumulators, shard_params

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    scene = build_scene(args)
    n_tris = len(scene.triangles)
    W = H = args.width
    P = W * H
    params = shard_params(lb.RenderParams(width=W, height=H, samples=args.spp, max_depth=args.depth,
                                          sampler="sobol", sampling="mis"), rank)
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

    def frame(flags=0):
        """One frame: this rank's sample range into a cleared accumulator,
        then (N > 1) the ranks' accumulators merged into the frame's."""
        acc.zero_()
        render_dev(flags)
        if world > 1:
            merge_accumulators(acc, gpu)

    for _ in range(args.warmup):
        frame()
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
            frame()
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
    out_t = torch.from_numpy(out_host.view(np.float32).reshape(-1))
    h2d = sum(a.nbytes for a in (pscene.materials, pscene.primitives, pscene.lights, pscene.positions,
                                 pscene.vertex_attrs, pscene.triangles, pscene.env_pixels, pscene.env_cdf))
    d2h = out_host.nbytes
    e2e_ms = []
    for k in range(args.e2e_steps + 1):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        gpu.upload(pscene, force=True)
        if world == 1:  # pt_gpu::render_with: render and read the accumulator back
            check(h, lib().luc_render(h, C.byref(u), args.spp, args.depth, 0, out_host.ctypes.data_as(C.c_void_p),
                                      None))
        else:  # this rank's samples, the merge, and the merged frame read back
            frame()
            out_t.copy_(acc, non_blocking=True)
        b.record(stream)
        torch.cuda.synchronize()
        if k > 0:  # the first call warms the pinned-path allocations
            e2e_ms.append(a.elapsed_time(b))
    e2e_step = max_over_ranks(statistics.median(e2e_ms), world)
    e2e_value = world * P * args.spp / (e2e_step / 1e3) / 1e6

    # --- bandwidth references measured on this GPU, now: a streaming read of
    # a 64 MiB buffer that stays L2-resident across passes (the peak the
    # traversal's node and triangle traffic, mostly L2 hits, is set against).
    l2_buf = torch.empty(64 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda").fill_(1.0)
    sink = torch.zeros(148 * 8, dtype=torch.int32, device="cuda")
    check(h, lib().luc_read_sweep(h, C.c_void_p(l2_buf.data_ptr()), l2_buf.numel() * 4, 3,
                                  C.c_void_p(sink.data_ptr())))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    passes = 50
    a.record(stream)
    check(h, lib().luc_read_sweep(h, C.c_void_p(l2_buf.data_ptr()), l2_buf.numel() * 4, passes,
                                  C.c_void_p(sink.data_ptr())))
    b.record(stream)
    torch.cuda.synchronize()
    l2_gbs = l2_buf.numel() * 4 * passes / (a.elapsed_time(b) / 1e3) / 1e9
    del l2_buf

    # --- roofline of the dominant kernel (EXTEND: closest-hit traversal)
    hbm, peak_kind = peaks()
    launches_extend = args.depth * args.steps
    ext_ms = stage["extend"] / launches_extend
    node_b, tri_b = WIDE_BYTES if wide else BINARY_BYTES
    bytes_per_launch = (counts["nodes_extend"] * node_b + counts["tris_extend"] * tri_b +
                        counts["rays_extend"] * RAY_IO_BYTES) / launches_extend
    achieved = bytes_per_launch / (ext_ms / 1e3) / 1e9
    traffic = EXTEND_DRAM_BYTES_PER_RAY * counts["rays_extend"] / launches_extend if wide else None
    dram_gbs = traffic / (ext_ms / 1e3) / 1e9 if traffic else None
    roofline = {"kernel": "k_extend (closest-hit BVH traversal)", "bound": "l2", "achieved": achieved,
                "peak": l2_gbs, "unit": "GB/s", "frac": achieved / l2_gbs,
                "peak_source": "measured in this run: luc_read_sweep, 128-bit streaming reads of a 64 MiB "
                               "L2-resident buffer, 50 passes, CUDA events",
                "frac_l2": achieved / l2_gbs, "frac_dram": dram_gbs / hbm if dram_gbs else None,
                "dram_gbs": dram_gbs, "frac_hbm_of_logical_bytes": achieved / hbm, "hbm_peak": hbm,
                "hbm_peak_source": peak_kind,
                "limiter": "instruction issue: ncu on a 512x512x4-spp frame of this scene shows 72-74% issue "
                           "active, the ALU pipe at 52-54%, 15-18 of 32 threads active per warp instruction, "
                           "68-79% L2 hit rate (profiles/k_extend_wide_small_case.md)",
                "traffic": traffic,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per EXTEND ray on a 512x512x4-spp "
                                  "frame of this scene, scaled by this launch size's rays",
                "model": f"{'wide' if wide else 'binary'} tree: node visits x {node_b} B + triangle tests x "
                         f"{tri_b} B + rays x {RAY_IO_BYTES} B per launch (measured counters), against the L2 "
                         "read bandwidth since most of those bytes are L2 hits",
                "ms_per_launch": ext_ms, "stage_ms_per_step": {k: v / args.steps for k, v in stage.items()},
                "stage_source": "CUDA events between stages on profiled repeats of the timed frames (stages in "
                                "sequence; the timed frames overlap each CONNECT with the next EXTEND)",
                "per_ray": {"nodes": counts["nodes_extend"] / max(1, counts["rays_extend"]),
                            "tris": counts["tris_extend"] / max(1, counts["rays_extend"]),
                            "rays_per_path": counts["rays_extend"] / (args.steps * P * args.spp)}}

    # --- wavefront queue/state traffic against HBM: the SoA path-pool fields
    # each stage reads and writes per live path (one 16-byte float4 per
    # field, a 4-byte queue entry), from the frame's own counters.
    paths = args.steps * P * args.spp
    re, rs = counts["rays_extend"], counts["rays_shadow"]
    survivors = re - paths  # every path extended after the first bounce survived a SHADE
    state = {
        # o_pdf, dir, thr, rad, prev (+ galb, gnrm: first-hit guides) written
        "generate": paths * (5 * 16 + 2 * 16),
        # queue entry (not at depth 0) + origin + direction read, hit written
        "extend": re * RAY_IO_BYTES - paths * 4,
        # read: queue, o_pdf, dir, hit, thr, rad; written: rad, and for
        # survivors o_pdf, dir, thr, prev + next-queue entry; guides at the
        # first hit; each shadow ray's origin, direction, contribution
        "shade": (re * (4 + 5 * 16) - paths * 4) + re * 16 + survivors * (4 * 16 + 4) + paths * 32 + rs * 48,
        # shadow origin + direction read (lower bound: an unoccluded ray also
        # reads its contribution and adds it to the path's radiance, 48 B)
        "connect": rs * 32,
        # per path radiance + guides read; per pixel the accumulator r/w
        "resolve": paths * 48 + args.steps * P * 128,
    }
    stage_state = {"unit": "GB/s", "hbm_peak": hbm,
                   "bytes_per_live_path_bounce": sum(state.values()) / max(1, re),
                   "model": "SoA path-pool fields read and written per live path by each stage (16 B per float4 "
                            "field, 4 B queue entries), from the frame's ray counters; CONNECT counts only the "
                            "shadow ray read (a lower bound)"}
    for k, v in state.items():
        t = stage[k] / 1e3
        stage_state[k] = {"bytes_per_step": v / args.steps, "gbs": v / t / 1e9 if t > 0 else None,
                          "frac_hbm": v / t / 1e9 / hbm if t > 0 else None}
    frame_s = sum(stage.values()) / 1e3
    stage_state["frame"] = {"bytes_per_step": sum(state.values()) / args.steps,
                            "gbs": sum(state.values()) / frame_s / 1e9,
                            "frac_hbm": sum(state.values()) / frame_s / 1e9 / hbm}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = CpuBaseline(scene, args).run(args.cpu_seconds)
        cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene, random materials)",
                "config": config_block(args, n_tris, world),
                "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_step,
                        "includes": "scene upload from pinned host memory + device LBVH rebuild + render + "
                                    "accumulator readback (pt_gpu::render_with per call); with N > 1 each "
                                    "rank's sample range, the accumulator merge (all-to-all of pixel "
                                    "slices, rank-order sums, all-gather), then the merged frame read back"},
                "gpu_launches": int(counts["launches"]),
                "roofline": roofline, "stage_state": stage_state, "cpu_baseline": cpu,
                "clocks": clocks.summary(),
                "scene_upload_s": upload_s}
        print(json.dumps(line), flush=True)
    gpu.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
