"""Equal-time error of guided against plain rendering on the path-guiding
workload (scenes.guided_room: the displaced-spheres geometry in a half-closed
room lit by two 0.2 x 0.2 emitters of radiance 200), 1024 x 1024, 8 bounces.

    python -m lucida_b200.guide_study [--budgets 2 8 32] [--ref-spp 65536]
                                      [--ref-cache PATH] [--out JSON]

The reference is a plain render of --ref-spp samples per pixel (Sobol, its
own scrambling seed), cached as .npy at --ref-cache.

Time to target (--target-spp, default 64): the wall-clock time plain
rendering takes to accumulate --target-spp samples per pixel, and its MSE
against the reference (the target); then, from a fresh guide, the wall-clock
time guided rendering (1-spp batches, one Adam step after each) takes until
its accumulated image first reaches that MSE. The error is evaluated after
every batch on the device, with the clock stopped. Optionally the guide first
trains on --warmup-frames guided frames at --warmup-res x --warmup-res (they
produce records, not image samples), which counts toward the guided time.
The ratio plain / guided is the speed-up to equal error (>= 2 is the target
the guided form is measured against).

Then, for every time
budget T (seconds of wall clock, each call synchronised), a plain render and a
guided render (a fresh guide, one Adam step on up to 2^18 path vertices after
every 1-spp batch) run until T has elapsed; both accumulate on the device and
are compared with the reference by mean squared error (and relative MSE,
(x - r)^2 / (r^2 + 1e-2)). One JSON line goes to stdout (and --out).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys
import time

import numpy as np

from . import scenes
from .gpu import Gpu, RenderParams, build_uniforms
from .guide import Guide
from .native import LUC_FLAG_GUIDED, LUC_FLAG_NO_GUIDES, check, lib


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--width", type=int, default=1024)
    ap.add_argument("--height", type=int, default=1024)
    ap.add_argument("--depth", type=int, default=8)
    ap.add_argument("--budgets", type=float, nargs="*", default=[2.0, 8.0, 32.0])
    ap.add_argument("--ref-spp", type=int, default=65536)
    ap.add_argument("--ref-batch", type=int, default=16)
    ap.add_argument("--ref-cache", default=None)
    ap.add_argument("--plain-batch", type=int, default=4)
    ap.add_argument("--guided-batch", type=int, default=1)
    ap.add_argument("--records", type=int, default=1 << 18)
    ap.add_argument("--lr", type=float, default=1e-2)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--level", type=int, default=4)
    ap.add_argument("--target-spp", type=int, default=64)
    ap.add_argument("--target-max-factor", type=float, default=8.0,
                    help="give up on the guided run after this multiple of plain's time to target")
    ap.add_argument("--warmup-frames", type=int, default=0)
    ap.add_argument("--warmup-res", type=int, default=256)
    ap.add_argument("--out", default=None)
    return ap.parse_args(argv)


class _Frame:
    """A device accumulator and the render call into it."""

    def __init__(self, gpu, u, width, height, depth):
        import torch
        self.torch = torch
        self.gpu, self.u, self.depth = gpu, u, depth
        self.pixels = width * height
        self.acc = torch.zeros(self.pixels * 16, dtype=torch.float32, device="cuda")
        self.shape = (height, width)

    def clear(self):
        self.acc.zero_()
        self.torch.cuda.synchronize()

    def render(self, spp, offset, flags):
        self.u.sample_offset = offset
        check(self.gpu.handle, lib().luc_render(self.gpu.handle, C.byref(self.u), spp, self.depth,
                                                flags | LUC_FLAG_NO_GUIDES, None, C.c_void_p(self.acc.data_ptr())))

    def image(self):
        a = self.acc.view(self.pixels, 16).cpu().numpy()
        return (a[:, 0:3] / np.maximum(a[:, 3:4], 1.0)).reshape(*self.shape, 3)


def _timed(frame, budget, batch, flags):
    frame.clear()
    n = 0
    t0 = time.perf_counter()
    while True:
        frame.render(batch, n, flags)
        n += batch
        if time.perf_counter() - t0 >= budget:
            break
    return n, time.perf_counter() - t0


def _device_mse(frame, ref_dev):
    """MSE of the frame's accumulated image against the reference, on the device."""
    a = frame.acc.view(frame.pixels, 16)
    img = a[:, 0:3] / a[:, 3:4].clamp(min=1.0)
    return float(((img.double() - ref_dev) ** 2).mean())


def _time_to_target(args, scene, gpu, ft, ref, guide):
    import torch
    ref_dev = torch.from_numpy(ref.reshape(-1, 3)).cuda()
    # Plain: --target-spp samples in the plain batches, timed, then its error.
    ft.clear()
    t0 = time.perf_counter()
    n = 0
    while n < args.target_spp:
        b = min(args.plain_batch, args.target_spp - n)
        ft.render(b, n, 0)
        n += b
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    target = _device_mse(ft, ref_dev)
    # Guided: a fresh guide; optional low-resolution training frames first.
    guide.reset(seed=args.seed)
    guide.configure(train=True, records_per_step=args.records, lr=args.lr)
    warm = None
    if args.warmup_frames > 0:
        wp = RenderParams(width=args.warmup_res, height=args.warmup_res, samples=1, max_depth=args.depth,
                          sampler="sobol", frame_seed=0x0BADCAFE)
        warm = _Frame(gpu, build_uniforms(scene, wp), args.warmup_res, args.warmup_res, args.depth)
        warm.render(1, 0, LUC_FLAG_GUIDED)  # capture the graph outside the clock
        guide.reset(seed=args.seed)
        guide.configure(train=True, records_per_step=args.records, lr=args.lr)
    ft.clear()
    elapsed, n, trace = 0.0, 0, []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(args.warmup_frames):
        warm.render(1, k, LUC_FLAG_GUIDED)
    torch.cuda.synchronize()
    warm_s = time.perf_counter() - t0
    elapsed += warm_s
    reached = None
    while elapsed < args.target_max_factor * t_plain:
        t0 = time.perf_counter()
        ft.render(args.guided_batch, n, LUC_FLAG_GUIDED)
        torch.cuda.synchronize()
        elapsed += time.perf_counter() - t0
        n += args.guided_batch
        e = _device_mse(ft, ref_dev)  # clock stopped
        trace.append((round(elapsed, 4), n, e))
        if e <= target:
            reached = elapsed
            break
    return {"target_spp": args.target_spp, "plain_seconds": round(t_plain, 4), "target_mse": target,
            "guided_seconds": None if reached is None else round(reached, 4), "guided_spp": n,
            "warmup_frames": args.warmup_frames, "warmup_res": args.warmup_res, "warmup_seconds": round(warm_s, 4),
            "speedup_plain_over_guided": None if reached is None else t_plain / reached,
            "gave_up_after_s": None if reached is not None else round(elapsed, 4),
            "trace_every_8": trace[::8]}


def _errors(img, ref):
    d = (img.astype(np.float64) - ref) ** 2
    return {"mse": float(d.mean()), "relmse": float((d / (ref * ref + 1e-2)).mean())}


def main(argv=None):
    args = parse(argv)
    scene = scenes.guided_room(level=args.level)
    gpu = Gpu(0)
    gpu.upload(scene)
    ref_params = RenderParams(width=args.width, height=args.height, samples=1, max_depth=args.depth,
                              sampler="sobol", frame_seed=0xA5A5F00D)
    test_params = RenderParams(width=args.width, height=args.height, samples=1, max_depth=args.depth,
                               sampler="sobol", frame_seed=0x5EED1234)
    ref = None
    if args.ref_cache and os.path.exists(args.ref_cache):
        ref = np.load(args.ref_cache)
        if ref.shape != (args.height, args.width, 3):
            ref = None
    fr = _Frame(gpu, build_uniforms(scene, ref_params), args.width, args.height, args.depth)
    ref_seconds = None
    if ref is None:
        fr.clear()
        t0 = time.perf_counter()
        for k in range(0, args.ref_spp, args.ref_batch):
            fr.render(min(args.ref_batch, args.ref_spp - k), k, 0)
        ref_seconds = time.perf_counter() - t0
        ref = fr.image().astype(np.float64)
        if args.ref_cache:
            os.makedirs(os.path.dirname(os.path.abspath(args.ref_cache)), exist_ok=True)
            np.save(args.ref_cache, ref.astype(np.float32))
    ref = ref.astype(np.float64)
    ft = _Frame(gpu, build_uniforms(scene, test_params), args.width, args.height, args.depth)
    guide = Guide(gpu, seed=args.seed)
    guide.configure(train=True, records_per_step=args.records, lr=args.lr)
    # Warm both paths once (graph capture, allocations) outside the budgets.
    ft.render(args.plain_batch, 0, 0)
    ft.render(args.guided_batch, 0, LUC_FLAG_GUIDED)
    ttt = _time_to_target(args, scene, gpu, ft, ref, guide) if args.target_spp > 0 else None
    if ttt:
        print(json.dumps({"time_to_target": {k: v for k, v in ttt.items() if k != "trace_every_8"}}),
              file=sys.stderr)
    rows = []
    for T in args.budgets:
        n_p, t_p = _timed(ft, T, args.plain_batch, 0)
        e_p = _errors(ft.image(), ref)
        guide.reset(seed=args.seed)
        guide.configure(train=True, records_per_step=args.records, lr=args.lr)
        n_g, t_g = _timed(ft, T, args.guided_batch, LUC_FLAG_GUIDED)
        e_g = _errors(ft.image(), ref)
        st = guide.stats()
        rows.append({"seconds": T,
                     "plain": {"spp": n_p, "elapsed_s": round(t_p, 3), **e_p},
                     "guided": {"spp": n_g, "elapsed_s": round(t_g, 3), "steps": st.steps,
                                "last_loss": st.last_loss, "last_records": st.last_records, **e_g},
                     "mse_ratio_plain_over_guided": e_p["mse"] / max(e_g["mse"], 1e-300),
                     "relmse_ratio_plain_over_guided": e_p["relmse"] / max(e_g["relmse"], 1e-300)})
        print(json.dumps(rows[-1]), file=sys.stderr)
    out = {"workload": f"guided-room {args.width}x{args.height} d{args.depth} ({len(scene.triangles)} triangles)",
           "ref_spp": args.ref_spp, "ref_seconds": ref_seconds, "ref_mean": float(ref.mean()),
           "records_per_step": args.records, "lr": args.lr, "time_to_target": ttt, "budgets": rows}
    line = json.dumps(out)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")
    gpu.close()


if __name__ == "__main__":
    main()
