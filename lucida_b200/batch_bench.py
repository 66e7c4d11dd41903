"""Uneven multi-scene batch: aggregate throughput and per-scene completion.

    python -m lucida_b200.batch_bench [--scenes 64] [--tune-waves 2] [--sequential] [--out JSON]

Workload (scenes.batch_workload): 64 scenes of the displaced-spheres recipe,
triangle counts log-uniform in [10k, 2M], resolution from {256^2, 512^2,
1024^2, 1920x1080}, spp from {4, 8, 16, 32, 64}, 4-12 bounces, all seeded.
Every scene is resident in its own context (device LBVH); the batch renders
through one shared pool as one CUDA graph after the autotuner has picked the
traversal launch shape on the first waves. --sequential also times the same
jobs one at a time through the same pool for comparison. Device time, CUDA
events; one JSON line.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import batch as B
from . import scenes
from .gpu import Gpu, RenderParams


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--scenes", type=int, default=64)
    ap.add_argument("--seed", type=int, default=4096)
    ap.add_argument("--tune-waves", type=int, default=2)
    ap.add_argument("--sequential", action="store_true")
    ap.add_argument("--out", default=None)
    return ap.parse_args(argv)


def main(argv=None):
    import torch
    args = parse(argv)
    t0 = time.time()
    spec = scenes.batch_workload(num_scenes=args.scenes, seed=args.seed)
    gen_s = time.time() - t0
    torch.cuda.init()
    runner = Gpu(0)
    ctxs, jobs = [], []
    t0 = time.time()
    for k, (sc, w, h, spp, depth) in enumerate(spec):
        g = Gpu(0)
        g.upload(sc)
        ctxs.append(g)
        p = RenderParams(width=w, height=h, samples=spp, max_depth=depth, sampler="sobol", frame_seed=0x5EED + k)
        jobs.append(B.BatchJob(g, sc, p, torch.zeros(w * h * 16, dtype=torch.float32, device="cuda")))
    torch.cuda.synchronize()
    upload_s = time.time() - t0
    t0 = time.time()
    best, tried = B.autotune(runner, jobs, waves=args.tune_waves)
    tune_s = time.time() - t0
    for j in jobs:
        j.accum.zero_()
    torch.cuda.synchronize()
    done, st = B.render_batch(runner, jobs)
    paths = int(st.paths)
    out = {"metric": "Mpaths/s", "value": paths / st.ms_total / 1e3, "unit": "Mpaths/s",
           "workload": f"{args.scenes} scenes, {sum(len(s.triangles) for s, *_ in spec)} triangles in total, "
                       f"{paths} paths", "batch_ms": st.ms_total, "autotune": {"best": list(best), "tried": tried,
                                                                             "seconds": round(tune_s, 2)},
           "per_scene": [{"triangles": len(s.triangles), "width": w, "height": h, "spp": spp, "bounces": d,
                          "done_ms": float(t)} for (s, w, h, spp, d), t in zip(spec, done)],
           "rays_extend": int(st.rays_extend), "rays_shadow": int(st.rays_shadow),
           "scene_generation_s": round(gen_s, 1), "upload_and_lbvh_s": round(upload_s, 1)}
    if args.sequential:
        # The same jobs one at a time through the same pool (a batch of one
        # each): what rendering the scenes back to back costs.
        total = 0.0
        for j in jobs:
            j.accum.zero_()
            _, s1 = B.render_batch(runner, [j])
            total += s1.ms_total
        out["sequential_ms"] = total
        out["sequential_Mpaths_s"] = paths / total / 1e3
    line = json.dumps(out)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")
    for g in ctxs:
        g.close()
    runner.close()


if __name__ == "__main__":
    main(sys.argv[1:])
