"""Wavefront against megakernel on the benchmark's configurations.

    python -m lucida_b200.arch_bench [--iters 3] [--out JSON]

C1: the analytic Cornell box (8 primitives, no BVH), 512 x 512, 64 spp,
8 bounces, independent sampler, MIS. C2: the displaced-sphere scene
(1,310,720 triangles, device LBVH collapsed to the wide tree), 1024 x 1024,
16 spp, 8 bounces, Sobol, MIS. Both architectures render into a device
accumulator; device time of luc_render (CUDA events inside the library),
best of --iters after one warm-up; Mpaths/s = W * H * spp / s. The two
accumulators are compared bit for bit. One JSON line.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys

from . import scenes
from .gpu import ARCHITECTURES, Gpu, RenderParams, build_uniforms
from .native import check, lib


def run(gpu, scene, p, arch, iters, accum):
    import torch
    gpu.upload(scene)
    u = build_uniforms(scene, p)
    best = None
    for k in range(iters + 1):
        accum.zero_()
        torch.cuda.synchronize()
        check(gpu.handle, lib().luc_render(gpu.handle, C.byref(u), p.samples, p.max_depth, ARCHITECTURES[arch],
                                           None, C.c_void_p(accum.data_ptr())))
        ms = gpu.stats().ms_total
        if k > 0:
            best = ms if best is None else min(best, ms)
    return best, accum.clone()


def main(argv=None):
    import torch
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--iters", type=int, default=3)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    gpu = Gpu(0)
    gpu.set_stream(0)
    cases = {
        "C1 cornell-analytic 512x512 64spp d8": (scenes.cornell_analytic(),
                                                 RenderParams(width=512, height=512, samples=64, max_depth=8,
                                                              sampler="independent")),
        "C2 displaced-spheres 1024x1024 16spp d8": (scenes.displaced_spheres(),
                                                    RenderParams(width=1024, height=1024, samples=16, max_depth=8)),
    }
    out = {"metric": "Mpaths/s", "cases": {}}
    for name, (scene, p) in cases.items():
        acc = torch.zeros(p.width * p.height * 16, dtype=torch.float32, device="cuda")
        res = {}
        images = {}
        for arch in ("wavefront", "megakernel"):
            ms, img = run(gpu, scene, p, arch, args.iters, acc)
            res[arch] = {"ms": ms, "Mpaths_s": p.width * p.height * p.samples / ms / 1e3}
            images[arch] = img
        res["identical"] = bool(torch.equal(images["wavefront"], images["megakernel"]))
        out["cases"][name] = res
    line = json.dumps(out)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")
    gpu.close()


if __name__ == "__main__":
    main(sys.argv[1:])
