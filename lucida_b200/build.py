"""Build liblucida_cuda.so in-tree for sm_100a.

Every translation unit is compiled by nvcc for `-gencode
arch=compute_100a,code=sm_100a` and linked with the static CUDA runtime into
lucida_b200/liblucida_cuda.so, which the package loads with ctypes.

Numerical flags: --fmad=false (no a*b+c contraction: the reference's Rust
never contracts), -prec-div=true -prec-sqrt=true (IEEE division and square
root), and -ffp-contract=off for the host-side C++ (the energy table and the
environment row table are computed on the host).
"""
from __future__ import annotations

import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "liblucida_cuda.so")
BUILD = os.path.join(HERE, "_build")
SOURCES = ["capi.cu", "wavefront.cu", "lbvh.cu", "denoise.cu", "sort_static.cu", "eval.cu", "guide.cu", "instances.cu", "batch.cu", "wide.cu", "megakernel.cu", "stats.cu", "guide_tc.cu", "shards.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-prec-div=true", "-prec-sqrt=true",
         "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers += [os.path.join(HERE, "..", "include", f) for f in ("lucida_layout.h", "luc_cuda.h")]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if _stale(o, [s] + headers) or ptxas_info:
            cmd = [nvcc()] + ARCH + FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + ["-dc", s, "-o", o]
            t0 = time.time()
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
            if verbose or ptxas_info:
                print(f"[build] {src} {time.time() - t0:.1f}s", file=sys.stderr)
                if r.stderr.strip():
                    print(r.stderr, file=sys.stderr)
    if _stale(OUT, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", OUT] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
