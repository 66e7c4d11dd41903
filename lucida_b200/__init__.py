"""lucida_b200 — Lucida's light-transport hot path on NVIDIA B200 (sm_100a).

A wavefront path integrator (camera rays, BVH extend, GGX/dielectric shading
with NEE + MIS, shadow connect, compacted SoA queues), a GPU LBVH builder and
an edge-avoiding à-trous denoiser, and a learned path-guiding proposal (a
BF16 tensor-core MLP trained online), written as CUDA kernels behind the C ABI
declared in include/luc_cuda.h (liblucida_cuda.so), with this package as the
Python-side mirror of Lucida's `pt_gpu` API.
"""
from .gpu import (Camera, DenoiseParams, Denoiser, Film, Gpu, GpuBuildOutput, GpuError, LbvhBuilder, RenderParams,
                  SceneDef, accum_to_film, build_uniforms, convergence, measure_convergence, render_accum,
                  render_native_denoised, render_native_on, render_with, render_with_measured)
from .guide import Guide, records_array

__all__ = ["Camera", "DenoiseParams", "Denoiser", "Film", "Gpu", "GpuBuildOutput", "GpuError", "LbvhBuilder",
           "RenderParams", "SceneDef", "accum_to_film", "build_uniforms", "render_accum", "render_native_denoised",
           "render_native_on", "render_with", "render_with_measured", "measure_convergence", "convergence", "Guide",
           "records_array"]
