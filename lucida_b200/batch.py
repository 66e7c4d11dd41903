"""Batched multi-scene rendering (no counterpart in Lucida's pt_gpu, which
renders one scene per call) over luc_render_batch / luc_batch_autotune.

    jobs = [BatchJob(gpu_i, scene_i, params_i, accum_i), ...]   # gpu_i holds scene_i
    done_ms, stats = render_batch(runner, jobs)
    best, tried = autotune(runner, jobs, waves=2)

Every job's scene lives in its own context (`Gpu`, same device); the batch
runs in `runner`'s context and pool. Accumulators are device buffers (torch
tensors of width*height*16 float32), accumulated into like luc_render.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from .gpu import Gpu, RenderParams, SceneDef, build_uniforms
from .native import BatchConfig, BatchJob as _Job, RenderStats, check, lib


@dataclass
class BatchJob:
    gpu: Gpu              # context whose resident scene is `scene`
    scene: SceneDef
    params: RenderParams
    accum: object         # device buffer with .data_ptr() (torch) or an int address


def _jobs(jobs):
    arr = (_Job * len(jobs))()
    for k, j in enumerate(jobs):
        j.gpu.upload(j.scene)
        arr[k].scene = j.gpu.handle
        arr[k].uniforms = build_uniforms(j.scene, j.params)
        arr[k].spp = j.params.samples
        arr[k].max_depth = j.params.max_depth
        arr[k].accum_dev = j.accum if isinstance(j.accum, int) else j.accum.data_ptr()
    return arr


def configure(runner: Gpu, block: int = 128, chunk: int = 32):
    cfg = BatchConfig(block, chunk)
    check(runner.handle, lib().luc_batch_configure(runner.handle, C.byref(cfg)))


def render_batch(runner: Gpu, jobs: list[BatchJob]):
    """Returns (per-job completion time in ms from the batch's start, RenderStats)."""
    arr = _jobs(jobs)
    done = np.zeros(len(jobs), np.float64)
    st = RenderStats()
    check(runner.handle, lib().luc_render_batch(runner.handle, arr, len(jobs), done.ctypes.data_as(C.c_void_p),
                                                C.byref(st)))
    return done, st


def autotune(runner: Gpu, jobs: list[BatchJob], waves: int = 2):
    """Time every launch shape on the first `waves` waves; the fastest becomes
    the runner's configuration. Returns ((block, chunk), [(block, chunk, ms)])."""
    arr = _jobs(jobs)
    best = BatchConfig()
    tried = np.zeros((12, 3), np.float64)
    check(runner.handle, lib().luc_batch_autotune(runner.handle, arr, len(jobs), int(waves), C.byref(best),
                                                  tried.ctypes.data_as(C.c_void_p)))
    return (best.block, best.chunk), [(int(b), int(c), float(ms)) for b, c, ms in tried]
