"""Sample-range sharding of one frame over several GPUs (one process per GPU).

Rank r of N renders samples [r*spp, (r+1)*spp) of every pixel into its own
accumulator: `shard_params` sets that range (RenderParams.sample_offset).
The RNG is a pure function of (frame, pixel, sample) (crates/core/src/
rng.rs:18-21) and accumulation is additive (crates/gpu/tests/
cpu_gpu_agreement.rs:119-168), so the frame's accumulator is the field-wise
sum of the ranks'. `merge_accumulators` is that exchange, done as a
reduce-scatter then an all-gather so that each rank moves about two
accumulators' worth of bytes whatever N is (all-gathering every rank's whole
accumulator moves N - 1): an all-to-all gives rank r the r-th pixel slice of
every rank's accumulator (torch.distributed; NCCL over NVLink on GPUs),
rank r sums them in rank order (luc_accum_merge), and an all-gather of the
summed slices gives every rank the frame. The fixed rank-order sum keeps
the merged image independent of the collectives' schedules.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

from .native import check, lib

__all__ = ["shard_params", "merge_accumulators"]


def shard_params(params, rank: int):
    """The RenderParams of rank `rank`'s shard: the same frame, samples
    [rank*spp, (rank+1)*spp) after the params' own sample_offset."""
    return dataclasses.replace(params, sample_offset=params.sample_offset + rank * params.samples)


def _sum_on_device(gpu, parts, out):
    n, pixels = parts.shape[0], parts.shape[1] // 16
    check(gpu.handle, lib().luc_accum_merge(gpu.handle, C.c_void_p(parts.data_ptr()), n, pixels,
                                            C.c_void_p(out.data_ptr())))


def merge_accumulators(accum, gpu=None, group=None, sum_parts=None):
    """Sum every rank's accumulator into `accum` (in place) and return it.

    accum: a contiguous float32 torch tensor of pixels * 16 floats (GpuAccum
    records) — on the rank's CUDA device, with `gpu` the rank's Gpu whose
    stream the sum runs on (the caller's torch stream must be that stream or
    be synchronised with it). Every rank of `group` must call this with the
    same shape, in the same order relative to its other collectives. With one
    rank (or no process group) it returns `accum` unchanged.

    sum_parts(parts, out): the rank-order sum of the gathered (N, pixels*16)
    array into `out`; defaults to the device kernel (CUDA tensors only)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    if world == 1:
        return accum
    if accum.dtype != torch.float32 or not accum.is_contiguous() or accum.numel() % 16:
        raise ValueError("accum must be a contiguous float32 tensor of GpuAccum records (16 floats each)")
    if sum_parts is None:
        if not accum.is_cuda or gpu is None:
            raise ValueError("the device merge needs a CUDA accumulator and its Gpu")
        sum_parts = lambda parts, out: _sum_on_device(gpu, parts, out)  # noqa: E731
    pixels = accum.numel() // 16
    per = -(-pixels // world)  # pixels of each rank's slice (the last padded with zero records)
    whole = accum.view(-1)
    if per * world != pixels:
        whole = torch.zeros(per * world * 16, dtype=accum.dtype, device=accum.device)
        whole[:accum.numel()].copy_(accum.view(-1))
    parts = torch.empty(world * per * 16, dtype=accum.dtype, device=accum.device)
    dist.all_to_all_single(parts, whole, group=group)  # parts[k] = rank k's copy of this rank's slice
    mine = torch.empty(per * 16, dtype=accum.dtype, device=accum.device)
    sum_parts(parts.view(world, per * 16), mine)
    dist.all_gather_into_tensor(whole, mine, group=group)
    if whole.data_ptr() != accum.data_ptr():
        accum.view(-1).copy_(whole[:accum.numel()])
    return accum
