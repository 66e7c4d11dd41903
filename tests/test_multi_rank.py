"""Two ranks over gloo on the CPU: the sample-range sharding `bench.py
--gpus N` runs (one process per GPU, rank r renders samples
[r*spp, (r+1)*spp) of every pixel, no exchange on the data path).

The reference's RNG is a pure function of (frame, pixel, sample)
(crates/core/src/rng.rs:18-21) and a progressive render equals a one-shot
render (crates/gpu/tests/cpu_gpu_agreement.rs:119-168), so the ranks'
accumulators summed equal one render of world*spp samples. The oracle plays
each rank's renderer here; the GPU renderer's offset handling is pinned
against the oracle in test_render_parity. Also covers bench.py's timing
helpers (barrier, max over ranks) on a gloo group.
"""
import datetime
import os
import socket

import numpy as np
import pytest

WORLD = 2
SPP = 2
W, H, DEPTH = 24, 16, 4


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(WORLD), LOCAL_RANK=str(rank))
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import oracle as O
        osc = O.Scene.builtin("cornell-box")
        u = osc.uniforms(W, H, SPP, DEPTH, sample_offset=rank * SPP, sampler=1)
        part = torch.from_numpy(osc.render_sums(u, threads=2)[:, :6].astype(np.float64))
        dist.all_reduce(part)  # what a user merging the replicas would run once, after the frames
        bench.barrier(WORLD)
        slowest = bench.max_over_ranks(10.0 + rank, WORLD)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), part.numpy())
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(repr(slowest))
    finally:
        dist.destroy_process_group()


def test_sample_range_shards_sum_to_the_one_shot_render(tmp_path):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, str(tmp_path))) for r in range(WORLD)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert [p.exitcode for p in procs] == [0] * WORLD

    import oracle as O
    osc = O.Scene.builtin("cornell-box")
    whole = osc.render_sums(osc.uniforms(W, H, WORLD * SPP, DEPTH, sampler=1), threads=2)[:, :6].astype(np.float64)
    for r in range(WORLD):
        merged = np.load(tmp_path / f"rank{r}.npy")
        # float32 partial sums in two halves vs one sequential float32 sum
        np.testing.assert_allclose(merged, whole, rtol=1e-5, atol=1e-6)
        assert float((tmp_path / f"rank{r}.txt").read_text()) == 10.0 + WORLD - 1
    # the shards are disjoint: each rank alone is not the whole
    half = osc.render_sums(osc.uniforms(W, H, SPP, DEPTH, sampler=1), threads=2)[:, :6]
    assert not np.allclose(half, whole)
