"""Two ranks over gloo on the CPU: the sample-range sharding `bench.py
--gpus N` runs (one process per GPU, rank r renders samples
[r*spp, (r+1)*spp) of every pixel) and the product's one exchange,
lucida_b200.shards.merge_accumulators (an all-to-all of pixel slices, each
rank's rank-order sum of its slice, an all-gather of the sums).

The reference's RNG is a pure function of (frame, pixel, sample)
(crates/core/src/rng.rs:18-21) and a progressive render equals a one-shot
render (crates/gpu/tests/cpu_gpu_agreement.rs:119-168), so the ranks'
accumulators summed equal one render of world*spp samples. With no GPU here
the oracle plays each rank's renderer and the rank-order sum runs on the
host; the device sum (luc_accum_merge) is pinned in test_shards_merge on a
GPU, and the GPU renderer's offset handling against the oracle in
test_render_parity. Also covers bench.py's timing helpers (barrier, max over
ranks) on a gloo group.
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


def _as_accum(sums, spp):
    """The oracle's per-pixel sums packed as GpuAccum records."""
    import lucida_b200 as lb
    a = np.zeros(len(sums), lb.layout.ACCUM)
    a["radiance"], a["radiance_sq"], a["albedo"] = sums[:, 0:3], sums[:, 3:6], sums[:, 6:9]
    a["normal"], a["depth"], a["samples"] = sums[:, 9:12], sums[:, 12], spp
    return a


def _rank_order_sum(parts, out):
    """The device merge's arithmetic on the host: parts[0] + parts[1] + ...,
    float32, rank order."""
    acc = parts[0].numpy().copy()
    for r in range(1, parts.shape[0]):
        acc += parts[r].numpy()
    out.copy_(__import__("torch").from_numpy(acc))


def _rank_main(rank, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(WORLD), LOCAL_RANK=str(rank))
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        import oracle as O
        import lucida_b200 as lb
        from lucida_b200.shards import merge_accumulators, shard_params
        osc = O.Scene.builtin("cornell-box")
        p = shard_params(lb.RenderParams(width=W, height=H, samples=SPP, max_depth=DEPTH), rank)
        assert p.sample_offset == rank * SPP
        u = osc.uniforms(W, H, SPP, DEPTH, sample_offset=p.sample_offset, sampler=1)
        acc = torch.from_numpy(_as_accum(osc.render_sums(u, threads=2), SPP).view(np.float32).reshape(-1).copy())
        np.save(os.path.join(out_dir, f"part{rank}.npy"), acc.numpy())
        merge_accumulators(acc, sum_parts=_rank_order_sum)
        bench.barrier(WORLD)
        slowest = bench.max_over_ranks(10.0 + rank, WORLD)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), acc.numpy())
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
    import lucida_b200 as lb
    osc = O.Scene.builtin("cornell-box")
    whole = _as_accum(osc.render_sums(osc.uniforms(W, H, WORLD * SPP, DEPTH, sampler=1), threads=2), WORLD * SPP)
    parts = [np.load(tmp_path / f"part{r}.npy") for r in range(WORLD)]
    expect = parts[0].copy()
    for r in range(1, WORLD):
        expect += parts[r]
    for r in range(WORLD):
        merged = np.load(tmp_path / f"rank{r}.npy")
        assert np.array_equal(merged, expect)  # every rank holds the same rank-order sum
        m = merged.view(lb.layout.ACCUM)
        assert np.all(m["samples"] == WORLD * SPP)
        for f in ("radiance", "radiance_sq", "albedo", "normal", "depth"):
            # float32 partial sums in two halves vs one sequential float32 sum
            np.testing.assert_allclose(m[f], whole[f], rtol=1e-5, atol=1e-6)
        assert float((tmp_path / f"rank{r}.txt").read_text()) == 10.0 + WORLD - 1
    # the shards are disjoint: each rank alone is not the whole
    assert not np.allclose(parts[0].view(lb.layout.ACCUM)["radiance"], whole["radiance"])


def _merge_only_main(rank, world, port, pixels, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from lucida_b200.shards import merge_accumulators
        rng = np.random.default_rng(100 + rank)
        acc = torch.from_numpy(rng.standard_normal(pixels * 16).astype(np.float32))
        np.save(os.path.join(out_dir, f"in{rank}.npy"), acc.numpy())
        merge_accumulators(acc, sum_parts=_rank_order_sum)
        np.save(os.path.join(out_dir, f"out{rank}.npy"), acc.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,pixels", [(3, 7), (3, 1), (4, 12)])
def test_merge_with_slices_that_do_not_divide_the_frame(tmp_path, world, pixels):
    """Pixel counts that leave the last rank's slice short (or some ranks
    with none): every rank still ends with the exact rank-order sum."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_merge_only_main, args=(r, world, port, pixels, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert [p.exitcode for p in procs] == [0] * world
    expect = np.load(tmp_path / "in0.npy")
    for r in range(1, world):
        expect = expect + np.load(tmp_path / f"in{r}.npy")
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"out{r}.npy"), expect)
