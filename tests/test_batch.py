"""Batched multi-scene rendering (luc_render_batch, luc_batch_autotune).

A batched job must produce exactly the accumulator a single-scene render of
the same job produces: every path's computation depends only on its scene,
pixel and sample (the sample index comes from the path's wave segment, never
from its queue position), and RESOLVE adds a segment's samples in sample
order, wave after wave. So each job of a mixed batch — different scenes,
sizes, spp, bounces and samplers, split across several waves of a small
pool — is compared bit for bit with luc_render, under every launch shape the
autotuner tries.
"""
import os

import numpy as np
import pytest

import lucida_b200 as lb
from lucida_b200 import batch as B, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def runner():
    os.environ["LUC_PATH_BUDGET"] = str(40_000)  # forces several waves and split jobs
    g = lb.Gpu(0)
    del os.environ["LUC_PATH_BUDGET"]
    yield g
    g.close()


@pytest.fixture(scope="module")
def workload():
    spec = scenes.batch_workload(num_scenes=5, tri_range=(1_000, 12_000), seed=11, level=2,
                                 resolutions=((64, 48), (96, 64), (80, 80)), spp_choices=(2, 3, 5),
                                 depth_range=(3, 7), env_size=(64, 32))
    gpus = [lb.Gpu(0) for _ in spec]
    jobs = []
    for k, ((sc, w, h, spp, depth), g) in enumerate(zip(spec, gpus)):
        sampler = "sobol" if k % 2 == 0 else "independent"
        sampling = ("mis", "nee", "bsdf")[k % 3]
        p = lb.RenderParams(width=w, height=h, samples=spp, max_depth=depth, sampler=sampler, sampling=sampling,
                            frame_seed=0x1234 + k, sample_offset=k)
        g.upload(sc)
        jobs.append((g, sc, p))
    yield jobs
    for g in gpus:
        g.close()


def _single(job):
    g, sc, p = job
    return lb.render_accum(g, sc, p).reshape(-1)


def _batch(runner, jobs):
    import torch
    acc = [torch.zeros(p.width * p.height * 16, dtype=torch.float32, device="cuda") for _, _, p in jobs]
    done, st = B.render_batch(runner, [B.BatchJob(g, sc, p, a) for (g, sc, p), a in zip(jobs, acc)])
    torch.cuda.synchronize()
    return [a.cpu().numpy().view(lb.layout.ACCUM) for a in acc], done, st


def test_batched_jobs_equal_single_renders(runner, workload):
    ref = [_single(j) for j in workload]
    outs, done, st = _batch(runner, workload)
    for k, (o, r) in enumerate(zip(outs, ref)):
        assert o.tobytes() == r.tobytes(), f"job {k}"
    assert st.paths == sum(p.width * p.height * p.samples for _, _, p in workload)
    assert np.all(done > 0) and np.all(np.diff(done) >= 0)  # jobs finish in order


def test_every_launch_shape_gives_the_same_images(runner, workload):
    ref = [_single(j) for j in workload]
    for block in (64, 128, 256):
        for chunk in (32, 1024, 4096):
            B.configure(runner, block, chunk)
            outs, _, _ = _batch(runner, workload)
            for k, (o, r) in enumerate(zip(outs, ref)):
                assert o.tobytes() == r.tobytes(), (block, chunk, k)
    B.configure(runner)


def test_autotune_leaves_accumulators_untouched(runner, workload):
    import torch
    acc = [torch.full((p.width * p.height * 16,), 7.0, dtype=torch.float32, device="cuda") for _, _, p in workload]
    best, tried = B.autotune(runner, [B.BatchJob(g, sc, p, a) for (g, sc, p), a in zip(workload, acc)], waves=2)
    torch.cuda.synchronize()
    assert all(bool((a == 7.0).all()) for a in acc)
    assert best in [(b, c) for b, c, _ in tried] and all(ms > 0 for _, _, ms in tried)
    print("autotune:", best, tried)
    B.configure(runner)


def test_batch_validation(runner, workload):
    g, sc, p = workload[0]
    import torch
    a = torch.zeros(16, device="cuda")
    bad = lb.RenderParams(width=p.width, height=p.height, samples=0, max_depth=3)
    with pytest.raises(lb.GpuError):
        B.render_batch(runner, [B.BatchJob(g, sc, bad, a)])
    with pytest.raises(lb.GpuError):
        B.configure(runner, 96, 32)
