"""The device half of the shard merge (luc_accum_merge): gathered per-rank
accumulators summed in rank order. The exchange itself (the all-gather) runs
on gloo ranks in test_multi_rank; here one process stands for the ranks.
"""
import numpy as np
import pytest

import lucida_b200 as lb
from lucida_b200 import scenes
from lucida_b200.shards import _sum_on_device, shard_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = lb.Gpu(0)
    yield g
    g.close()


@pytest.mark.parametrize("nparts,pixels", [(1, 5), (2, 1), (3, 4097), (8, 1 << 16)])
def test_rank_order_sum_is_exact(gpu, nparts, pixels):
    import torch
    rng = np.random.default_rng(nparts * 7 + pixels)
    parts = rng.standard_normal((nparts, pixels * 16)).astype(np.float32) * 1e3
    expect = parts[0].copy()
    for r in range(1, nparts):
        expect += parts[r]
    dev = torch.from_numpy(parts).cuda()
    out = torch.full((pixels * 16,), float("nan"), dtype=torch.float32, device="cuda")
    _sum_on_device(gpu, dev, out)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), expect)
    _sum_on_device(gpu, dev, dev[0])  # in place onto the first part
    torch.cuda.synchronize()
    assert np.array_equal(dev[0].cpu().numpy(), expect)


def test_shards_merge_to_the_one_shot_render(gpu):
    """Two sample-range shards rendered on the device and merged equal a
    one-shot render of both ranges to float32 summation order."""
    import torch
    s = scenes.cornell_analytic()
    base = lb.RenderParams(width=64, height=48, samples=4, max_depth=6, sampler="sobol")
    parts = [lb.render_accum(gpu, s, shard_params(base, r)).reshape(-1) for r in range(2)]
    whole = lb.render_accum(gpu, s, lb.RenderParams(width=64, height=48, samples=8, max_depth=6,
                                                    sampler="sobol")).reshape(-1)
    dev = torch.from_numpy(np.stack([p.view(np.float32).reshape(-1) for p in parts])).cuda()
    out = torch.empty(dev.shape[1], dtype=torch.float32, device="cuda")
    _sum_on_device(gpu, dev, out)
    torch.cuda.synchronize()
    m = out.cpu().numpy().view(lb.layout.ACCUM)
    assert np.all(m["samples"] == 8)
    for f in ("radiance", "radiance_sq", "albedo", "normal", "depth"):
        np.testing.assert_allclose(m[f], whole[f], rtol=1e-5, atol=1e-6)
    assert not np.allclose(parts[0]["radiance"], whole["radiance"])
