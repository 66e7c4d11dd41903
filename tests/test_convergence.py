"""Convergence meter (luc_convergence / LUC_FLAG_MEASURE), after the
reference's crates/gpu/tests/convergence.rs: the figure is the documented
formula over the accumulator, falls with the sample count near 1/sqrt(N),
separates a worse sampling strategy, agrees between the architectures,
matches the measured spread of sixteen independent renders with the
independent sampler, and over-reports (never under-reports) with Sobol.
"""
import math

import numpy as np
import pytest

import lucida_b200 as lb
import oracle as O
from tests.bridge import scene_from_oracle

pytestmark = pytest.mark.gpu

LUM = np.array([0.2126, 0.7152, 0.0722])


@pytest.fixture(scope="module")
def gpu():
    g = lb.Gpu(0)
    yield g
    g.close()


@pytest.fixture(scope="module")
def box():
    return scene_from_oracle(O.Scene.builtin("cornell-box"))


def params(spp, **kw):  # convergence.rs:26-33
    return lb.RenderParams(width=96, height=96, samples=spp, max_depth=5, **kw)


def meter_restated(acc):
    """convergence.wgsl:81-108 in float64."""
    n = acc["samples"].astype(np.float64)
    rad = acc["radiance"].astype(np.float64)
    sq = acc["radiance_sq"].astype(np.float64)
    ok = n >= 2
    mean = rad[ok] / n[ok, None]
    ml = mean @ LUM
    keep = ml > 1e-3
    var = np.maximum(sq[ok][keep] / n[ok][keep, None] - mean[keep] ** 2, 0.0)
    se = np.sqrt((var @ LUM) / n[ok][keep])
    return float(np.mean(se / ml[keep])) if keep.any() else -1.0


def test_meter_is_the_documented_formula(gpu, box):
    import torch
    acc = lb.render_accum(gpu, box, params(64), measure=True).reshape(-1)
    reported = gpu.stats().convergence
    ref = meter_restated(acc)
    assert abs(reported - ref) <= 1e-3 * ref, (reported, ref)  # float32 sums vs float64
    # The standalone entry point over a device accumulator gives the same figure.
    dev = torch.from_numpy(acc.view(np.float32).reshape(-1).copy()).cuda()
    assert lb.convergence(gpu, dev, len(acc)) == pytest.approx(reported, rel=0, abs=0)


def test_nothing_measurable_reports_minus_one(gpu, box):
    lb.render_accum(gpu, box, params(1), measure=True)
    assert gpu.stats().convergence == -1.0
    lb.render_accum(gpu, box, params(4))
    assert gpu.stats().convergence == -1.0  # not requested


def test_readout_falls_with_sample_count(gpu, box):  # convergence.rs:45-85
    first, prev = None, math.inf
    for spp in (16, 64, 256, 1024):
        e = lb.measure_convergence(gpu, box, params(spp))
        assert e > 0.0
        model = e if first is None else first[1] * math.sqrt(first[0] / spp)
        first = first or (spp, e)
        print(spp, e, e / model)
        assert e < prev
        prev = e
    expected = first[1] * math.sqrt(first[0] / 1024)
    assert 0.5 * expected < prev < 2.0 * expected


def test_worse_strategy_reports_more_error(gpu, box):  # convergence.rs:102-118
    good = lb.measure_convergence(gpu, box, params(64, sampling="mis"))
    bad = lb.measure_convergence(gpu, box, params(64, sampling="bsdf"))
    print("mis", good, "bsdf", bad)
    assert bad > 1.5 * good


def test_both_architectures_report_the_same(gpu, box):  # convergence.rs:130-145
    _, mega = lb.render_with_measured(gpu, box, params(64), "megakernel")
    _, wave = lb.render_with_measured(gpu, box, params(64), "wavefront")
    assert mega == wave  # one shading function, one accumulation order


def _spread(gpu, s, p, runs=16):  # convergence.rs:148-192
    sums, sq = 0.0, 0.0
    for k in range(runs):
        q = lb.RenderParams(**{**p.__dict__, "frame_seed": (p.frame_seed + k * 0x9E3779B9) & 0xFFFFFFFF})
        f = lb.render_with(gpu, s, q, "megakernel").data.astype(np.float64).reshape(-1, 3)
        sums = sums + f
        sq = sq + f * f
    mean = sums / runs
    ml = mean @ LUM
    keep = ml > 1e-3
    var = np.maximum((sq / runs - mean ** 2) * (runs / (runs - 1)), 0.0)
    c4 = math.sqrt(2.0 / (runs - 1)) * math.exp(math.lgamma(runs / 2) - math.lgamma((runs - 1) / 2))
    return float(np.mean(np.sqrt(np.maximum(var[keep] @ LUM, 0.0)) / c4 / ml[keep]))


def test_readout_matches_spread_of_independent_renders(gpu, box):  # convergence.rs:220-239
    p = params(64, sampler="independent")
    reported = lb.measure_convergence(gpu, box, p)
    actual = _spread(gpu, box, p)
    print("independent: meter", reported, "spread", actual, reported / actual)
    assert 0.80 < reported / actual < 1.25


def test_stratification_makes_the_readout_conservative(gpu, box):  # convergence.rs:249-267
    p = params(64, sampler="sobol")
    reported = lb.measure_convergence(gpu, box, p)
    actual = _spread(gpu, box, p)
    print("sobol: meter", reported, "spread", actual, reported / actual)
    assert reported >= 0.95 * actual
