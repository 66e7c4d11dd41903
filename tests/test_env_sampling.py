"""Environment importance sampling on the GPU (EnvMap::sample,
envmap.rs:235-275, through luc_eval_env) against the oracle's restatement.

Inputs: random pairs plus the edges of the two CDF searches
(envmap.rs:290-317) — 0, 1, values outside [0, 1), and k/256 with the
floats either side of it. Each sample must land in the oracle's texel
(radiance and pdf bit for bit) at the oracle's direction (the oracle's
sin/cos come from the host libm, the device's from its own restatement: a
few ulps). A CDF that is not non-decreasing is searched the same way too
(the halving search's probe order decides the cell there).
"""
import numpy as np
import pytest

import oracle as O
from tests.bridge import oracle_from_scene, scene_from_oracle


def _inputs():
    rng = np.random.default_rng(7)
    u = rng.random((20000, 2), dtype=np.float32)
    k = np.arange(257, dtype=np.float32) / np.float32(256)
    edges = np.concatenate([k, np.nextafter(k, np.float32(-1)), np.nextafter(k, np.float32(2)),
                            np.float32([0.0, 1.0, 1.0 - 2.0 ** -24, -0.25, 1.5])]).astype(np.float32)
    g = np.stack(np.meshgrid(edges, edges[::7]), -1).reshape(-1, 2)
    return np.concatenate([u, g, g[:, ::-1]]).astype(np.float32)


def _check(gpu_out, ref_out):
    d, r, p = gpu_out
    rd, rr, rp = ref_out
    np.testing.assert_array_equal(r, rr)
    np.testing.assert_array_equal(p, rp)
    np.testing.assert_allclose(d, rd, rtol=0, atol=2e-6)


@pytest.fixture(scope="module")
def gpu():
    import lucida_b200 as lb
    g = lb.Gpu(0)
    yield g
    g.close()


@pytest.mark.gpu
def test_env_sample_matches_the_oracle(gpu):
    s = scene_from_oracle(O.Scene.builtin("sunset"))
    assert s.env_cdf is not None
    gpu.upload(s, force=True)
    u = _inputs()
    _check(gpu.env_sample(u), oracle_from_scene(s).env_sample(u))


@pytest.mark.gpu
def test_env_sample_on_a_row_that_is_not_monotone(gpu):
    s = scene_from_oracle(O.Scene.builtin("sunset"))
    h, w = s.env_pixels.shape[0], s.env_pixels.shape[1]
    cdf = s.env_cdf.copy()
    j = h // 2
    row = cdf[j, :w + 1]
    a, b = w // 3, 2 * w // 3
    row[a], row[b] = row[b], row[a]  # a decreasing pair inside one conditional row
    assert np.any(np.diff(row) < 0)
    cdf[h, h // 3], cdf[h, h // 3 + 1] = cdf[h, h // 3 + 1], cdf[h, h // 3]  # and in the marginal
    s.env_cdf = cdf
    gpu.upload(s, force=True)
    u = _inputs()
    _check(gpu.env_sample(u), oracle_from_scene(s).env_sample(u))
