"""The oracle's à-trous denoiser against the behaviours crates/core/src/
denoise.rs:238-431 asserts (restated). CPU only."""
import numpy as np

import oracle as O

W = H = 32


def guides(normal=(0.0, 0.0, 1.0), depth=5.0, albedo=0.5):
    n = W * H
    return (np.full((n, 3), albedo, np.float32), np.tile(np.asarray(normal, np.float32), (n, 1)),
            np.full(n, depth, np.float32))


def test_a_constant_image_is_unchanged():
    a, n, d = guides()
    film = np.full((W * H, 3), 0.7, np.float32)
    out = O.denoise(film, a, n, d, W, H)
    np.testing.assert_allclose(out, film, rtol=1e-5)


def test_zero_iterations_is_a_no_op():
    rng = np.random.default_rng(1)
    a, n, d = guides()
    film = rng.uniform(0, 1, (W * H, 3)).astype(np.float32)
    out = O.denoise(film, a, n, d, W, H, iterations=0)
    np.testing.assert_allclose(out, film, rtol=1e-6)


def test_noise_is_reduced():
    rng = np.random.default_rng(2)
    a, n, d = guides()
    film = (0.5 + rng.normal(0, 0.2, (W * H, 3))).astype(np.float32)
    out = O.denoise(film, a, n, d, W, H)
    assert out.std() < 0.5 * film.std()
    assert abs(out.mean() - film.mean()) < 0.02


def test_normals_stop_the_filter():
    a, n, d = guides()
    n = n.reshape(H, W, 3)
    n[:, W // 2:] = (1.0, 0.0, 0.0)  # a crease: perpendicular normals
    film = np.zeros((H, W, 3), np.float32)
    film[:, W // 2:] = 1.0
    out = O.denoise(film.reshape(-1, 3), a, n.reshape(-1, 3), d, W, H).reshape(H, W, 3)
    assert out[:, W // 2 - 1].max() < 1e-3  # nothing bled across the crease
    assert out[:, W // 2].min() > 0.99


def test_depth_stops_the_filter():
    a, n, d = guides()
    d = d.reshape(H, W)
    d[:, W // 2:] = 50.0
    film = np.zeros((H, W, 3), np.float32)
    film[:, W // 2:] = 1.0
    out = O.denoise(film.reshape(-1, 3), a, n, d.reshape(-1), W, H).reshape(H, W, 3)
    assert out[:, W // 2 - 1].max() < 1e-3
