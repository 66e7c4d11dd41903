"""Chi-squared goodness of fit: every sampler against its own pdf.

Restates crates/core/src/chi2.rs:104-420 and crates/core/tests/bsdf_chi2.rs:
draw N directions from a sampler, histogram them on a (cos theta, phi) grid
over the whole sphere, integrate the sampler's pdf over each cell (midpoint
sub-grid in (cos theta, phi), where the solid-angle measure is flat), pool
cells expecting fewer than 5 samples, and require Pearson's statistic to pass
at alpha = 0.01 with a Sidak correction over the family of tests. Invalid
samples (pdf = 0) are dropped and the pdf is *not* renormalised, so a sampler
whose acceptance rate disagrees with its pdf's total mass fails.

Roughnesses stay at or above 0.3 (the reference's own sweep starts at 0.1
with adaptive Simpson quadrature): the midpoint sub-grid cannot resolve a
lobe narrower than a cell. Sharp lobes are covered by the sample-by-sample
device-vs-oracle comparison below instead.

CPU tests run the oracle's samplers; `gpu` tests run the device's, through
the per-function eval entry points, and also diff device against oracle
sample by sample.
"""
import math

import numpy as np
import pytest
from scipy import stats

import oracle as O
from lucida_b200 import layout as L

NT, NP, SUB = 32, 64, 6
N = 400_000
MATERIALS = {
    "diffuse": L.diffuse((0.8, 0.8, 0.8)),
    "glossy-0.3": L.glossy((0.2, 0.4, 0.8), 0.3),
    "metal-0.3": L.metal((0.95, 0.8, 0.4), 0.3),
    "metal-0.7": L.metal((0.95, 0.8, 0.4), 0.7),
    "glass-0.35": L.glass((1.0, 1.0, 1.0), 0.35, 1.5),
    "glass-0.6": L.glass((1.0, 1.0, 1.0), 0.6, 1.5),
    "conductor": L.material(base_color=(0.9, 0.6, 0.5), metallic=1.0, roughness=0.35, ior=1.5,
                            eta=(0.200438, 0.924033, 1.102212), k=(3.9124, 2.44753, 2.13764)),
}
CASES = [(m, front, c) for m in MATERIALS for front in (1, 0) for c in (0.85, 0.35)
         if front == 1 or m.startswith("glass")]
ALPHA = 1.0 - (1.0 - 0.01) ** (1.0 / (2 * len(CASES) + 2))  # Sidak over CPU + GPU families


def _wo(cos_t):
    return np.array([math.sqrt(1 - cos_t * cos_t), 0.0, cos_t], np.float32)


def _bins(w):
    ct = np.clip(w[:, 2], -1, 1)
    i = np.minimum(((ct + 1) * 0.5 * NT).astype(np.int64), NT - 1)
    ph = np.mod(np.arctan2(w[:, 1], w[:, 0]), 2 * np.pi)
    j = np.minimum((ph / (2 * np.pi) * NP).astype(np.int64), NP - 1)
    return i * NP + j


def _cell_dirs(sub=SUB):
    """Midpoint sub-grid of every (cos theta, phi) cell: (NT*NP*sub*sub, 3)."""
    ct = -1 + (np.arange(NT * sub) + 0.5) * (2.0 / (NT * sub))
    ph = (np.arange(NP * sub) + 0.5) * (2 * np.pi / (NP * sub))
    C, P = np.meshgrid(ct, ph, indexing="ij")
    s = np.sqrt(np.maximum(1 - C * C, 0))
    return np.stack([s * np.cos(P), s * np.sin(P), C], -1).reshape(-1, 3).astype(np.float32)


def _expected(pdf_values, sub=SUB):
    """Integrate pdf over each cell: sum of midpoint values x sub-cell solid angle."""
    dw = (2.0 / (NT * sub)) * (2 * np.pi / (NP * sub))
    p = pdf_values.reshape(NT, sub, NP, sub).astype(np.float64)
    return p.sum(axis=(1, 3)).reshape(-1) * dw * N


def _chi2(observed, expected):
    order = np.argsort(expected)
    obs, exp = observed[order].astype(np.float64), expected[order]
    small = exp < 5
    o = np.concatenate([[obs[small].sum()], obs[~small]]) if small.any() else obs
    e = np.concatenate([[exp[small].sum()], exp[~small]]) if small.any() else exp
    keep = e > 0
    if (o[~keep] > 0).any():
        return 0.0, np.inf  # samples where the pdf says there can be none
    o, e = o[keep], e[keep]
    chi = float(((o - e) ** 2 / e).sum())
    return float(stats.chi2.sf(chi, len(o) - 1)), chi


def _uniforms(seed):
    rng = np.random.default_rng(seed)
    return rng.random((N, 3), dtype=np.float32).clip(0, np.float32(1 - 2 ** -24))


def _pdf_grid(mat, front, wo):
    dirs = _cell_dirs()
    _, pdf = O.bsdf_eval(mat, front, np.tile(wo, (len(dirs), 1)), dirs)
    return pdf


@pytest.mark.parametrize("name,front,cos_t", CASES)
def test_oracle_bsdf_sampler_matches_its_pdf(name, front, cos_t):
    mat = MATERIALS[name]
    wo = _wo(cos_t)
    wi, w, pdf = O.bsdf_sample(mat, front, np.tile(wo, (N, 1)), _uniforms(1))
    valid = pdf > 0
    obs = np.bincount(_bins(wi[valid]), minlength=NT * NP)
    p, chi = _chi2(obs, _expected(_pdf_grid(mat, front, wo)))
    assert p > ALPHA, (name, front, cos_t, p, chi)


def test_oracle_env_sampler_matches_its_pdf():
    sc = O.Scene.builtin("sunset")
    rng = np.random.default_rng(3)
    d, r, pdf = sc.env_sample(rng.random((N, 2), dtype=np.float32))
    valid = pdf > 0
    # The pdf is constant per texel (256 x 128, 1.4 degrees) and the sun spans
    # about two texels: integrate on a 24 x 24 sub-grid per cell (~0.23 deg).
    sub = 24
    dirs = _cell_dirs(sub)
    epdf = np.zeros(len(dirs), np.float32)
    rad = np.zeros((len(dirs), 3), np.float32)
    # The env sampler works in the world frame (y up): rotate y -> z for the grid.
    obs = np.bincount(_bins(d[valid][:, [2, 0, 1]]), minlength=NT * NP)
    dirs_w = np.ascontiguousarray(dirs[:, [1, 2, 0]])
    O.lib().orc_env_pdf_batch(sc._h, O._p(dirs_w), len(dirs), O._p(epdf), O._p(rad))
    p, chi = _chi2(obs, _expected(epdf, sub))
    assert p > ALPHA, (p, chi)


# ---------------------------------------------------------------- device samplers
@pytest.fixture(scope="module")
def gpu():
    import lucida_b200 as lb
    g = lb.Gpu(0)
    yield g
    g.close()


def _device_sample(gpu, mat, front, wo, u):
    import ctypes as C
    from lucida_b200.native import check, lib, ptr
    n = len(u)
    m = np.ascontiguousarray(np.asarray(mat, L.MATERIAL).reshape(1))
    wo_a = np.ascontiguousarray(np.tile(wo, (n, 1)), np.float32)
    wi = np.zeros((n, 3), np.float32)
    f = np.zeros((n, 3), np.float32)
    pdf = np.zeros(n, np.float32)
    check(gpu.handle, lib().luc_eval_bsdf(gpu.handle, ptr(m), front, ptr(wo_a), ptr(np.ascontiguousarray(u)), n, 0,
                                          ptr(wi), ptr(f), ptr(pdf)))
    return wi, f, pdf


@pytest.mark.gpu
@pytest.mark.parametrize("name,front,cos_t", CASES)
def test_device_bsdf_sampler_matches_its_pdf_and_the_oracle(gpu, name, front, cos_t):
    mat = MATERIALS[name]
    wo = _wo(cos_t)
    u = _uniforms(2)
    wi, w, pdf = _device_sample(gpu, mat, front, wo, u)
    valid = pdf > 0
    obs = np.bincount(_bins(wi[valid]), minlength=NT * NP)
    p, chi = _chi2(obs, _expected(_pdf_grid(mat, front, wo)))
    assert p > ALPHA, (name, front, cos_t, p, chi)
    # Sample by sample against the oracle on the same uniforms.
    owi, ow, opdf = O.bsdf_sample(mat, front, np.tile(wo, (N, 1)), u)
    assert np.array_equal(opdf > 0, valid) or np.mean((opdf > 0) != valid) < 1e-4
    both = valid & (opdf > 0)
    # Directions agree to rounding; near the horizon z = sqrt(1 - x^2 - y^2)
    # amplifies a one-ulp difference of the trigonometry, hence the max bound.
    err = np.max(np.abs(wi[both] - owi[both]), axis=1)
    assert np.quantile(err, 0.9999) < 1e-5 and err.max() < 1e-3, (np.quantile(err, 0.9999), err.max())
    rel = np.abs(w[both] - ow[both]) / np.maximum(np.abs(ow[both]), 1e-6)
    assert np.quantile(rel, 0.9999) < 1e-4, np.max(rel)
    print(name, front, cos_t, "bit-identical samples:", float(np.mean(np.all(wi[both] == owi[both], axis=1))))
