"""The learned guide on the device against the numpy oracle (oracle/guide.py).

  * forward: BF16 tensor-core MLP vs the oracle's BF16-emulating forward;
    the device must sit closer to the BF16 oracle than to an FP32 one;
  * gradient: fused backward (weight gradients accumulated across tiles) vs
    the oracle's analytic gradient, per parameter block;
  * mixture: sampling and density of the vMF mixture vs the oracle, sample by
    sample, and the device sampler's chi-squared fit to its own pdf;
  * training: Adam steps on the device reduce the loss like the oracle's;
  * guided renders stay unbiased: with one-sample MIS against the guide (any
    guide, trained or not) the image converges to the plain render's.

Tolerances: BF16 rounds activations to 8 bits of mantissa; the device and
the oracle accumulate in different orders, so an activation near a rounding
boundary can land one BF16 ulp apart. The bounds below are a few such ulps
on the outputs (forward) and 3% in norm per parameter block (gradient).
"""
import numpy as np
import pytest

from oracle import guide as OG
from tests.test_samplers_chi2 import _bins, _cell_dirs, _chi2, NT, NP, SUB

LO = np.array([-4.0, -1.0, -3.0], np.float32)
HI = np.array([4.0, 3.0, 5.0], np.float32)


def _unit(a):
    a = np.asarray(a, np.float64)
    return (a / np.linalg.norm(a, axis=-1, keepdims=True)).astype(np.float32)


def _params(seed):
    p = OG.init_params(seed)
    P = OG.unpack(p)  # views into p
    rng = np.random.default_rng(seed + 100)
    for b in ("b1", "b2", "b3", "b4"):
        P[b][:] = rng.normal(0, 0.1, P[b].shape)
    return p


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(LO - 0.5, HI + 0.5, (n, 3)).astype(np.float32)  # a few outside the box (clamped)
    return x, _unit(rng.normal(size=(n, 3))), _unit(rng.normal(size=(n, 3)))


@pytest.fixture(scope="module")
def gpu():
    import lucida_b200 as lb
    g = lb.Gpu(0)
    yield g
    g.close()


@pytest.mark.gpu
def test_forward_matches_the_bf16_oracle(gpu):
    from lucida_b200 import Guide
    p = _params(1)
    guide = Guide(gpu, params=p, lo=LO, hi=HI)
    assert np.array_equal(guide.params(), p)
    x, n, wo = _inputs(5000, 2)  # not a multiple of the 64-row tile
    raw = guide.forward(x, n, wo)
    X = OG.encode(x, n, wo, LO, HI)
    ref, _ = OG.forward(p, X, emulate_bf16=True)
    ref32, _ = OG.forward(p, X, emulate_bf16=False)
    scale = np.abs(ref).max()
    err = np.abs(raw - ref)
    assert err.max() < 3e-2 * scale and err.mean() < 1e-3 * scale, (err.max() / scale, err.mean() / scale)
    assert err.mean() < 0.5 * np.abs(raw - ref32).mean()  # the device really rounds to BF16
    print("forward: max/mean err (of max |out|):", err.max() / scale, err.mean() / scale)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 127, 128, 129, 40_000])
def test_tcgen05_forward_matches_mma_sync(gpu, n):
    """The tcgen05 (TMEM) forward against the mma.sync one: the same BF16
    operands and activations, FP32 accumulation in a different order."""
    from lucida_b200 import Guide
    guide = Guide(gpu, params=_params(3), lo=LO, hi=HI)
    x, nrm, wo = _inputs(n, 5)
    a = guide.forward(x, nrm, wo, path="tcgen05")
    b = guide.forward(x, nrm, wo, path="mma.sync")
    scale = max(np.abs(b).max(), 1e-6)
    err = np.abs(a - b)
    print(n, "tcgen05 vs mma.sync max/mean err (of max |out|):", err.max() / scale, err.mean() / scale)
    assert np.all(np.isfinite(a)) and err.max() < 2e-2 * scale and err.mean() < 2e-4 * scale


def _records(n, seed):
    rng = np.random.default_rng(seed)
    x, nrm, wo = _inputs(n, seed + 1)
    wi = _unit(rng.normal(size=(n, 3)) * 0.5 + np.array([0.3, 1.0, -0.2]))
    F = rng.exponential(1.0, n).astype(np.float32)
    F[rng.random(n) < 0.1] = 0.0  # records whose path gathered nothing
    return x, nrm, wo, wi, F


@pytest.mark.gpu
def test_gradient_matches_the_oracle(gpu):
    from lucida_b200 import Guide, records_array
    p = _params(3)
    guide = Guide(gpu, params=p, lo=LO, hi=HI)
    x, nrm, wo, wi, F = _records(3000, 4)
    g_dev, loss_dev = guide.gradient(records_array(x, nrm, wo, wi, F))
    assert np.array_equal(guide.params(), p)  # a gradient evaluation does not step
    X = OG.encode(x, nrm, wo, LO, HI)
    o, acts = OG.forward(p, X)
    loss, go = OG.loss_and_grad_outputs(o, wi, F)
    g_ref = OG.backward(p, acts, go)
    assert abs(loss_dev - loss) < 1e-3 * abs(loss) + 1e-4, (loss_dev, loss)
    off = 0
    for name, shape in OG.SHAPES:
        k = int(np.prod(shape))
        a, b = g_dev[off:off + k].astype(np.float64), g_ref[off:off + k].astype(np.float64)
        off += k
        if name == "W1":  # the zero padding columns get a zero gradient
            b = b.reshape(shape)[:, :120].ravel()
            assert np.all(g_dev[:k].reshape(shape)[:, 120:] == 0)
            a = a.reshape(shape)[:, :120].ravel()
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        cos = a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-30)
        print(f"grad {name}: rel {rel:.2e} cos {cos:.6f}")
        assert rel < 3e-2 and cos > 0.999, (name, rel, cos)


def _mixture_raw(n, seed):
    rng = np.random.default_rng(seed)
    raw = rng.normal(0, 1.0, (n, 40)).astype(np.float32)
    raw[:, 3::5] = rng.uniform(-3, 7, (n, 8))  # kappa from ~1 to ~1100
    raw[:, 4::5] *= 2.0
    return raw


@pytest.mark.gpu
def test_mixture_sampling_and_density_match_the_oracle(gpu):
    from lucida_b200 import Guide
    guide = Guide(gpu, seed=0, lo=LO, hi=HI)
    n = 100_000
    raw = _mixture_raw(n, 5)
    u = np.random.default_rng(6).random((n, 3), dtype=np.float32).clip(0, np.float32(1 - 2 ** -24))
    d_dev, pdf_dev = guide.mixture_sample(raw, u)
    d_ref = OG.sample(raw, u.astype(np.float64))
    # Lobe choice can flip where u0 sits on a cumulative-weight boundary.
    err = np.abs(d_dev - d_ref).max(1)
    assert np.mean(err > 1e-4) < 1e-3, np.mean(err > 1e-4)
    assert np.allclose(np.linalg.norm(d_dev, axis=1), 1, atol=1e-5)
    pdf_at_dev = OG.mixture_pdf(raw, d_dev.astype(np.float64))
    rel = np.abs(pdf_dev - pdf_at_dev) / pdf_at_dev
    assert np.quantile(rel, 0.999) < 1e-3 and np.median(rel) < 1e-5, (np.quantile(rel, 0.999), np.median(rel))
    pdf1 = guide.mixture_pdf(raw, d_ref.astype(np.float32))
    rel1 = np.abs(pdf1 - OG.mixture_pdf(raw, d_ref)) / OG.mixture_pdf(raw, d_ref)
    assert np.quantile(rel1, 0.999) < 1e-3, np.quantile(rel1, 0.999)


@pytest.mark.gpu
def test_device_mixture_sampler_matches_its_pdf(gpu):
    from lucida_b200 import Guide
    guide = Guide(gpu, seed=0, lo=LO, hi=HI)
    raw = _mixture_raw(1, 7)
    raw[0, 3::5] = np.random.default_rng(8).uniform(-1, 3, 8)  # kappa <= ~20: cells resolve the lobes
    N = 400_000
    u = np.random.default_rng(9).random((N, 3), dtype=np.float32).clip(0, np.float32(1 - 2 ** -24))
    d, _ = guide.mixture_sample(np.repeat(raw, N, 0), u)
    obs = np.bincount(_bins(d), minlength=NT * NP)
    dirs = _cell_dirs()
    pdf = guide.mixture_pdf(np.repeat(raw, len(dirs), 0), dirs)
    dw = (2.0 / (NT * SUB)) * (2 * np.pi / (NP * SUB))
    exp = pdf.reshape(NT, SUB, NP, SUB).astype(np.float64).sum(axis=(1, 3)).reshape(-1) * dw * N
    p, chi = _chi2(obs, exp)
    assert p > 1e-3, (p, chi)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [3000, 100_000])
def test_tensor_core_gradient_matches_mma_sync(gpu, gpu_mma, n):
    """The tcgen05 training kernel (the default) and the mma.sync one give
    the same gradient and loss up to summation order and the bias gradients'
    BF16 operands (3000 records: 24 tiles, one per CTA; 100,000: several
    tiles accumulated per CTA in tensor memory), and both match the oracle."""
    from lucida_b200 import Guide, records_array
    p = _params(5)
    x, nrm, wo, wi, F = _records(n, 6)
    rec = records_array(x, nrm, wo, wi, F)
    g_tc, l_tc = Guide(gpu, params=p, lo=LO, hi=HI).gradient(rec)
    g_mm, l_mm = Guide(gpu_mma, params=p, lo=LO, hi=HI).gradient(rec)
    X = OG.encode(x, nrm, wo, LO, HI)
    o, acts = OG.forward(p, X)
    loss, go = OG.loss_and_grad_outputs(o, wi, F)
    g_ref = OG.backward(p, acts, go)
    assert abs(l_tc - l_mm) < 1e-4 * abs(l_mm) + 1e-6, (l_tc, l_mm)
    assert abs(l_tc - loss) < 1e-3 * abs(loss) + 1e-4, (l_tc, loss)
    off = 0
    for name, shape in OG.SHAPES:
        k = int(np.prod(shape))
        a, b, c = (v[off:off + k].astype(np.float64) for v in (g_tc, g_mm, g_ref))
        off += k
        if name == "W1":
            assert np.all(a.reshape(shape)[:, 120:] == 0)
            a, b, c = (v.reshape(shape)[:, :120].ravel() for v in (a, b, c))
        rel_mm = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        rel_ref = np.linalg.norm(a - c) / max(np.linalg.norm(c), 1e-12)
        print(f"grad {name}: tcgen05 vs mma.sync {rel_mm:.2e}, vs oracle {rel_ref:.2e}")
        assert rel_mm < 1e-2, (name, rel_mm)
        assert rel_ref < 3e-2, (name, rel_ref)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["tcgen05", "mma.sync"])
def test_device_training_tracks_the_oracle(request, kernel):
    from lucida_b200 import Guide, records_array
    gpu = request.getfixturevalue("gpu" if kernel == "tcgen05" else "gpu_mma")
    p0 = OG.init_params(11)
    guide = Guide(gpu, params=p0, lo=LO, hi=HI)
    n = 2048
    x, nrm, wo = _inputs(n, 12)
    rng = np.random.default_rng(13)
    # Radiance from a cone around a direction that depends on the position.
    axis = _unit(np.stack([np.sign(x[:, 0]) * 0.8, np.ones(n), 0.3 * np.ones(n)], 1))
    wi = _unit(axis + rng.normal(size=(n, 3)) * 0.15)
    F = np.ones(n, np.float32)
    rec = records_array(x, nrm, wo, wi, F)
    X = OG.encode(x, nrm, wo, LO, HI)
    p, m, v = p0.copy(), np.zeros(p0.size), np.zeros(p0.size)
    ref = []
    for t in range(1, 41):
        o, acts = OG.forward(p, X)
        loss, go = OG.loss_and_grad_outputs(o, wi, F)
        ref.append(loss)
        p, m, v = OG.adam(p, OG.backward(p, acts, go), m, v, t)
    dev = [guide.train(rec, steps=1) for _ in range(40)]
    st = guide.stats()
    assert st.steps == 40 and st.last_records == n
    print("loss oracle", ref[0], ref[-1], "device", dev[0], dev[-1])
    assert abs(dev[0] - ref[0]) < 1e-3 * abs(ref[0])
    assert dev[-1] < dev[0] - 1.0  # it learns the cone
    assert abs(dev[-1] - ref[-1]) < 0.1 * abs(ref[0] - ref[-1])


# ---------------------------------------------------------------- guided renders
def _block_means(gpu, scene, spp, depth, guided, sampling, calls, seed):
    """Per-call 8 x 8-pixel block means of the luminance, (calls, 64)."""
    import lucida_b200 as lb
    params = lb.RenderParams(width=64, height=64, samples=spp, max_depth=depth, sampling=sampling,
                             sampler="independent", frame_seed=seed)
    out = []
    for k in range(calls):
        params.sample_offset = k * spp
        acc = lb.render_accum(gpu, scene, params, guided=guided)
        lum = (acc["radiance"] / spp) @ np.array([0.2126, 0.7152, 0.0722])
        out.append(lum.reshape(8, 8, 8, 8).mean((1, 3)).ravel())
    return np.array(out)


@pytest.fixture(scope="module")
def gpu_mma():
    """A context whose renders run the guide inference on the mma.sync
    kernel (the default is tcgen05)."""
    import os
    import lucida_b200 as lb
    os.environ["LUC_GUIDE_TC"] = "0"
    try:
        g = lb.Gpu(0)
    finally:
        del os.environ["LUC_GUIDE_TC"]
    yield g
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("sampling", ["mis", "nee", "bsdf"])
@pytest.mark.parametrize("inference", ["mma.sync", "tcgen05"])
def test_guided_render_is_unbiased(gpu, gpu_mma, sampling, inference):
    """Cornell box, 64 x 64: 64 guided batches of 8 spp (an untrained guide
    that takes one Adam step per batch) against 16 plain batches of 64 spp.
    Block means must agree within their standard errors (estimated from the
    spread across batches): |z| < 5 for each of the 64 blocks, mean |z| < 1.5,
    and the image means within 1%."""
    from lucida_b200 import Guide, scenes
    gpu = gpu_mma if inference == "mma.sync" else gpu
    scene = scenes.cornell_analytic()
    gpu.upload(scene, force=True)
    guide = Guide(gpu, seed=3)
    guide.configure(train=True, records_per_step=1 << 14, lr=1e-2)
    g = _block_means(gpu, scene, 8, 6, True, sampling, 64, 0x5EED1234)
    st = guide.stats()
    assert st.steps == 64 and st.last_records > 0
    assert st.tc_error == 0  # every tensor-core inference tile completed
    r = _block_means(gpu, scene, 64, 6, False, sampling, 16, 0xC0FFEE)
    mg, mr = g.mean(0), r.mean(0)
    se = np.sqrt(g.var(0, ddof=1) / len(g) + r.var(0, ddof=1) / len(r))
    z = (mg - mr) / np.maximum(se, 1e-12)
    print(sampling, "image mean guided/plain", mg.mean() / mr.mean(), "max |z|", np.abs(z).max(),
          "mean |z|", np.abs(z).mean(), "guide loss", st.last_loss)
    assert abs(mg.mean() / mr.mean() - 1) < 0.01
    assert np.abs(z).max() < 5.0 and np.abs(z).mean() < 1.5
