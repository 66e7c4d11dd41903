"""The device denoiser against the oracle on a real accumulator
(crates/gpu/tests/denoise_agreement.rs asks mean relative error < 4e-3).

The device follows the reference's GPU semantics (atrous.wgsl): guides are
accumulator sums divided by max(samples, 1), the albedo floored at 1e-3
before use. The oracle's CPU filter (denoise.rs:134-228) is fed the same
per-pixel averages, so both filter identical inputs; pow/exp are rounded
from a double evaluation on the device, so agreement is to a few ULPs."""
import numpy as np
import pytest

import oracle as O
import lucida_b200 as lb
from lucida_b200 import layout as L, scenes
from tests.bridge import compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = lb.Gpu(0)
    yield g
    g.close()


def _oracle_inputs(acc):
    a = acc.reshape(-1)
    inv = (np.float32(1) / np.maximum(a["samples"], np.float32(1))).astype(np.float32)[:, None]
    film = (a["radiance"] * inv).astype(np.float32)
    alb = np.maximum((a["albedo"] * inv).astype(np.float32), np.float32(1e-3))
    nrm = (a["normal"] * inv).astype(np.float32)
    dep = (a["depth"] * inv[:, 0]).astype(np.float32)
    return film, alb, nrm, dep


@pytest.mark.parametrize("iterations,sn,sd,sl,sa", [(4, 64.0, 0.08, 4.0, 0.1), (5, 128.0, 1.0, 4.0, 0.1),
                                                     (0, 64.0, 0.08, 4.0, 0.1)])
def test_denoise_matches_oracle(gpu, iterations, sn, sd, sl, sa):
    s = scenes.cornell_analytic()
    acc = lb.render_accum(gpu, s, lb.RenderParams(width=96, height=80, samples=4, max_depth=6))
    dp = lb.DenoiseParams(iterations, sn, sd, sl, sa)
    out = lb.Denoiser(gpu).run(acc, dp).reshape(-1)
    film, alb, nrm, dep = _oracle_inputs(acc)
    ref = O.denoise(film, alb, nrm, dep, 96, 80, iterations, sn, sd, sl, sa)
    st = compare(out["radiance"], ref)
    print(st)
    assert st["mean_rel"] < 1e-5 and st["max_rel"] < 1e-3, st
    assert np.all(out["samples"] == 1.0)
    np.testing.assert_array_equal(out["albedo"].reshape(-1, 3), alb)


def test_accumulator_untouched_and_noise_reduced(gpu):
    """denoise_agreement.rs:69-92: the accumulator is a separate product."""
    s = scenes.cornell_analytic()
    p = lb.RenderParams(width=64, height=64, samples=2, max_depth=6)
    acc = lb.render_accum(gpu, s, p)
    before = acc.copy()
    out = lb.Denoiser(gpu).run(acc)
    assert acc.tobytes() == before.tobytes()
    ref = lb.render_accum(gpu, s, lb.RenderParams(width=64, height=64, samples=256, max_depth=6))
    truth = ref["radiance"] / ref["samples"][..., None]
    noisy = acc["radiance"] / acc["samples"][..., None]
    err_noisy = np.median(np.abs(noisy - truth))
    err_dn = np.median(np.abs(out["radiance"] - truth))
    assert err_dn < err_noisy, (err_dn, err_noisy)


@pytest.mark.parametrize("iterations,sn,sd,sl", [(5, 128.0, 1.0, 4.0), (4, 64.0, 0.08, 4.0)])
def test_half_precision_guides(gpu, iterations, sn, sd, sl):
    """luc_denoise_dev on device buffers: FP32 guides give exactly the host
    entry point's image; FP16 guides stay within the reference's own
    GPU-vs-CPU agreement bound (mean relative error < 4e-3) of the oracle."""
    import ctypes as C
    import torch
    from lucida_b200.native import DenoiseParams as DP, LUC_DENOISE_HALF_GUIDES, check, lib
    s = scenes.cornell_analytic()
    w, h = 96, 80
    acc = lb.render_accum(gpu, s, lb.RenderParams(width=w, height=h, samples=4, max_depth=6))
    dp = lb.DenoiseParams(iterations, sn, sd, sl, 0.1)
    host = lb.Denoiser(gpu).run(acc, dp).reshape(-1)
    d_in = torch.from_numpy(np.ascontiguousarray(acc).view(np.uint8).reshape(-1).copy()).cuda()
    d_out = torch.zeros_like(d_in)
    p = DP(iterations, sn, sd, sl, 0.1)
    outs = {}
    for flags in (0, LUC_DENOISE_HALF_GUIDES):
        torch.cuda.synchronize()
        check(gpu.handle, lib().luc_denoise_dev(gpu.handle, C.c_void_p(d_in.data_ptr()), w, h, C.byref(p), flags,
                                                C.c_void_p(d_out.data_ptr())))
        torch.cuda.synchronize()
        outs[flags] = d_out.cpu().numpy().view(L.ACCUM)
    assert outs[0].tobytes() == host.tobytes()
    film, alb, nrm, dep = _oracle_inputs(acc)
    ref = O.denoise(film, alb, nrm, dep, w, h, iterations, sn, sd, sl, 0.1)
    st = compare(outs[LUC_DENOISE_HALF_GUIDES]["radiance"], ref)
    print("fp16 guides vs oracle", st)
    assert st["mean_rel"] < 4e-3, st
    assert d_in.cpu().numpy().tobytes() == np.ascontiguousarray(acc).view(np.uint8).reshape(-1).tobytes()
