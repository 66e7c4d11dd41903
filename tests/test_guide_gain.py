"""What the trained guide gains over rendering without it.

On a small guided room (24 displaced spheres in the half-closed room lit by
two small emitters facing the ceiling; 128 x 128, 8 bounces) the guide is
trained online on the tracer's own records (guided 1-spp frames, one Adam
step each), then frozen; guided and plain renders of the same sample count
(their own seeds) are compared with a 4096-spp plain reference by mean
squared error per pixel. The trained guide must lower the error at equal
sample count by the stated margin, and a freshly initialised guide must not
(the gain comes from training, not from the one-sample MIS alone).
"""
import numpy as np
import pytest

import lucida_b200 as lb
from lucida_b200 import Guide, scenes

pytestmark = pytest.mark.gpu

W = H = 128
DEPTH = 8
TRAIN_FRAMES = 1500
SPP = 128
MARGIN = 3.0


def _image(acc):
    a = acc.reshape(-1)
    return a["radiance"].astype(np.float64) / np.maximum(a["samples"], 1.0)[:, None]


def _mse(img, ref):
    return float(((img - ref) ** 2).mean())


def test_trained_guide_lowers_error_at_equal_samples():
    g = lb.Gpu(0)
    s = scenes.guided_room(count=24, level=3)
    ref = _image(lb.render_accum(g, s, lb.RenderParams(width=W, height=H, samples=4096, max_depth=DEPTH,
                                                         frame_seed=0xA5A5F00D)))
    test = lb.RenderParams(width=W, height=H, samples=SPP, max_depth=DEPTH, frame_seed=0x5EED1234,
                           sample_offset=1 << 20)
    plain = _mse(_image(lb.render_accum(g, s, test)), ref)

    guide = Guide(g, seed=7)
    guide.configure(train=False)
    untrained = _mse(_image(lb.render_accum(g, s, test, guided=True)), ref)

    guide.configure(train=True, records_per_step=1 << 16, lr=1e-2)
    train = lb.RenderParams(width=W, height=H, samples=1, max_depth=DEPTH, frame_seed=0x0BADCAFE)
    for k in range(TRAIN_FRAMES):
        train.sample_offset = k
        lb.render_accum(g, s, train, guided=True)
    guide.configure(train=False)
    trained = _mse(_image(lb.render_accum(g, s, test, guided=True)), ref)
    st = guide.stats()
    g.close()
    print(f"MSE at {SPP} spp: plain {plain:.4g}, untrained guide {untrained:.4g}, "
          f"trained guide ({st.steps} steps) {trained:.4g}: gain {plain / trained:.2f}x, untrained "
          f"{plain / untrained:.2f}x")
    assert st.steps >= TRAIN_FRAMES - 1 and st.tc_error == 0
    assert plain / trained > MARGIN, (plain, trained)
    assert plain / untrained < plain / trained
