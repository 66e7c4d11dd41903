"""The instanced frame loop end to end at a small size (lucida_b200.
frame_bench: per-frame TLAS rebuild by LBVH, guided render with training,
denoiser with FP16 guides), and its error table against a converged render:
the denoised guided frame is closer to it than the undenoised plain render of
the same sample count, by the denoiser's own metric (the median per-pixel
distance, crates/core/tests/denoise_render.rs:43-88)."""
import json

import pytest

pytestmark = pytest.mark.gpu


def test_frame_loop_and_error_table(tmp_path):
    from lucida_b200 import frame_bench
    out = tmp_path / "frames.json"
    frame_bench.main(["--frames", "3", "--warmup", "1", "--width", "240", "--height", "135", "--meshes", "3",
                      "--min-tris", "2000", "--max-tris", "8000", "--instances", "96", "--reference-spp", "512",
                      "--profile-frames", "1", "--out", str(out)])
    r = json.loads(out.read_text())
    print(json.dumps(r, indent=1))
    assert r["value"] > 0 and r["guided"] and r["denoise"]
    assert r["guide"]["steps"] >= 4  # a step per loop frame, warm-up and profiled repeat
    st = r["stage_ms_profiled"]
    assert st["extend_ms"] > 0 and st["shade_ms"] > 0 and st["guide_ms"] > 0
    e = {k: v for k, v in r["error_vs_reference"].items() if k != "reference_spp"}
    assert set(e) == {"guided", "guided_denoised", "plain", "plain_denoised"}
    for k, v in e.items():
        assert v["mse"] > 0 and v["median_distance"] > 0, k
    gain = r["denoised_guided_vs_undenoised_plain"]
    assert gain["median_distance"] > 1.3, gain
    # the filter alone helps the typical pixel of the plain render too
    assert e["plain"]["median_distance"] > 1.3 * e["plain_denoised"]["median_distance"]
