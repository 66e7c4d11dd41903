"""Scene upload validation (luc_upload_scene): triangle indices are checked on
the device before any kernel reads through them, and a failed upload leaves
the context usable."""
import dataclasses

import numpy as np
import pytest

import lucida_b200 as lb
from lucida_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    g = lb.Gpu(0)
    yield g
    g.close()


@pytest.mark.parametrize("field,value", [("i0", 10**8), ("i2", 2**32 - 1), ("material", 999)])
@pytest.mark.parametrize("with_tree", [False, True])
def test_bad_triangle_is_rejected(gpu, field, value, with_tree):
    s = scenes.displaced_spheres(count=4, level=2, env_size=(64, 32))
    tris = s.triangles.copy()
    tris[field][777] = value
    bad = dataclasses.replace(s, triangles=tris)
    if with_tree:  # a caller-supplied tree: the same check on the caller's triangles
        import oracle as O
        nodes, prims, _, _ = O.sah_build(s.triangles.view(O.TRIANGLE), s.positions)
        tris = s.triangles[prims].copy()
        tris[field][777] = value
        bad = dataclasses.replace(s, triangles=tris, bvh_nodes=nodes.view(lb.layout.BVH_NODE))
    with pytest.raises(lb.GpuError, match="triangle 777 indexes out of range"):
        gpu.upload(bad, force=True)
    # The context still renders a valid scene afterwards.
    f = lb.render_with(gpu, s, lb.RenderParams(width=32, height=24, samples=2, max_depth=3))
    assert np.all(np.isfinite(f.data)) and f.data.mean() > 0
