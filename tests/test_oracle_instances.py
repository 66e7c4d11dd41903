"""The oracle's instancing (instance.rs, scene.rs:252-345) against the
reference's packed `instance-forest` scene and its own unit tests.

Pinned bit for bit: materials, positions, vertex normals, the BLAS (binned
SAH over the shared icosphere, compacted triangle order, rebased nodes), the
TLAS topology (child and leaf indices, counts) and every instance row's
metadata (BLAS root, kind tag, material override). Two things are pinned to
rounding instead: the world-to-object matrices and the TLAS boxes. The
reference inverts with glam's 4x4 inverse and recovers the forward matrix for
the world bounds by inverting again; the oracle (and the device) use the
adjugate of the 3x3 part, which agrees to an ulp or two.

The properties restated from instance.rs:144-311 (t preserved by the ray
transform, normals perpendicular to transformed tangents, world bounds that
contain the rotated box and grow under rotation, the inverse round trip) run
on the oracle's transforms with the reference's probe matrices.
"""
import base64
import hashlib
import json
import math
import os

import numpy as np
import pytest

import oracle as O

FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "scene_fixtures.json")))["instance-forest"]
SEC = FIX["sections"]


@pytest.fixture(scope="module")
def forest():
    return O.Scene.builtin("instance-forest")


def test_instancing_counts(forest):
    assert list(forest.instancing()) == FIX["instancing"]
    assert len(forest.array(O.W_PRIMITIVES)) == SEC["primitives"]["count"]
    assert len(forest.array(O.W_BVH_NODES)) == SEC["bvhNodes"]["count"]


@pytest.mark.parametrize("sec,which", [("materials", O.W_MATERIALS), ("positions", O.W_POSITIONS),
                                       ("triangles", O.W_TRIANGLES), ("lights", O.W_LIGHTS),
                                       ("envRadiance", O.W_ENV_PIXELS)])
def test_sections_bit_exact(forest, sec, which):
    assert hashlib.sha256(forest.array(which).tobytes()).hexdigest() == SEC[sec]["sha256"], sec


def test_normals_and_blas_bit_exact(forest):
    lanes = forest.array(O.W_ATTRS).view(np.uint8).reshape(-1, 32)[:, :16].tobytes()
    assert hashlib.sha256(lanes).hexdigest() == SEC["vertexAttrs"]["normal_lanes_sha256"]
    root = forest.instancing()[2]
    nodes = forest.array(O.W_BVH_NODES)
    assert hashlib.sha256(nodes[:root].tobytes()).hexdigest() == SEC["bvhNodes"]["blas_sha256"]


def test_tlas_topology_exact_bounds_to_rounding(forest):
    root = forest.instancing()[2]
    mine = forest.array(O.W_BVH_NODES)[root:]
    ref = np.frombuffer(base64.b64decode(SEC["bvhNodes"]["tlas_raw"]), O.BVH_NODE)
    np.testing.assert_array_equal(mine["left_first"], ref["left_first"])
    np.testing.assert_array_equal(mine["count"], ref["count"])
    for f in ("bounds_min", "bounds_max"):
        np.testing.assert_allclose(mine[f], ref[f], rtol=0, atol=4e-6)


def test_instance_rows(forest):
    ref = np.frombuffer(base64.b64decode(SEC["primitives"]["raw"]), np.uint32).reshape(-1, 16)
    mine = forest.array(O.W_PRIMITIVES).view(np.uint32).reshape(-1, 16)
    np.testing.assert_array_equal(mine[0], ref[0])  # the ground quad
    meta = [3, 7, 11, 15]  # blas_root, kind, material, pad
    np.testing.assert_array_equal(mine[1:, meta], ref[1:, meta])
    mat = [0, 1, 2, 4, 5, 6, 8, 9, 10, 12, 13, 14]
    np.testing.assert_allclose(mine[1:, mat].view(np.float32), ref[1:, mat].view(np.float32), rtol=0, atol=2e-6)


# ---------------------------------------------------------------- instance.rs:144-311
def _rot_y(a):
    c, s = math.cos(a), math.sin(a)
    return np.array([[c, 0, s, 0], [0, 1, 0, 0], [-s, 0, c, 0]], np.float64)


def _rot_z(a):
    c, s = math.cos(a), math.sin(a)
    return np.array([[c, -s, 0, 0], [s, c, 0, 0], [0, 0, 1, 0]], np.float64)


def _compose(*ms):
    out = np.eye(4)
    for m in ms:
        m4 = np.eye(4)
        m4[:3] = m
        out = out @ m4
    return out[:3]


def _probes():
    t = np.eye(3, 4)
    t[:, 3] = (3, -2, 5)
    return {"identity": np.eye(3, 4), "translate": t,
            "uniform scale": np.diag([2.5, 2.5, 2.5, 1.0])[:3], "non-uniform scale": np.diag([2.0, 0.5, 3.0, 1.0])[:3],
            "rotate": _rot_y(math.pi / 4),
            "compound": _compose(np.hstack([np.eye(3), [[1], [2], [3]]]), _rot_z(0.7),
                                 np.diag([1.5, 0.4, 2.0, 1.0])[:3])}


def _instance(m):
    return O.pack_instance(O.affine_inverse(m.astype(np.float32)))


@pytest.mark.parametrize("name", list(_probes()))
def test_t_is_preserved_by_the_ray_transform(name):
    m = _probes()[name]
    inst = _instance(m)
    origin = np.array([-1.0, 0.5, -4.0])
    d = np.array([0.2, 0.1, 1.0])
    d /= np.linalg.norm(d)
    o_obj = O.instance_transform(inst, origin, 0)[0].astype(np.float64)
    d_obj = O.instance_transform(inst, d, 1)[0].astype(np.float64)
    m4 = np.vstack([m, [0, 0, 0, 1]])
    for t in (0.5, 1.0, 7.25):
        expected = (np.linalg.inv(m4) @ np.append(origin + t * d, 1.0))[:3]
        assert np.linalg.norm(o_obj + t * d_obj - expected) < 1e-3, (name, t)


@pytest.mark.parametrize("name", list(_probes()))
def test_normals_stay_perpendicular(name):
    m = _probes()[name]
    inst = _instance(m)
    n = np.array([0.3, 0.8, -0.5])
    n /= np.linalg.norm(n)
    t1 = np.cross(n, [1, 0, 0])
    t1 /= np.linalg.norm(t1)
    t2 = np.cross(n, t1)
    t2 /= np.linalg.norm(t2)
    nw = O.instance_transform(inst, n, 2)[0].astype(np.float64)
    for t in (t1, t2):
        tw = m[:, :3] @ t
        assert abs(nw @ (tw / np.linalg.norm(tw))) < 1e-3, name
    assert abs(np.linalg.norm(nw) - 1) < 1e-4


@pytest.mark.parametrize("name", list(_probes()))
def test_world_bounds_contain_the_transformed_box(name):
    m = _probes()[name]
    inst = _instance(m)
    lo, hi = np.array([-1.0, -2.0, -0.5]), np.array([1.0, 2.0, 0.5])
    w = O.instance_world_bounds(inst, np.concatenate([lo, hi]))
    for i in range(8):
        c = np.array([hi[0] if i & 1 else lo[0], hi[1] if i & 2 else lo[1], hi[2] if i & 4 else lo[2]])
        p = m[:, :3] @ c + m[:, 3]
        assert np.all(p >= w[:3]) and np.all(p <= w[3:]), (name, i)


def test_rotation_grows_the_bounds():
    inst = _instance(_rot_y(math.pi / 4))
    w = O.instance_world_bounds(inst, np.array([-1, -1, -1, 1, 1, 1.0]))
    ext = w[3:] - w[:3]
    assert ext[0] > 2.7 and ext[2] > 2.7 and abs(ext[1] - 2.0) < 0.01


@pytest.mark.parametrize("name", list(_probes()))
def test_inverse_round_trips(name):
    m = _probes()[name].astype(np.float32)
    back = O.affine_inverse(O.affine_inverse(m))
    np.testing.assert_allclose(back, m, rtol=0, atol=1e-4)
