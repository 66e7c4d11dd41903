"""Test helpers: move scenes between the oracle and the product, and compare
accumulators with the reference's image metrics (crates/core/src/image.rs:
158-216)."""
import numpy as np

import oracle as O
from lucida_b200 import SceneDef, layout as L
from lucida_b200.gpu import Camera


def scene_from_oracle(osc: "O.Scene", with_bvh=True) -> SceneDef:
    """Hand the oracle's finalized scene (SAH tree, compacted triangles,
    lights, env map + packed CDF) to the product unchanged."""
    bg, total, w, h = osc.misc()
    cam = osc.camera()
    env_px = env_cdf = None
    if w:
        env_px = osc.array(O.W_ENV_PIXELS).reshape(h, w, 4)
        cw = max(w, h) + 1
        env_cdf = np.zeros((h + 1, cw), np.float32)
        env_cdf[:h, :w + 1] = osc.array(O.W_ENV_COND).reshape(h, w + 1)
        env_cdf[h, :h + 1] = osc.array(O.W_ENV_MARG)
    tris = osc.array(O.W_TRIANGLES)
    ni, _, tlas_root = osc.instancing()
    return SceneDef(num_instances=ni, tlas_root=tlas_root,materials=osc.array(O.W_MATERIALS).view(L.MATERIAL),
                    primitives=osc.array(O.W_PRIMITIVES).view(L.PRIMITIVE),
                    lights=osc.array(O.W_LIGHTS).view(L.LIGHT),
                    positions=osc.array(O.W_POSITIONS).reshape(-1, 4),
                    vertex_attrs=osc.array(O.W_ATTRS).view(L.VERTEX_ATTR),
                    triangles=tris.view(L.TRIANGLE),
                    bvh_nodes=(osc.array(O.W_BVH_NODES).view(L.BVH_NODE) if with_bvh and len(tris) else None),
                    camera=Camera(eye=tuple(cam[0:3]), look_at=tuple(cam[3:6]), vfov_deg=float(cam[9]),
                                  up=tuple(cam[6:9])),
                    background=tuple(bg), env_pixels=env_px, env_cdf=env_cdf, env_total_weight=total)


def oracle_from_scene(s: SceneDef, bvh="sah") -> "O.Scene":
    """The oracle scene for a product SceneDef; a device-built instanced
    scene (meshes + placements) gets the oracle's restatement of the device
    BLAS/TLAS build."""
    if s.meshes is not None:
        osc = _oracle_arrays(s, "none")
        o2w, mesh, material = s.placements
        osc.build_instances_lbvh(s.meshes, o2w, mesh, material)
        return osc
    return _oracle_arrays(s, bvh)


def _oracle_arrays(s: SceneDef, bvh) -> "O.Scene":
    env = None
    w, h = s.env_size
    if w:
        env = (s.env_pixels.reshape(-1, 4), s.env_cdf[:h, :w + 1].reshape(-1), s.env_cdf[h, :h + 1],
               s.env_total_weight, w, h)
    cam = s.camera
    return O.Scene.from_arrays(s.materials.view(O.MATERIAL), s.primitives.view(O.PRIMITIVE), s.positions,
                               s.vertex_attrs.view(O.VERTEX_ATTR), s.triangles.view(O.TRIANGLE),
                               lights=s.lights.view(O.LIGHT), env=env, background=s.background,
                               camera=dict(eye=cam.eye, look_at=cam.look_at, vfov_deg=cam.vfov_deg, up=cam.up,
                                           aperture=cam.aperture, focus_distance=cam.focus_distance), bvh=bvh,
                               instancing=((s.bvh_nodes, s.num_instances, s.tlas_root) if s.num_instances else None))


def compare(a: np.ndarray, b: np.ndarray) -> dict:
    """image::compare over (..., 3) radiance arrays, plus per-pixel stats."""
    a = np.asarray(a, np.float64).reshape(-1, 3)
    b = np.asarray(b, np.float64).reshape(-1, 3)
    d = np.abs(a - b)
    rel = d / (np.abs(a) + np.abs(b) + 1e-4)
    px_rel = rel.max(axis=1)
    return {"rmse": float(np.sqrt((d * d).mean())), "max_abs": float(d.max()), "mean_rel": float(rel.mean()),
            "max_rel": float(px_rel.max()), "p999_rel": float(np.quantile(px_rel, 0.999)),
            "frac_within_1e3": float((px_rel <= 1e-3).mean()),
            "bit_exact": float((a == b).all(axis=1).mean()),
            "energy_ratio": float(a.sum() / max(b.sum(), 1e-30))}
