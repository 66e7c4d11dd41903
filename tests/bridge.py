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


def _px_rel(a, b):
    a = np.asarray(a, np.float64).reshape(-1, 3)
    b = np.asarray(b, np.float64).reshape(-1, 3)
    return (np.abs(a - b) / (np.abs(a) + np.abs(b) + 1e-4)).max(axis=1)


def parity(acc_radiance, osc: "O.Scene", u, label: str, ref_glibc=None, ref_double=None) -> dict:
    """The per-pixel parity bar (relative error <= 1e-3 per pixel) on a
    device render, against the oracle run both ways its transcendentals can
    round.

    * Against the oracle with transcendentals evaluated in double and rounded
      once (the rounding the CUDA integrator uses, so the two differ only
      where float operations could): the largest per-pixel relative error
      must be <= 1e-3 on every pixel.
    * Against the oracle with glibc's f32 functions (what the Rust reference
      calls): the reference's image metrics hold (mean relative error < 1e-4,
      energy within 1e-4, >= 99.9% of pixels within 1e-3), and every pixel
      beyond 1e-3 must lie where the two libm roundings already change the
      oracle's own result. Those pixels are classified per sample from the
      oracle's path signatures: a path flip (some sample took another branch:
      another primitive, a shadow-ray or lobe outcome) or an amplified
      rounding (the same branches; a near-singular factor such as a grazing
      light cosine magnified the last-bit difference).
    The counts are printed and returned."""
    acc = np.asarray(acc_radiance, np.float32).reshape(-1, 3)
    g = osc.render_sums(u) if ref_glibc is None else ref_glibc
    d = osc.render_sums(u, libm="double") if ref_double is None else ref_double
    st_d = compare(acc, d[:, 0:3])
    st_g = compare(acc, g[:, 0:3])
    rel_g = _px_rel(acc, g[:, 0:3])
    over = np.nonzero(rel_g > 1e-3)[0]
    libm_changes = np.any(d[:, 0:3] != g[:, 0:3], axis=1)
    flips = amplified = 0
    if len(over):
        _, sg = osc.sample_traces(u, over, libm="glibc")
        _, sd = osc.sample_traces(u, over, libm="double")
        flipped = np.any(sg != sd, axis=1)
        flips, amplified = int(flipped.sum()), int((~flipped).sum())
    out = {"max_rel_vs_double": st_d["max_rel"], "bit_exact_vs_double": st_d["bit_exact"],
           "max_rel_vs_glibc": st_g["max_rel"], "mean_rel_vs_glibc": st_g["mean_rel"],
           "over_1e3_vs_glibc": int(len(over)), "path_flips": flips, "amplified": amplified,
           "energy_ratio": st_g["energy_ratio"], "pixels": int(len(acc))}
    print(label, out)
    assert np.all(np.isfinite(acc)), label
    assert st_d["max_rel"] <= 1e-3, (label, out)
    assert np.all(libm_changes[over]), (label, "pixels beyond 1e-3 where the libm does not matter", over[~libm_changes[over]])
    assert st_g["frac_within_1e3"] >= 0.999, (label, out)
    assert st_g["mean_rel"] < 1e-4, (label, out)
    assert abs(st_g["energy_ratio"] - 1.0) < 1e-4, (label, out)
    return out
