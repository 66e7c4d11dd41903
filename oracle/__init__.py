"""ORACLE — test infrastructure only.

ctypes access to the CPU restatement of Lucida's Rust reference tracer
(crates/core/src), compiled from the C++ sources in this directory into
``liblucida_oracle.so``. Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module, and only as the checker;
the product (``lucida_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblucida_oracle.so")
_lib = None

# Record dtypes matching include/lucida_layout.h (gpu_layout.rs).
MATERIAL = np.dtype([("base_color", "<f4", 3), ("metallic", "<f4"), ("emissive", "<f4", 3),
                     ("roughness", "<f4"), ("ior", "<f4"), ("transmission", "<f4"),
                     ("_pad0", "<f4"), ("_pad1", "<f4"), ("eta", "<f4", 3), ("_pad2", "<f4"),
                     ("k", "<f4", 3), ("_pad3", "<f4")])
PRIMITIVE = np.dtype([("position", "<f4", 3), ("radius", "<f4"), ("edge_u", "<f4", 3), ("kind", "<u4"),
                      ("edge_v", "<f4", 3), ("material", "<u4"), ("normal", "<f4", 3), ("_pad0", "<f4")])
LIGHT = np.dtype([("origin", "<f4", 3), ("area", "<f4"), ("edge_u", "<f4", 3), ("kind", "<u4"),
                  ("edge_v", "<f4", 3), ("material", "<u4"), ("normal", "<f4", 3), ("_pad0", "<f4")])
VERTEX_ATTR = np.dtype([("normal", "<f4", 3), ("_pad0", "<f4"), ("uv", "<f4", 2), ("_pad1", "<f4", 2)])
TRIANGLE = np.dtype([("i0", "<u4"), ("i1", "<u4"), ("i2", "<u4"), ("material", "<u4")])
BVH_NODE = np.dtype([("bounds_min", "<f4", 3), ("left_first", "<u4"), ("bounds_max", "<f4", 3),
                     ("count", "<u4")])
assert MATERIAL.itemsize == 80 and PRIMITIVE.itemsize == 64 and LIGHT.itemsize == 64
assert VERTEX_ATTR.itemsize == 32 and TRIANGLE.itemsize == 16 and BVH_NODE.itemsize == 32


class Uniforms(C.Structure):
    """GpuUniforms (gpu_layout.rs:393-472), 160 bytes."""
    _fields_ = [("cam_origin", C.c_float * 3), ("lens_radius", C.c_float),
                ("cam_upper_left", C.c_float * 3), ("focus_distance", C.c_float),
                ("cam_horizontal", C.c_float * 3), ("_pad1", C.c_float),
                ("cam_vertical", C.c_float * 3), ("_pad2", C.c_float),
                ("width", C.c_uint32), ("height", C.c_uint32), ("sample_offset", C.c_uint32),
                ("samples_per_launch", C.c_uint32), ("max_depth", C.c_uint32), ("frame_seed", C.c_uint32),
                ("num_primitives", C.c_uint32), ("num_lights", C.c_uint32), ("background", C.c_float * 3),
                ("num_triangles", C.c_uint32), ("num_bvh_nodes", C.c_uint32), ("render_mode", C.c_uint32),
                ("sampling_mode", C.c_uint32), ("env_width", C.c_uint32), ("env_height", C.c_uint32),
                ("env_total_weight", C.c_float), ("sampler_kind", C.c_uint32), ("num_instances", C.c_uint32),
                ("tlas_root", C.c_uint32), ("_pad3", C.c_uint32), ("_pad4", C.c_uint32), ("_pad5", C.c_uint32)]


assert C.sizeof(Uniforms) == 160


def build() -> str:
    """Compile the restatement (make in this directory); returns the .so path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, u32, f32, i32, sz = C.c_void_p, C.c_uint32, C.c_float, C.c_int, C.c_size_t
        L.orc_scene_builtin.restype = vp
        L.orc_scene_builtin.argtypes = [C.c_char_p]
        L.orc_scene_from_arrays.restype = vp
        L.orc_scene_from_arrays.argtypes = [vp, u32, vp, u32, vp, u32, vp, u32, vp, vp, u32, vp, u32, u32,
                                            vp, vp, f32, vp, i32]
        L.orc_scene_free.argtypes = [vp]
        L.orc_scene_count.restype = sz
        L.orc_scene_count.argtypes = [vp, i32]
        L.orc_scene_copy.argtypes = [vp, i32, vp]
        L.orc_scene_set_camera.argtypes = [vp, vp, vp, vp, f32, f32, f32]
        L.orc_scene_get_camera.argtypes = [vp, vp]
        L.orc_scene_get_misc.argtypes = [vp, vp, vp, vp]
        L.orc_scene_set_instancing.argtypes = [vp, vp, u32, u32, u32]
        L.orc_scene_instancing.argtypes = [vp, vp]
        L.orc_scene_set_reference_shadows.argtypes = [vp, i32]
        L.orc_affine_inverse.argtypes = [vp, vp]
        L.orc_scene_build_instances_lbvh.argtypes = [vp, vp, vp, u32, vp, vp, vp, u32]
        L.orc_pack_instance.argtypes = [vp, u32, u32, vp]
        L.orc_instance_transform.argtypes = [vp, i32, vp, u32, vp]
        L.orc_instance_world_bounds.argtypes = [vp, vp, vp]
        L.orc_build_uniforms.argtypes = [vp, u32, u32, u32, u32, u32, u32, u32, u32, vp]
        L.orc_render_sums.argtypes = [vp, vp, u32, u32, u32, u32, vp]
        L.orc_render_row_list.argtypes = [vp, vp, u32, vp, u32, vp]
        L.orc_set_libm_mode.argtypes = [i32]
        L.orc_get_libm_mode.restype = i32
        L.orc_sample_traces.argtypes = [vp, vp, vp, u32, u32, vp, vp]
        L.orc_intersect_batch.argtypes = [vp, vp, u32, vp]
        for f in ("orc_pcg_hash", "orc_hash_u32", "orc_expand_bits"):
            getattr(L, f).restype = u32
            getattr(L, f).argtypes = [u32]
        L.orc_owen_scramble.restype = u32
        L.orc_owen_scramble.argtypes = [u32, u32]
        L.orc_sobol.restype = u32
        L.orc_sobol.argtypes = [u32, u32]
        L.orc_sobol_sample.restype = f32
        L.orc_sobol_sample.argtypes = [u32, u32, u32]
        L.orc_sampler_stream.argtypes = [u32, u32, u32, u32, C.c_char_p, vp]
        L.orc_energy_table.argtypes = [vp]
        L.orc_bsdf_eval_batch.argtypes = [vp, i32, vp, vp, u32, vp, vp]
        L.orc_bsdf_sample_batch.argtypes = [vp, i32, vp, vp, u32, vp, vp, vp]
        L.orc_env_sample_batch.argtypes = [vp, vp, u32, vp, vp, vp]
        L.orc_env_pdf_batch.argtypes = [vp, vp, u32, vp, vp]
        L.orc_env_build.restype = f32
        L.orc_env_build.argtypes = [vp, u32, u32, vp, vp]
        L.orc_lbvh_build.restype = vp
        L.orc_lbvh_build.argtypes = [vp, u32, vp, u32, u32]
        L.orc_lbvh_build_over_bounds.restype = vp
        L.orc_lbvh_build_over_bounds.argtypes = [vp, u32, u32]
        L.orc_lbvh_field.restype = sz
        L.orc_lbvh_field.argtypes = [vp, i32, vp]
        L.orc_lbvh_sah_cost.restype = f32
        L.orc_lbvh_sah_cost.argtypes = [vp]
        L.orc_lbvh_free.argtypes = [vp]
        L.orc_morton3d.restype = u32
        L.orc_morton3d.argtypes = [f32, f32, f32]
        L.orc_lcp.restype = C.c_int32
        L.orc_lcp.argtypes = [vp, C.c_int64, C.c_int32, C.c_int32]
        L.orc_sah_build.restype = vp
        L.orc_sah_build.argtypes = [vp, u32, vp, u32]
        L.orc_bvh_nodes.restype = sz
        L.orc_bvh_nodes.argtypes = [vp, vp]
        L.orc_bvh_prims.restype = sz
        L.orc_bvh_prims.argtypes = [vp, vp]
        L.orc_bvh_sah_cost.restype = f32
        L.orc_bvh_sah_cost.argtypes = [vp]
        L.orc_bvh_validate.restype = i32
        L.orc_bvh_validate.argtypes = [vp, u32]
        L.orc_bvh_free.argtypes = [vp]
        L.orc_nodes_sah_cost.restype = f32
        L.orc_nodes_sah_cost.argtypes = [vp, u32]
        L.orc_sort_pairs.argtypes = [vp, vp, u32, vp, vp]
        L.orc_denoise.argtypes = [vp, vp, vp, vp, u32, u32, u32, f32, f32, f32, f32, vp]
        L.orc_icosphere.restype = u32
        L.orc_icosphere.argtypes = [f32, f32, f32, f32, u32, vp, vp, vp, vp]
        L.orc_transcendental_batch.argtypes = [i32, vp, vp, u32, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


W_MATERIALS, W_PRIMITIVES, W_LIGHTS, W_POSITIONS, W_ATTRS, W_TRIANGLES, W_BVH_NODES, W_BVH_PRIMS, \
    W_ENV_PIXELS, W_ENV_COND, W_ENV_MARG = range(11)
_FIELD_DTYPES = {W_MATERIALS: MATERIAL, W_PRIMITIVES: PRIMITIVE, W_LIGHTS: LIGHT,
                 W_POSITIONS: np.dtype(("<f4", 4)), W_ATTRS: VERTEX_ATTR, W_TRIANGLES: TRIANGLE,
                 W_BVH_NODES: BVH_NODE, W_BVH_PRIMS: np.dtype("<u4"), W_ENV_PIXELS: np.dtype(("<f4", 4)),
                 W_ENV_COND: np.dtype("<f4"), W_ENV_MARG: np.dtype("<f4")}


class Scene:
    """A finalized oracle scene (crates/core Scene + camera + background)."""

    def __init__(self, handle):
        if not handle:
            raise ValueError("oracle scene construction failed")
        self._h = handle

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_scene_free(self._h)
            self._h = None

    @classmethod
    def builtin(cls, name: str) -> "Scene":
        return cls(lib().orc_scene_builtin(name.encode()))

    @classmethod
    def from_arrays(cls, materials, primitives, positions, vertex_attrs, triangles, lights=None,
                    env=None, background=(0.0, 0.0, 0.0), camera=None, bvh="sah", instancing=None) -> "Scene":
        """`env` = (pixels[h*w,4], conditional[(w+1)*h], marginal[h+1], total_weight, w, h).
        `instancing` = (flattened nodes, num_instances, tlas_root) for an
        instanced scene whose last num_instances primitives are instance rows."""
        L = lib()
        materials = np.ascontiguousarray(materials, MATERIAL)
        primitives = np.ascontiguousarray(primitives, PRIMITIVE)
        positions = np.ascontiguousarray(positions, np.float32).reshape(-1, 4)
        vertex_attrs = np.ascontiguousarray(vertex_attrs, VERTEX_ATTR)
        triangles = np.ascontiguousarray(triangles, TRIANGLE)
        lights_arr = None if lights is None else np.ascontiguousarray(lights, LIGHT)
        bg = np.asarray(background, np.float32)
        if env is not None:
            px, cond, marg, total, w, h = env
            px = np.ascontiguousarray(px, np.float32)
            cond = np.ascontiguousarray(cond, np.float32)
            marg = np.ascontiguousarray(marg, np.float32)
        else:
            px = cond = marg = None
            total, w, h = 0.0, 0, 0
        hnd = L.orc_scene_from_arrays(_p(materials), len(materials), _p(primitives), len(primitives),
                                      _p(lights_arr), 0 if lights_arr is None else len(lights_arr),
                                      _p(positions), len(positions), _p(vertex_attrs), _p(triangles),
                                      len(triangles), _p(px), w, h, _p(cond), _p(marg), float(total), _p(bg),
                                      2 if (instancing is not None or bvh == "none") else (1 if bvh == "lbvh" else 0))
        s = cls(hnd)
        if instancing is not None:
            nodes, ni, root = instancing
            nodes = np.ascontiguousarray(nodes, BVH_NODE)
            L.orc_scene_set_instancing(hnd, _p(nodes), len(nodes), int(ni), int(root))
        if camera is not None:
            s.set_camera(**camera)
        return s

    def instancing(self):
        """(instance count, analytic primitive count, TLAS root)."""
        out = np.zeros(3, np.uint32)
        lib().orc_scene_instancing(self._h, _p(out))
        return int(out[0]), int(out[1]), int(out[2])

    def build_instances_lbvh(self, meshes, object_to_world, mesh, material):
        """The device's luc_upload_meshes + luc_set_instances, restated."""
        ms = np.ascontiguousarray(meshes, np.uint32).reshape(-1, 2)
        first, count = np.ascontiguousarray(ms[:, 0]), np.ascontiguousarray(ms[:, 1])
        m = np.ascontiguousarray(object_to_world, np.float32).reshape(-1, 12)
        me = np.ascontiguousarray(mesh, np.uint32)
        mat = np.ascontiguousarray(material, np.uint32)
        lib().orc_scene_build_instances_lbvh(self._h, _p(first), _p(count), len(ms), _p(m), _p(me), _p(mat), len(m))

    def set_reference_shadows(self, on: bool):
        """Shadow rays of an instanced scene as the reference casts them
        (untransformed object-space triangles) instead of the two-level any-hit."""
        lib().orc_scene_set_reference_shadows(self._h, 1 if on else 0)

    def set_camera(self, eye, look_at, vfov_deg, up=(0.0, 1.0, 0.0), aperture=0.0, focus_distance=None):
        eye = np.asarray(eye, np.float32)
        at = np.asarray(look_at, np.float32)
        up = np.asarray(up, np.float32)
        if focus_distance is None:  # Camera::look_at: |look_at - eye| in f32
            d = (at - eye).astype(np.float32)
            focus_distance = np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1]) + np.float32(d[2] * d[2]))
        lib().orc_scene_set_camera(self._h, _p(eye), _p(at), _p(up), float(vfov_deg), float(aperture),
                                   float(np.float32(focus_distance)))

    def array(self, which: int) -> np.ndarray:
        L = lib()
        n = L.orc_scene_count(self._h, which)
        out = np.zeros(n, _FIELD_DTYPES[which])
        if n:
            L.orc_scene_copy(self._h, which, _p(out))
        return out

    def camera(self):
        out = np.zeros(10, np.float32)
        lib().orc_scene_get_camera(self._h, _p(out))
        return out

    def misc(self):
        bg = np.zeros(3, np.float32)
        tot = np.zeros(1, np.float32)
        wh = np.zeros(2, np.uint32)
        lib().orc_scene_get_misc(self._h, _p(bg), _p(tot), _p(wh))
        return bg, float(tot[0]), int(wh[0]), int(wh[1])

    def uniforms(self, width, height, spp, max_depth, frame_seed=0x5EED1234, sample_offset=0,
                 sampling=2, sampler=1) -> Uniforms:
        u = Uniforms()
        lib().orc_build_uniforms(self._h, width, height, spp, max_depth, frame_seed, sample_offset, sampling,
                                 sampler, C.byref(u))
        return u

    def render_sums(self, u: Uniforms, threads: int = 0, rows=None, band: int = 32,
                    libm: str = "glibc") -> np.ndarray:
        """Per-pixel [radiance sum 3, radiance^2 sum 3, albedo 3, normal 3, depth 1] in sample order,
        rows [r0, r1) handed to `threads` workers in `band`-row bands (integrator.rs:635-699 uses 32).
        `libm`: "glibc" (the reference's f32 transcendentals) or "double" (evaluated in double and
        rounded once, as the CUDA integrator rounds them)."""
        r0, r1 = (0, u.height) if rows is None else rows
        out = np.zeros(((r1 - r0) * u.width, 13), np.float32)
        with libm_mode(libm):
            lib().orc_render_sums(self._h, C.byref(u), threads, r0, r1, band, _p(out))
        return out

    def render_rows(self, u: Uniforms, rows, threads: int = 0) -> np.ndarray:
        """render_sums over an explicit list of image rows, one row per work item over `threads`
        workers (0 = every core); (len(rows) * width, 13), rows in list order."""
        rows = np.ascontiguousarray(rows, np.uint32).reshape(-1)
        assert rows.size == 0 or int(rows.max()) < u.height
        out = np.zeros((len(rows) * u.width, 13), np.float32)
        lib().orc_render_row_list(self._h, C.byref(u), threads, _p(rows), len(rows), _p(out))
        return out

    def sample_traces(self, u: Uniforms, pixels, libm: str = "glibc", threads: int = 0):
        """Every sample of the listed pixels (indices y * width + x) traced on its own: radiance
        (n, spp, 3) and path signatures (n, spp) u64 — a hash of the path's discrete events (the
        primitive each ray hit, shadow-ray outcomes, BSDF lobe choices and rejections, light picks)."""
        pixels = np.ascontiguousarray(pixels, np.uint32).reshape(-1)
        n, spp = len(pixels), u.samples_per_launch
        rad = np.zeros((n, spp, 3), np.float32)
        sig = np.zeros((n, spp), np.uint64)
        with libm_mode(libm):
            lib().orc_sample_traces(self._h, C.byref(u), _p(pixels), n, threads, _p(rad), _p(sig))
        return rad, sig

    def intersect(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        out = np.zeros((len(rays), 12), np.float32)
        lib().orc_intersect_batch(self._h, _p(rays), len(rays), _p(out))
        return out

    def env_sample(self, u2):
        u2 = np.ascontiguousarray(u2, np.float32).reshape(-1, 2)
        n = len(u2)
        d, r, p = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        lib().orc_env_sample_batch(self._h, _p(u2), n, _p(d), _p(r), _p(p))
        return d, r, p


class libm_mode:
    """Context manager: render-time transcendentals as glibc's f32 functions ("glibc", the
    reference's) or evaluated in double and rounded once ("double", the CUDA integrator's)."""

    def __init__(self, mode: str):
        if mode not in ("glibc", "double"):
            raise ValueError(mode)
        self.mode = 1 if mode == "double" else 0

    def __enter__(self):
        self.prev = lib().orc_get_libm_mode()
        lib().orc_set_libm_mode(self.mode)
        return self

    def __exit__(self, *exc):
        lib().orc_set_libm_mode(self.prev)


def sampler_stream(kind, frame_seed, pixel, sample, pattern: str) -> np.ndarray:
    n = sum(2 if c == "v" else 1 for c in pattern)
    out = np.zeros(n, np.float32)
    lib().orc_sampler_stream(kind, frame_seed, pixel, sample, pattern.encode(), _p(out))
    return out


def energy_table() -> np.ndarray:
    out = np.zeros(32 * 32, np.float32)
    lib().orc_energy_table(_p(out))
    return out


def bsdf_eval(material, front, wo, wi):
    m = np.ascontiguousarray(np.asarray(material, MATERIAL).reshape(1))
    wo = np.ascontiguousarray(wo, np.float32).reshape(-1, 3)
    wi = np.ascontiguousarray(wi, np.float32).reshape(-1, 3)
    f = np.zeros_like(wo)
    pdf = np.zeros(len(wo), np.float32)
    lib().orc_bsdf_eval_batch(_p(m), int(front), _p(wo), _p(wi), len(wo), _p(f), _p(pdf))
    return f, pdf


def bsdf_sample(material, front, wo, u3):
    m = np.ascontiguousarray(np.asarray(material, MATERIAL).reshape(1))
    wo = np.ascontiguousarray(wo, np.float32).reshape(-1, 3)
    u3 = np.ascontiguousarray(u3, np.float32).reshape(-1, 3)
    wi, w = np.zeros_like(wo), np.zeros_like(wo)
    pdf = np.zeros(len(wo), np.float32)
    lib().orc_bsdf_sample_batch(_p(m), int(front), _p(wo), _p(u3), len(wo), _p(wi), _p(w), _p(pdf))
    return wi, w, pdf


def env_build(pixels4: np.ndarray, w: int, h: int):
    px = np.ascontiguousarray(pixels4, np.float32)
    cond = np.zeros((w + 1) * h, np.float32)
    marg = np.zeros(h + 1, np.float32)
    tot = lib().orc_env_build(_p(px), w, h, _p(cond), _p(marg))
    return cond, marg, float(tot)


class Lbvh:
    """Every stage of the CPU LBVH build (lbvh.rs:422-538)."""
    FIELDS = {"tri_bounds": (0, "box"), "centroid_bounds": (1, "box"), "codes": (2, "u32"),
              "order": (3, "u32"), "sorted_codes": (4, "u32"), "karras": (5, "u32"), "parent": (6, "u32"),
              "node_bounds": (7, "box"), "subtree_size": (8, "u32"), "nodes": (9, "node"),
              "prim_indices": (10, "u32")}

    def __init__(self, triangles=None, positions=None, max_leaf=4, boxes=None):
        L = lib()
        if boxes is not None:
            b = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
            self._h = L.orc_lbvh_build_over_bounds(_p(b), len(b), max_leaf)
        else:
            t = np.ascontiguousarray(triangles, TRIANGLE)
            p = np.ascontiguousarray(positions, np.float32).reshape(-1, 4)
            self._h = L.orc_lbvh_build(_p(t), len(t), _p(p), len(p), max_leaf)
        for name, (fid, kind) in self.FIELDS.items():
            n = L.orc_lbvh_field(self._h, fid, None)
            if kind == "box":
                a = np.zeros((n, 6), np.float32)
            elif kind == "node":
                a = np.zeros(n, BVH_NODE)
            else:
                a = np.zeros(n, np.uint32)
            if n:
                L.orc_lbvh_field(self._h, fid, _p(a))
            setattr(self, name, a)
        self.sah_cost = L.orc_lbvh_sah_cost(self._h)
        L.orc_lbvh_free(self._h)
        self._h = None


def sah_build(triangles, positions):
    L = lib()
    t = np.ascontiguousarray(triangles, TRIANGLE)
    p = np.ascontiguousarray(positions, np.float32).reshape(-1, 4)
    h = L.orc_sah_build(_p(t), len(t), _p(p), len(p))
    nodes = np.zeros(L.orc_bvh_nodes(h, None), BVH_NODE)
    prims = np.zeros(L.orc_bvh_prims(h, None), np.uint32)
    L.orc_bvh_nodes(h, _p(nodes))
    L.orc_bvh_prims(h, _p(prims))
    cost = L.orc_bvh_sah_cost(h)
    problems = L.orc_bvh_validate(h, len(t))
    L.orc_bvh_free(h)
    return nodes, prims, cost, problems


def nodes_sah_cost(nodes) -> float:
    n = np.ascontiguousarray(nodes, BVH_NODE)
    return float(lib().orc_nodes_sah_cost(_p(n), len(n)))


def sort_pairs(keys, vals):
    k = np.ascontiguousarray(keys, np.uint32)
    v = np.ascontiguousarray(vals, np.uint32)
    ko, vo = np.zeros_like(k), np.zeros_like(v)
    lib().orc_sort_pairs(_p(k), _p(v), len(k), _p(ko), _p(vo))
    return ko, vo


def denoise(film, albedo, normal, depth, w, h, iterations=4, sigma_normal=64.0, sigma_depth=0.08,
            sigma_luminance=4.0, sigma_albedo=0.1):
    f = np.ascontiguousarray(film, np.float32).reshape(-1, 3)
    a = np.ascontiguousarray(albedo, np.float32).reshape(-1, 3)
    n = np.ascontiguousarray(normal, np.float32).reshape(-1, 3)
    d = np.ascontiguousarray(depth, np.float32).reshape(-1)
    out = np.zeros_like(f)
    lib().orc_denoise(_p(f), _p(a), _p(n), _p(d), w, h, iterations, sigma_normal, sigma_depth,
                      sigma_luminance, sigma_albedo, _p(out))
    return out


def icosphere(center, radius, levels):
    L = lib()
    nv = L.orc_icosphere(center[0], center[1], center[2], radius, levels, None, None, None, None)
    nt = 20 * 4 ** levels
    pos = np.zeros((nv, 4), np.float32)
    nrm = np.zeros((nv, 3), np.float32)
    uv = np.zeros((nv, 2), np.float32)
    idx = np.zeros((nt, 3), np.uint32)
    L.orc_icosphere(center[0], center[1], center[2], radius, levels, _p(pos), _p(nrm), _p(uv), _p(idx))
    return pos, nrm, uv, idx


def transcendental(fn: str, x, y=None) -> np.ndarray:
    code = {"sin": 0, "cos": 1, "acos": 2, "atan2": 3, "exp": 4, "pow": 5, "asin": 6, "tan": 7}[fn]
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(np.zeros_like(x) if y is None else y, np.float32)
    out = np.zeros_like(x)
    lib().orc_transcendental_batch(code, _p(x), _p(y), len(x), _p(out))
    return out


# ---------------------------------------------------------------- instance maths
def affine_inverse(m34):
    m = np.ascontiguousarray(m34, np.float32).reshape(3, 4)
    out = np.zeros((3, 4), np.float32)
    lib().orc_affine_inverse(_p(m), _p(out))
    return out


def pack_instance(world_to_object34, blas_root=0, material=0xFFFFFFFF):
    m = np.ascontiguousarray(world_to_object34, np.float32).reshape(3, 4)
    out = np.zeros(1, PRIMITIVE)
    lib().orc_pack_instance(_p(m), int(blas_root), int(material), _p(out))
    return out[0]


def instance_transform(inst, v, mode):
    """mode 0: points, 1: vectors (not normalised), 2: normals."""
    g = np.ascontiguousarray(np.asarray(inst, PRIMITIVE).reshape(1))
    a = np.ascontiguousarray(v, np.float32).reshape(-1, 3)
    out = np.zeros_like(a)
    lib().orc_instance_transform(_p(g), int(mode), _p(a), len(a), _p(out))
    return out


def instance_world_bounds(inst, box6):
    g = np.ascontiguousarray(np.asarray(inst, PRIMITIVE).reshape(1))
    b = np.ascontiguousarray(box6, np.float32).reshape(6)
    out = np.zeros(6, np.float32)
    lib().orc_instance_world_bounds(_p(g), _p(b), _p(out))
    return out
