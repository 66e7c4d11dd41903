"""numpy / ctypes views of the boundary structs (include/lucida_layout.h,
restating crates/core/src/gpu_layout.rs)."""
from __future__ import annotations

import ctypes as C

import numpy as np

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
ACCUM = np.dtype([("radiance", "<f4", 3), ("samples", "<f4"), ("albedo", "<f4", 3), ("depth", "<f4"),
                  ("normal", "<f4", 3), ("traversal", "<f4"), ("radiance_sq", "<f4", 3), ("_pad0", "<f4")])
for _dt, _n in ((MATERIAL, 80), (PRIMITIVE, 64), (LIGHT, 64), (VERTEX_ATTR, 32), (TRIANGLE, 16),
                (BVH_NODE, 32), (ACCUM, 64)):
    assert _dt.itemsize == _n

PRIM_KIND_SPHERE, PRIM_KIND_QUAD, PRIM_KIND_INSTANCE = 0, 1, 2
LIGHT_KIND_QUAD, LIGHT_KIND_TRIANGLE = 0, 1
SAMPLING = {"bsdf": 0, "nee": 1, "mis": 2}
SAMPLER = {"independent": 0, "sobol": 1}


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


def uniforms_from_bytes(b: bytes) -> Uniforms:
    u = Uniforms()
    C.memmove(C.byref(u), b, 160)
    return u


def material(base_color=(0, 0, 0), metallic=0.0, emissive=(0, 0, 0), roughness=1.0, ior=1.5,
             transmission=0.0, eta=(0, 0, 0), k=(0, 0, 0)):
    m = np.zeros(1, MATERIAL)
    m["base_color"] = base_color
    m["metallic"] = metallic
    m["emissive"] = emissive
    m["roughness"] = roughness
    m["ior"] = ior
    m["transmission"] = transmission
    m["eta"] = eta
    m["k"] = k
    return m[0]


# The GpuMaterial constructors of gpu_layout.rs:77-168.
def diffuse(c):
    return material(base_color=c, roughness=1.0, ior=1.5)


def glossy(c, roughness):
    return material(base_color=c, roughness=roughness, ior=1.5)


def metal(c, roughness):
    return material(base_color=c, metallic=1.0, roughness=roughness, ior=1.5)


def glass(tint, roughness, ior):
    return material(base_color=tint, roughness=roughness, ior=ior, transmission=1.0)


def emissive(radiance):
    return material(base_color=(0, 0, 0), emissive=radiance, roughness=1.0, ior=1.0)


def _cross32(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    return np.array([np.float32(a[1] * b[2]) - np.float32(b[1] * a[2]),
                     np.float32(a[2] * b[0]) - np.float32(b[2] * a[0]),
                     np.float32(a[0] * b[1]) - np.float32(b[0] * a[1])], np.float32)


def _normalize32(v):
    v = np.asarray(v, np.float32)
    d = np.float32(np.float32(np.float32(v[0] * v[0]) + np.float32(v[1] * v[1])) + np.float32(v[2] * v[2]))
    r = np.float32(np.float32(1.0) / np.sqrt(d))
    return (v * r).astype(np.float32)


def sphere(center, radius, mat):  # gpu_layout.rs:214-222
    p = np.zeros(1, PRIMITIVE)
    p["position"] = center
    p["radius"] = radius
    p["kind"] = PRIM_KIND_SPHERE
    p["material"] = mat
    return p[0]


def quad(origin, edge_u, edge_v, mat):  # gpu_layout.rs:229-239
    p = np.zeros(1, PRIMITIVE)
    p["position"] = origin
    p["edge_u"] = edge_u
    p["edge_v"] = edge_v
    p["kind"] = PRIM_KIND_QUAD
    p["material"] = mat
    p["normal"] = _normalize32(_cross32(edge_u, edge_v))
    return p[0]


def quad_lights(materials, primitives):
    """light::build_lights (light.rs:62-123) for the analytic quads."""
    out = []
    for p in primitives:
        if p["kind"] != PRIM_KIND_QUAD or not (materials[p["material"]]["emissive"] > 0).any():
            continue
        cr = _cross32(p["edge_u"], p["edge_v"])
        l = np.zeros(1, LIGHT)
        l["origin"] = p["position"]
        l["area"] = np.sqrt(np.float32(np.float32(np.float32(cr[0] * cr[0]) + np.float32(cr[1] * cr[1]))
                                       + np.float32(cr[2] * cr[2])))
        l["edge_u"] = p["edge_u"]
        l["edge_v"] = p["edge_v"]
        l["kind"] = LIGHT_KIND_QUAD
        l["material"] = p["material"]
        l["normal"] = p["normal"]
        out.append(l[0])
    return np.array(out, LIGHT)
