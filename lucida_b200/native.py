"""ctypes binding of liblucida_cuda.so (include/luc_cuda.h).

The library is built in-tree by lucida_b200/build.py. Loading fails loudly
when it is missing: there is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import layout as L

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblucida_cuda.so")

LUC_OK = 0
ERRORS = {-1: "NoDevice", -2: "Launch", -3: "Readback", -4: "Validation", -5: "OutOfMemory"}
LUC_FLAG_NO_GUIDES = 0x100
LUC_FLAG_PROFILE = 0x200
LUC_FLAG_GUIDED = 0x400
LUC_FLAG_REFERENCE_SHADOWS = 0x800
LUC_FLAG_MEASURE = 0x1000
LUC_DEBUG_NONE, LUC_DEBUG_SORT_ORPHAN_TILE, LUC_DEBUG_TC_NO_COMMIT = 0, 1, 2
LUC_ARCH_WAVEFRONT = 0x0
LUC_ARCH_MEGAKERNEL = 0x1
LUC_DENOISE_HALF_GUIDES = 0x1


class GpuError(RuntimeError):
    """pt_gpu::GpuError (crates/gpu/src/lib.rs:100-112): `kind` is one of
    NoDevice, Launch (Shader), Readback, Validation, OutOfMemory."""

    def __init__(self, code: int, message: str):
        self.code = code
        self.kind = ERRORS.get(code, f"Unknown({code})")
        super().__init__(f"{self.kind}: {message}")


class SceneView(C.Structure):
    _fields_ = [("materials", C.c_void_p), ("num_materials", C.c_uint32),
                ("primitives", C.c_void_p), ("num_primitives", C.c_uint32), ("num_instances", C.c_uint32),
                ("lights", C.c_void_p), ("num_lights", C.c_uint32),
                ("positions", C.c_void_p), ("vertex_attrs", C.c_void_p), ("num_vertices", C.c_uint32),
                ("triangles", C.c_void_p), ("num_triangles", C.c_uint32),
                ("bvh_nodes", C.c_void_p), ("num_bvh_nodes", C.c_uint32), ("tlas_root", C.c_uint32),
                ("env_pixels", C.c_void_p), ("env_width", C.c_uint32), ("env_height", C.c_uint32),
                ("env_cdf", C.c_void_p), ("env_cdf_width", C.c_uint32), ("env_total_weight", C.c_float)]


class LbvhOut(C.Structure):
    _fields_ = [("codes", C.c_void_p), ("order", C.c_void_p), ("karras", C.c_void_p), ("parent", C.c_void_p),
                ("node_bounds", C.c_void_p), ("subtree_size", C.c_void_p), ("scene_bounds", C.c_void_p),
                ("nodes", C.c_void_p), ("prim_indices", C.c_void_p), ("num_nodes", C.c_uint32)]


class DenoiseParams(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("sigma_normal", C.c_float), ("sigma_depth", C.c_float),
                ("sigma_luminance", C.c_float), ("sigma_albedo", C.c_float)]


class RenderStats(C.Structure):
    _fields_ = [("ms_total", C.c_double), ("ms_generate", C.c_double), ("ms_extend", C.c_double),
                ("ms_shade", C.c_double), ("ms_connect", C.c_double), ("ms_resolve", C.c_double),
                ("launches", C.c_uint64), ("rays_extend", C.c_uint64), ("rays_shadow", C.c_uint64),
                ("paths", C.c_uint64), ("nodes_extend", C.c_uint64), ("tris_extend", C.c_uint64),
                ("nodes_shadow", C.c_uint64), ("tris_shadow", C.c_uint64), ("ms_guide", C.c_double),
                ("ms_train", C.c_double), ("convergence", C.c_double), ("blas_extend", C.c_uint64),
                ("blas_shadow", C.c_uint64)]


class BatchJob(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("uniforms", L.Uniforms), ("spp", C.c_uint32), ("max_depth", C.c_uint32),
                ("accum_dev", C.c_void_p)]


class BatchConfig(C.Structure):
    _fields_ = [("block", C.c_uint32), ("chunk", C.c_uint32)]


class GuideInfo(C.Structure):
    _fields_ = [("steps", C.c_uint32), ("last_records", C.c_uint32), ("last_loss", C.c_float),
                ("threshold", C.c_uint32), ("num_params", C.c_uint32), ("tc_error", C.c_uint32)]


# Every entry point include/luc_cuda.h declares, with its ctypes signature.
_SIGS = {
    "luc_layout_version": (C.c_uint32, []),
    "luc_sizeof": (C.c_uint32, [C.c_uint32]),
    "luc_create": (C.c_int32, [C.c_int32, C.POINTER(C.c_void_p)]),
    "luc_destroy": (None, [C.c_void_p]),
    "luc_last_error": (C.c_char_p, [C.c_void_p]),
    "luc_set_stream": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "luc_upload_scene": (C.c_int32, [C.c_void_p, C.POINTER(SceneView)]),
    "luc_render": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                               C.c_void_p]),
    "luc_get_stats": (C.c_int32, [C.c_void_p, C.POINTER(RenderStats)]),
    "luc_camera_uniforms": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float,
                                        C.c_uint32, C.c_uint32, C.c_void_p]),
    "luc_lbvh_build": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32,
                                   C.POINTER(LbvhOut)]),
    "luc_lbvh_build_boxes": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(LbvhOut)]),
    "luc_sort_u32": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    "luc_sort_u32_dev": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    "luc_eval_bsdf": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_uint32,
                                  C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "luc_eval_env": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int32, C.c_void_p, C.c_void_p,
                                 C.c_void_p]),
    "luc_intersect": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int32, C.c_void_p]),
    "luc_convergence": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "luc_read_sweep": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p]),
    "luc_accum_merge": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]),
    "luc_debug_waits": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_uint32]),
    "luc_set_tlas_leaf": (C.c_int32, [C.c_void_p, C.c_uint32]),
    "luc_sort_u32_static": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_char_p,
                                        C.c_uint32]),
    "luc_sort_u32_static_max": (C.c_uint32, []),
    "luc_denoise": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(DenoiseParams),
                                C.c_void_p]),
    "luc_denoise_dev": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(DenoiseParams),
                                    C.c_uint32, C.c_void_p]),
    "luc_batch_configure": (C.c_int32, [C.c_void_p, C.POINTER(BatchConfig)]),
    "luc_render_batch": (C.c_int32, [C.c_void_p, C.POINTER(BatchJob), C.c_uint32, C.c_void_p, C.POINTER(RenderStats)]),
    "luc_batch_autotune": (C.c_int32, [C.c_void_p, C.POINTER(BatchJob), C.c_uint32, C.c_uint32,
                                       C.POINTER(BatchConfig), C.c_void_p]),
    "luc_upload_meshes": (C.c_int32, [C.c_void_p, C.POINTER(SceneView), C.c_void_p, C.c_void_p, C.c_uint32]),
    "luc_set_instances": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]),
    "luc_read_scene": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    "luc_guide_init": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    "luc_guide_configure": (C.c_int32, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_float]),
    "luc_guide_get_params": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "luc_guide_stats": (C.c_int32, [C.c_void_p, C.POINTER(GuideInfo)]),
    "luc_guide_forward": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]),
    "luc_guide_forward_ex": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_int32, C.c_void_p]),
    "luc_guide_train_records": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                            C.c_void_p]),
    "luc_guide_mixture": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_int32, C.c_void_p,
                                      C.c_void_p]),
}

_lib = None


def lib():
    """Load liblucida_cuda.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m lucida_b200.build` "
                               "(there is no CPU fallback)")
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def check(ctx, rc: int):
    if rc != LUC_OK:
        msg = lib().luc_last_error(ctx).decode(errors="replace") if ctx else ""
        raise GpuError(rc, msg)


def camera_uniforms(eye, look_at, vfov_deg, width, height, up=(0.0, 1.0, 0.0), aperture=0.0,
                    focus_distance=None) -> L.Uniforms:
    e = np.asarray(eye, np.float32)
    a = np.asarray(look_at, np.float32)
    u = np.asarray(up, np.float32)
    if focus_distance is None:  # Camera::look_at (camera.rs:318-327): |look_at - eye| in f32
        d = (a - e).astype(np.float32)
        focus_distance = np.float32(np.sqrt(np.float32(np.float32(d[0] * d[0]) + np.float32(d[1] * d[1]))
                                            + np.float32(d[2] * d[2])))
    out = L.Uniforms()
    check(None, lib().luc_camera_uniforms(ptr(e), ptr(a), ptr(u), float(vfov_deg), float(aperture),
                                          float(focus_distance), int(width), int(height), C.byref(out)))
    return out
