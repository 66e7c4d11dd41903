"""The host-side mirror of Lucida's `pt_gpu` crate (crates/gpu/src), backed by
the CUDA library through its C ABI.

    pt_gpu::Gpu::new()                      -> Gpu(device)
    pt_gpu::render_with(gpu, def, params, Architecture::Wavefront)
                                            -> render_with(gpu, scene, params)
    pt_gpu::wavefront::render_native_on     -> render_native_on(gpu, scene, params)
    pt_gpu::render_native_denoised          -> render_native_denoised(...)
    pt_gpu::lbvh::LbvhBuilder               -> LbvhBuilder(gpu)
    pt_gpu::GpuError                        -> GpuError

Names, argument meaning and error behaviour follow the reference; images come
back as `Film` (row 0 = top, radiance / samples, like
crates/gpu/src/lib.rs:600-627 read_accum).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import layout as L
from .native import (LUC_ARCH_MEGAKERNEL, LUC_ARCH_WAVEFRONT, LUC_FLAG_GUIDED, LUC_FLAG_MEASURE,
                     LUC_FLAG_NO_GUIDES, LUC_FLAG_PROFILE, LUC_FLAG_REFERENCE_SHADOWS, DenoiseParams as _DP, GpuError, LbvhOut, RenderStats, SceneView, camera_uniforms, check, lib,
                     ptr)

__all__ = ["Gpu", "SceneDef", "Camera", "RenderParams", "Film", "render_with", "render_native_on",
           "render_accum", "render_native_denoised", "LbvhBuilder", "GpuBuildOutput", "DenoiseParams",
           "GpuError", "Denoiser", "render_with_measured", "measure_convergence", "convergence"]


@dataclass
class Camera:
    """crates/core/src/camera.rs:302-327 (Camera::look_at when focus is None)."""
    eye: tuple
    look_at: tuple
    vfov_deg: float
    up: tuple = (0.0, 1.0, 0.0)
    aperture: float = 0.0
    focus_distance: float | None = None


@dataclass
class SceneDef:
    """The SceneBlob arrays (gpu_layout.rs:706-770) plus camera, background
    and the environment map (pixels RGBA32F, packed CDF, total weight)."""
    materials: np.ndarray
    primitives: np.ndarray = field(default_factory=lambda: np.zeros(0, L.PRIMITIVE))
    lights: np.ndarray = field(default_factory=lambda: np.zeros(0, L.LIGHT))
    positions: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.float32))
    vertex_attrs: np.ndarray = field(default_factory=lambda: np.zeros(0, L.VERTEX_ATTR))
    triangles: np.ndarray = field(default_factory=lambda: np.zeros(0, L.TRIANGLE))
    bvh_nodes: np.ndarray | None = None  # None: the device builds an LBVH
    camera: Camera | None = None
    background: tuple = (0.0, 0.0, 0.0)
    env_pixels: np.ndarray | None = None  # (h, w, 4) float32
    env_cdf: np.ndarray | None = None  # (h + 1, cdf_w) float32, lib.rs:322-338 packing
    env_total_weight: float = 0.0
    name: str = "scene"
    # Instanced scenes (scene.rs:252-345 layout): the last `num_instances`
    # rows of `primitives` are GpuInstance rows in TLAS-leaf order and
    # `bvh_nodes` holds every BLAS followed by the TLAS from `tlas_root` on.
    num_instances: int = 0
    tlas_root: int = 0
    # Device-built instancing: `meshes` (M, 2) = (first triangle, count) per
    # mesh of object-space triangles (one LBVH each, luc_upload_meshes) and
    # `placements` = (object_to_world (N, 3, 4), mesh (N,), material (N,),
    # 0xFFFFFFFF keeping the triangles' own) for the TLAS (luc_set_instances).
    meshes: np.ndarray | None = None
    placements: tuple | None = None

    @property
    def env_size(self):
        if self.env_pixels is None:
            return 0, 0
        return self.env_pixels.shape[1], self.env_pixels.shape[0]


@dataclass
class RenderParams:
    """integrator::RenderParams (crates/core/src/integrator.rs:96-127)."""
    width: int = 512
    height: int = 512
    samples: int = 256
    max_depth: int = 8
    frame_seed: int = 0x5EED1234
    sample_offset: int = 0
    sampling: str = "mis"
    sampler: str = "sobol"


@dataclass
class DenoiseParams:
    """denoise::DenoiseParams (crates/core/src/denoise.rs:62-94)."""
    iterations: int = 4
    sigma_normal: float = 64.0
    sigma_depth: float = 0.08
    sigma_luminance: float = 4.0
    sigma_albedo: float = 0.1


class Film:
    """A linear-HDR image, row-major, row 0 = top (integrator.rs:129-148)."""

    def __init__(self, width, height, data):
        self.width, self.height = width, height
        self.data = data  # (height, width, 3) float32

    def pixel(self, x, y):
        return self.data[y, x]


class Gpu:
    """pt_gpu::Gpu — one CUDA context (device + stream + resident scene)."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        h = C.c_void_p()
        check(None, self._lib.luc_create(device, C.byref(h)))
        self._h = h
        self._scene = None  # strong reference: an id() could be reused after a free

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.luc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle: int | None):
        """Run on a caller's cudaStream_t (e.g. torch.cuda.current_stream().cuda_stream).
        None returns to the context's own stream; 0, the legacy default
        stream's handle in torch, is passed as cudaStreamLegacy so the
        library's work stays ordered with torch's default-stream work."""
        handle = None if stream_handle is None else (stream_handle if stream_handle != 0 else 1)
        check(self._h, self._lib.luc_set_stream(self._h, C.c_void_p(handle)))

    def upload(self, scene: SceneDef, force: bool = False):
        """Make `scene` resident. A SceneDef already resident is not sent
        again unless `force` (use it after mutating the arrays in place)."""
        if self._scene is scene and not force:
            return
        v = SceneView()
        keep = []

        def arr(a, dt):
            a = np.ascontiguousarray(a, dt)
            keep.append(a)
            return a

        m = arr(scene.materials, L.MATERIAL)
        v.materials, v.num_materials = ptr(m), len(m)
        p = arr(scene.primitives, L.PRIMITIVE)
        v.primitives, v.num_primitives, v.num_instances = ptr(p), len(p) - scene.num_instances, scene.num_instances
        v.tlas_root = scene.tlas_root
        li = arr(scene.lights, L.LIGHT)
        v.lights, v.num_lights = ptr(li), len(li)
        pos = arr(scene.positions, np.float32).reshape(-1, 4)
        at = arr(scene.vertex_attrs, L.VERTEX_ATTR)
        v.positions, v.vertex_attrs, v.num_vertices = ptr(pos), ptr(at), len(pos)
        t = arr(scene.triangles, L.TRIANGLE)
        v.triangles, v.num_triangles = ptr(t), len(t)
        if scene.bvh_nodes is not None and len(scene.bvh_nodes):
            n = arr(scene.bvh_nodes, L.BVH_NODE)
            v.bvh_nodes, v.num_bvh_nodes = ptr(n), len(n)
        w, h = scene.env_size
        if w:
            px = arr(scene.env_pixels, np.float32).reshape(h, w, 4)
            cdf = arr(scene.env_cdf, np.float32)
            v.env_pixels, v.env_width, v.env_height = ptr(px), w, h
            v.env_cdf, v.env_cdf_width = ptr(cdf), cdf.shape[1]
            v.env_total_weight = float(scene.env_total_weight)
        self._scene = None
        if scene.meshes is not None:
            ms = np.ascontiguousarray(scene.meshes, np.uint32).reshape(-1, 2)
            first, count = np.ascontiguousarray(ms[:, 0]), np.ascontiguousarray(ms[:, 1])
            check(self._h, self._lib.luc_upload_meshes(self._h, C.byref(v), ptr(first), ptr(count), len(ms)))
            if scene.placements is not None:
                self.set_instances(*scene.placements)
        else:
            check(self._h, self._lib.luc_upload_scene(self._h, C.byref(v)))
        self._scene = scene

    def set_tlas_leaf(self, max_leaf: int):
        """Leaf size of the TLAS the next instance placement builds
        (luc_set_tlas_leaf): 4 reproduces the reference's node layout, the
        default 1 renders the same image faster."""
        check(self._h, self._lib.luc_set_tlas_leaf(self._h, int(max_leaf)))

    def set_instances(self, object_to_world, mesh, material=None):
        """Place the uploaded meshes (luc_set_instances): rebuilds the TLAS on
        the device. object_to_world (N, 3, 4) row-major; material None keeps
        every triangle's own."""
        m = np.ascontiguousarray(object_to_world, np.float32).reshape(-1, 12)
        me = np.ascontiguousarray(mesh, np.uint32).reshape(-1)
        mat = (np.full(len(m), 0xFFFFFFFF, np.uint32) if material is None
               else np.ascontiguousarray(material, np.uint32).reshape(-1))
        if not (len(m) == len(me) == len(mat)):
            raise ValueError("object_to_world, mesh and material must have one entry per instance")
        check(self._h, self._lib.luc_set_instances(self._h, ptr(m), ptr(me), ptr(mat), len(m)))

    def read_scene(self, which: str) -> np.ndarray:
        """The resident scene's 'nodes', 'triangles' or 'primitives' (instance
        rows after the analytic primitives); 'wide_nodes' (uint32 rows of 20
        words) and 'wide_soup' (float32 rows of 12) of the compressed 8-wide
        tree, empty when the scene traverses the binary tree."""
        code, dt = {"nodes": (0, L.BVH_NODE), "triangles": (1, L.TRIANGLE), "primitives": (2, L.PRIMITIVE),
                    "wide_nodes": (3, np.dtype((np.uint32, 20))), "wide_soup": (4, np.dtype((np.float32, 12)))}[which]
        n = C.c_uint64(0)
        check(self._h, self._lib.luc_read_scene(self._h, code, None, 0, C.byref(n)))
        out = np.zeros(n.value // dt.itemsize, dt)
        check(self._h, self._lib.luc_read_scene(self._h, code, ptr(out), out.nbytes, C.byref(n)))
        return out

    def intersect(self, origins, directions, t_max=None):
        """Closest hits of rays against the resident scene: (t, u, v, id)
        with id uint32 (0xFFFFFFFF on a miss). With `t_max`, the occlusion
        query within (1e-4, t_max) instead: a bool per ray."""
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, np.float32).reshape(-1, 3)
        rays = np.zeros((len(o), 8), np.float32)
        rays[:, 0:3], rays[:, 4:7] = o, d
        if t_max is None:
            out = np.zeros((len(o), 4), np.float32)
            check(self._h, self._lib.luc_intersect(self._h, ptr(rays), len(o), 0, ptr(out)))
            return out[:, 0], out[:, 1], out[:, 2], out[:, 3].view(np.uint32)
        rays[:, 3] = np.broadcast_to(np.asarray(t_max, np.float32), len(o))
        occ = np.zeros(len(o), np.uint32)
        check(self._h, self._lib.luc_intersect(self._h, ptr(rays), len(o), 1, ptr(occ)))
        return occ.astype(bool)

    def env_sample(self, u2):
        """EnvMap::sample (envmap.rs:235-275) of the resident scene's
        environment at each (u, v) pair: (direction, radiance, pdf)."""
        u = np.ascontiguousarray(u2, np.float32).reshape(-1, 2)
        n = len(u)
        d, r, p = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros(n, np.float32)
        check(self._h, self._lib.luc_eval_env(self._h, ptr(u), n, 0, ptr(d), ptr(r), ptr(p)))
        return d, r, p

    def stats(self) -> RenderStats:
        s = RenderStats()
        check(self._h, self._lib.luc_get_stats(self._h, C.byref(s)))
        return s


def build_uniforms(scene: SceneDef, params: RenderParams) -> L.Uniforms:
    """integrator::build_uniforms (integrator.rs:153-178)."""
    cam = scene.camera
    u = camera_uniforms(cam.eye, cam.look_at, cam.vfov_deg, params.width, params.height, up=cam.up,
                        aperture=cam.aperture, focus_distance=cam.focus_distance)
    u.sample_offset = params.sample_offset
    u.samples_per_launch = params.samples
    u.max_depth = params.max_depth
    u.frame_seed = params.frame_seed & 0xFFFFFFFF
    u.num_primitives = len(scene.primitives) - scene.num_instances
    u.num_instances = scene.num_instances
    u.tlas_root = scene.tlas_root
    u.num_lights = len(scene.lights)
    u.num_triangles = len(scene.triangles)
    u.num_bvh_nodes = 0 if scene.bvh_nodes is None else len(scene.bvh_nodes)
    for k in range(3):
        u.background[k] = float(np.float32(scene.background[k]))
    u.sampling_mode = L.SAMPLING[params.sampling]
    w, h = scene.env_size
    u.env_width, u.env_height = w, h
    u.env_total_weight = float(scene.env_total_weight)
    u.sampler_kind = L.SAMPLER[params.sampler]
    return u


ARCHITECTURES = {"wavefront": LUC_ARCH_WAVEFRONT, "megakernel": LUC_ARCH_MEGAKERNEL}


def render_accum(gpu: Gpu, scene: SceneDef, params: RenderParams, uniforms: L.Uniforms | None = None,
                 guides: bool = True, profile: bool = False, guided: bool = False,
                 reference_shadows: bool = False, architecture: str = "wavefront",
                 measure: bool = False) -> np.ndarray:
    """Render and return the raw GpuAccum array, shape (height, width).
    guided=True samples with the context's learned guide (lucida_b200.guide),
    which must have been initialised, and trains it after every batch.
    architecture: "wavefront" or "megakernel" (same accumulator). measure:
    run the convergence meter afterwards (gpu.stats().convergence)."""
    if architecture not in ARCHITECTURES:
        raise GpuError(-4, f"unknown architecture {architecture!r}")
    gpu.upload(scene)
    u = uniforms if uniforms is not None else build_uniforms(scene, params)
    out = np.zeros(params.width * params.height, L.ACCUM)
    flags = (ARCHITECTURES[architecture] | (0 if guides else LUC_FLAG_NO_GUIDES) | (LUC_FLAG_PROFILE if profile else 0)
             | (LUC_FLAG_GUIDED if guided else 0) | (LUC_FLAG_REFERENCE_SHADOWS if reference_shadows else 0)
             | (LUC_FLAG_MEASURE if measure else 0))
    check(gpu.handle, lib().luc_render(gpu.handle, C.byref(u), params.samples, params.max_depth, flags, ptr(out),
                                       None))
    return out.reshape(params.height, params.width)


def accum_to_film(acc: np.ndarray) -> Film:
    h, w = acc.shape
    s = np.maximum(acc["samples"], 1.0)[..., None]
    return Film(w, h, (acc["radiance"] / s).astype(np.float32))


def render_with(gpu: Gpu, scene: SceneDef, params: RenderParams, arch: str = "wavefront") -> Film:
    """pt_gpu::render_with (crates/gpu/src/lib.rs:69-79): "wavefront" or
    "megakernel"."""
    return accum_to_film(render_accum(gpu, scene, params, architecture=arch))


def render_with_measured(gpu: Gpu, scene: SceneDef, params: RenderParams, arch: str = "wavefront"):
    """pt_gpu::render_with_measured (crates/gpu/src/lib.rs:86-97): the film
    and the convergence meter's figure (-1 when nothing is measurable)."""
    film = accum_to_film(render_accum(gpu, scene, params, architecture=arch, measure=True))
    return film, float(gpu.stats().convergence)


def measure_convergence(gpu: Gpu, scene: SceneDef, params: RenderParams) -> float:
    """pt_gpu::measure_convergence (crates/gpu/src/lib.rs:419-426), which
    renders with the megakernel."""
    return render_with_measured(gpu, scene, params, "megakernel")[1]


def convergence(gpu: Gpu, accum_dev, pixels: int) -> float:
    """The convergence meter over a device accumulator (torch tensor or
    address) of `pixels` GpuAccum (ConvergenceMeter::record + read)."""
    out = C.c_float(0.0)
    addr = accum_dev if isinstance(accum_dev, int) else accum_dev.data_ptr()
    check(gpu.handle, lib().luc_convergence(gpu.handle, C.c_void_p(addr), int(pixels), C.byref(out)))
    return float(out.value)


def render_native_on(gpu: Gpu, scene: SceneDef, params: RenderParams) -> Film:
    """pt_gpu::wavefront::render_native_on (crates/gpu/src/wavefront.rs:134-140)."""
    return render_with(gpu, scene, params, "wavefront")


class Denoiser:
    """pt_gpu::denoise::Denoiser (crates/gpu/src/denoise.rs:103-210)."""

    def __init__(self, gpu: Gpu):
        self.gpu = gpu

    def run(self, accum: np.ndarray, params: DenoiseParams = DenoiseParams()) -> np.ndarray:
        h, w = accum.shape
        a = np.ascontiguousarray(accum.reshape(-1), L.ACCUM)
        out = np.zeros_like(a)
        p = _DP(params.iterations, params.sigma_normal, params.sigma_depth, params.sigma_luminance,
                params.sigma_albedo)
        check(self.gpu.handle, lib().luc_denoise(self.gpu.handle, ptr(a), w, h, C.byref(p), ptr(out)))
        return out.reshape(h, w)


def render_native_denoised(gpu: Gpu, scene: SceneDef, params: RenderParams,
                           dparams: DenoiseParams = DenoiseParams()) -> Film:
    """pt_gpu::render_native_denoised (crates/gpu/src/lib.rs:405-412): the
    accumulator is left untouched; the denoised image is a separate product."""
    acc = render_accum(gpu, scene, params, guides=True)
    return accum_to_film(Denoiser(gpu).run(acc, dparams))


@dataclass
class GpuBuildOutput:
    """crates/gpu/src/lbvh.rs:724-733 plus the relaid-out tree."""
    codes: np.ndarray
    order: np.ndarray
    karras: np.ndarray
    parent: np.ndarray
    node_bounds: np.ndarray
    subtree_size: np.ndarray
    scene_bounds: np.ndarray
    nodes: np.ndarray
    prim_indices: np.ndarray


class LbvhBuilder:
    """pt_gpu::lbvh::LbvhBuilder (crates/gpu/src/lbvh.rs:124-715)."""

    def __init__(self, gpu: Gpu):
        self.gpu = gpu

    def _run(self, n, call):
        o = LbvhOut()
        m = max(n - 1, 0)
        res = GpuBuildOutput(codes=np.zeros(n, np.uint32), order=np.zeros(n, np.uint32),
                             karras=np.zeros(2 * m, np.uint32), parent=np.zeros(max(2 * n - 1, 0), np.uint32),
                             node_bounds=np.zeros((max(2 * n - 1, 0), 6), np.float32),
                             subtree_size=np.zeros(m, np.uint32), scene_bounds=np.zeros(6, np.float32),
                             nodes=np.zeros(max(2 * n - 1, 1), L.BVH_NODE), prim_indices=np.zeros(n, np.uint32))
        for f in ("codes", "order", "karras", "parent", "node_bounds", "subtree_size", "scene_bounds", "nodes",
                  "prim_indices"):
            setattr(o, f, ptr(getattr(res, f)))
        check(self.gpu.handle, call(C.byref(o)))
        res.nodes = res.nodes[:o.num_nodes].copy()
        return res

    def build_parts(self, triangles, positions) -> GpuBuildOutput:
        t = np.ascontiguousarray(triangles, L.TRIANGLE)
        p = np.ascontiguousarray(positions, np.float32).reshape(-1, 4)
        return self._run(len(t), lambda o: lib().luc_lbvh_build(self.gpu.handle, ptr(t), len(t), ptr(p), len(p), o))

    def build(self, triangles, positions):
        """Returns (nodes, prim_indices): Lbvh (crates/core/src/lbvh.rs:318-324)."""
        r = self.build_parts(triangles, positions)
        return r.nodes, r.prim_indices

    def build_boxes(self, boxes) -> GpuBuildOutput:
        b = np.ascontiguousarray(boxes, np.float32).reshape(-1, 6)
        return self._run(len(b), lambda o: lib().luc_lbvh_build_boxes(self.gpu.handle, ptr(b), len(b), o))

    def sort(self, keys, vals):
        k = np.ascontiguousarray(keys, np.uint32)
        v = np.ascontiguousarray(vals, np.uint32)
        ko, vo = np.zeros_like(k), np.zeros_like(v)
        check(self.gpu.handle, lib().luc_sort_u32(self.gpu.handle, ptr(k), ptr(v), len(k), ptr(ko), ptr(vo)))
        return ko, vo
