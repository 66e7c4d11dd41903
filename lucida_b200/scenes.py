"""Seeded synthetic scenes with the shapes of the benchmark configurations.

* `cornell_analytic()` — the analytic open-front Cornell box in [-1, 1]^3:
  five Lambertian quads, two spheres, a 0.5 x 0.5 ceiling light (17, 12, 4),
  pinhole camera at (0, 0, 3.5) looking down -z, vfov 40 degrees.
* `displaced_spheres()` — 256 icospheres (20 * 4^level triangles each; level
  4 gives 1,310,720 triangles) radially displaced by 3-octave value noise of
  relative amplitude 0.05, placed uniformly in a 20 x 5 x 20 box over a
  ground quad, with per-mesh materials (40% Lambertian, 40% GGX conductor,
  20% rough dielectric) under a procedural 1024 x 512 sky whose sun (0.5
  degree radius, peak 1e4) is importance-sampled through the 2-D CDF.

"Lambertian" is Lucida's GpuMaterial::diffuse (gpu_layout.rs:77-84): a
diffuse base under a roughness-1, IOR-1.5 GGX coat. The value-noise lattice
hash and the sphere layout are defined here: a 32-bit avalanche hash of the
integer cell and the octave seed, trilinear with smoothstep, octaves at
frequency 2, 4, 8 with weights 1, 1/2, 1/4.
"""
from __future__ import annotations

import numpy as np

from . import layout as L
from .gpu import Camera, SceneDef

F32 = np.float32


# ----------------------------------------------------------------- config 1
def cornell_analytic() -> SceneDef:
    mats = np.array([L.diffuse((0.73, 0.73, 0.73)),      # 0 floor / ceiling / back
                     L.diffuse((0.65, 0.05, 0.05)),      # 1 left (red)
                     L.diffuse((0.12, 0.45, 0.15)),      # 2 right (green)
                     L.emissive((17.0, 12.0, 4.0)),      # 3 light
                     L.diffuse((0.73, 0.73, 0.73))],     # 4 spheres
                    L.MATERIAL)
    prims = np.array([
        L.quad((-1, -1, -1), (0, 0, 2), (2, 0, 0), 0),          # floor y=-1, normal +y
        L.quad((-1, 1, -1), (2, 0, 0), (0, 0, 2), 0),           # ceiling y=+1, normal -y
        L.quad((-1, -1, -1), (2, 0, 0), (0, 2, 0), 0),          # back z=-1, normal +z
        L.quad((-1, -1, -1), (0, 2, 0), (0, 0, 2), 1),          # left x=-1, normal +x
        L.quad((1, -1, -1), (0, 0, 2), (0, 2, 0), 2),           # right x=+1, normal -x
        L.quad((-0.25, 0.99, -0.25), (0.5, 0, 0), (0, 0, 0.5), 3),  # light, normal -y
        L.sphere((-0.45, -0.65, -0.3), 0.35, 4),
        L.sphere((0.45, -0.65, 0.3), 0.35, 4),
    ], L.PRIMITIVE)
    return SceneDef(materials=mats, primitives=prims, lights=L.quad_lights(mats, prims),
                    camera=Camera(eye=(0.0, 0.0, 3.5), look_at=(0.0, 0.0, 0.0), vfov_deg=40.0),
                    background=(0.0, 0.0, 0.0), name="cornell-analytic")


# ----------------------------------------------------------------- meshes
def icosphere_unit(levels: int):
    """Unit geodesic sphere: icosahedron subdivided `levels` times with shared
    midpoints (mesh.rs:171-244 construction). Returns (verts[n,3] f64, faces[m,3])."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(levels):
        cache = {}
        nxt = []

        def mid(a, b):
            k = (a, b) if a < b else (b, a)
            if k in cache:
                return cache[k]
            m = verts[a] + verts[b]
            verts.append(m / np.linalg.norm(m))
            cache[k] = len(verts) - 1
            return cache[k]

        for (a, b, c) in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nxt += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nxt
    return np.array(verts), np.array(faces, np.int64)


def _lattice_hash(ix, iy, iz, seed):
    """Integer lattice hash -> [0, 1): a 32-bit avalanche of the cell
    coordinates and the octave seed."""
    h = (ix.astype(np.uint32) * np.uint32(0x8DA6B343) ^ iy.astype(np.uint32) * np.uint32(0xD8163841)
         ^ iz.astype(np.uint32) * np.uint32(0xCB1AB31F) ^ np.uint32(seed & 0xFFFFFFFF))
    h ^= h >> np.uint32(16)
    h *= np.uint32(0x7FEB352D)
    h ^= h >> np.uint32(15)
    h *= np.uint32(0x846CA68B)
    h ^= h >> np.uint32(16)
    return (h >> np.uint32(8)).astype(np.float64) * (1.0 / 16777216.0)


def value_noise3(p: np.ndarray, seed: int, octaves: int = 3, base_freq: float = 2.0) -> np.ndarray:
    """Fractal value noise in [0, 1]: trilinear interpolation of lattice values
    with a smoothstep fade, octaves at frequency f, 2f, 4f weighted 1, 1/2, 1/4."""
    total = np.zeros(len(p))
    norm = 0.0
    amp, freq = 1.0, base_freq
    for o in range(octaves):
        q = p * freq
        i0 = np.floor(q).astype(np.int64)
        f = q - i0
        w = f * f * (3.0 - 2.0 * f)
        acc = np.zeros(len(p))
        for dx in (0, 1):
            for dy in (0, 1):
                for dz in (0, 1):
                    val = _lattice_hash(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz, seed * 7919 + o * 104729)
                    wx = w[:, 0] if dx else 1.0 - w[:, 0]
                    wy = w[:, 1] if dy else 1.0 - w[:, 1]
                    wz = w[:, 2] if dz else 1.0 - w[:, 2]
                    acc += val * wx * wy * wz
        total += amp * acc
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return total / norm


def _vertex_normals(pos: np.ndarray, faces: np.ndarray) -> np.ndarray:
    fn = np.cross(pos[faces[:, 1]] - pos[faces[:, 0]], pos[faces[:, 2]] - pos[faces[:, 0]])
    vn = np.zeros_like(pos)
    for k in range(3):
        np.add.at(vn, faces[:, k], fn)
    return vn / np.maximum(np.linalg.norm(vn, axis=1, keepdims=True), 1e-30)


# ----------------------------------------------------------------- sky
def procedural_sky(width, height, sun_dir, sun_intensity, sun_radius_deg):
    """envmap::procedural_sky (envmap.rs:343-408) plus EnvMap::new's CDF
    (:114-178), in f32, returning (pixels[h,w,4], cdf[h+1, max(w,h)+1],
    total_weight). Row 0 is the zenith."""
    sun = np.asarray(sun_dir, np.float64)
    sun = (sun / np.linalg.norm(sun)).astype(F32)
    texel = max(np.pi / height, 2 * np.pi / width)
    req = np.radians(sun_radius_deg)
    rad = max(req, texel)
    ratio = (1 - np.cos(req)) / max(1 - np.cos(rad), 1e-20)
    inten = F32(sun_intensity * min(ratio, 1.0))
    cos_r = F32(np.cos(rad))
    v = ((np.arange(height, dtype=F32) + F32(0.5)) / F32(height)).astype(F32)
    u = ((np.arange(width, dtype=F32) + F32(0.5)) / F32(width)).astype(F32)
    theta = (v * F32(np.pi)).astype(F32)[:, None]
    phi = (u * F32(2 * np.pi)).astype(F32)[None, :]
    st, ct = np.sin(theta).astype(F32), np.cos(theta).astype(F32)
    d = np.stack(np.broadcast_arrays(st * np.cos(phi).astype(F32), ct, st * np.sin(phi).astype(F32)), -1)
    d = d.astype(F32)
    up = d[..., 1] >= 0
    t = np.power(np.maximum(d[..., 1], 0), F32(0.45)).astype(F32)[..., None]
    sky = (np.array([0.75, 0.86, 1.0], F32) * t + np.array([0.85, 0.70, 0.55], F32) * (F32(1) - t)).astype(F32)
    c = np.where(up[..., None], sky, F32(0.12)).astype(F32) * F32(0.40)
    dots = (d @ sun).astype(F32)
    c = c + np.where((dots >= cos_r)[..., None], np.array([1.0, 0.92, 0.78], F32) * inten, F32(0))
    px = np.zeros((height, width, 4), F32)
    px[..., :3] = c
    # EnvMap::new: per-row running sums of luminance * sin(theta_row), in f32.
    lum = (((px[..., 0] * F32(0.2126)).astype(F32) + (px[..., 1] * F32(0.7152)).astype(F32)).astype(F32)
           + (px[..., 2] * F32(0.0722)).astype(F32)).astype(F32)
    row_sin = np.sin(((np.arange(height, dtype=F32) + F32(0.5)) / F32(height) * F32(np.pi)).astype(F32)).astype(F32)
    wgt = (np.maximum(lum, F32(0)) * row_sin[:, None]).astype(F32)
    cw = max(width, height) + 1
    cdf = np.zeros((height + 1, cw), F32)
    run = np.cumsum(wgt, axis=1, dtype=F32)
    rows = run[:, -1].copy()
    cdf[:height, 1:width + 1] = run
    nz = rows > 0
    inv = (F32(1) / np.where(nz, rows, F32(1))).astype(F32)
    cdf[:height, 1:width + 1] = np.where(nz[:, None], (cdf[:height, 1:width + 1] * inv[:, None]).astype(F32),
                                         cdf[:height, 1:width + 1])
    cdf[:height, width] = np.where(nz, F32(1), cdf[:height, width])
    marg = np.cumsum(rows, dtype=F32)
    total = F32(marg[-1])
    cdf[height, 1:height + 1] = (marg * (F32(1) / total)).astype(F32) if total > 0 else marg
    if total > 0:
        cdf[height, height] = F32(1)
    return px, cdf, float(total)


# ----------------------------------------------------------------- config 2
def displaced_spheres(count: int = 256, level: int = 4, seed: int = 2024, env_size=(1024, 512),
                      amplitude: float = 0.05, radius_range=(0.45, 0.95), sky=None) -> SceneDef:
    rng = np.random.default_rng(seed)
    unit, faces = icosphere_unit(level)
    nv, nf = len(unit), len(faces)
    mats = [L.diffuse((0.5, 0.5, 0.5))]  # 0: ground
    positions = np.zeros((count * nv, 4), F32)
    attrs = np.zeros(count * nv, L.VERTEX_ATTR)
    tris = np.zeros(count * nf, L.TRIANGLE)
    for s in range(count):
        r = rng.uniform(*radius_range)
        c = np.array([rng.uniform(-10, 10), rng.uniform(r, 5.0), rng.uniform(-10, 10)])
        disp = 1.0 + amplitude * (2.0 * value_noise3(unit, seed * 1000 + s) - 1.0)
        pos = c + unit * (r * disp)[:, None]
        nrm = _vertex_normals(pos, faces)
        kind = rng.uniform()
        if kind < 0.4:
            mats.append(L.diffuse(tuple(rng.uniform(0.1, 0.9, 3))))
        elif kind < 0.8:
            mats.append(L.metal(tuple(rng.uniform(0.5, 1.0, 3)), rng.uniform(0.05, 0.8)))
        else:
            mats.append(L.glass((1.0, 1.0, 1.0), rng.uniform(0.0, 0.3), 1.5))
        base = s * nv
        positions[base:base + nv, :3] = pos
        attrs["normal"][base:base + nv] = nrm
        sl = slice(s * nf, (s + 1) * nf)
        tris["i0"][sl] = faces[:, 0] + base
        tris["i1"][sl] = faces[:, 1] + base
        tris["i2"][sl] = faces[:, 2] + base
        tris["material"][sl] = len(mats) - 1
    mats = np.array(mats, L.MATERIAL)
    prims = np.array([L.quad((-30, 0, -30), (0, 0, 60), (60, 0, 0), 0)], L.PRIMITIVE)
    w, h = env_size
    if sky is not None:  # a precomputed procedural_sky(...) triple, shared between scenes
        px, cdf, total = sky
    else:
        px, cdf, total = procedural_sky(w, h, (-0.4, 0.55, -0.7), 1.0e4, 0.5) if w > 0 else (None, None, 0.0)
    return SceneDef(materials=mats, primitives=prims, lights=L.quad_lights(mats, prims), positions=positions,
                    vertex_attrs=attrs, triangles=tris, bvh_nodes=None,
                    camera=Camera(eye=(0.0, 7.0, 24.0), look_at=(0.0, 1.5, 0.0), vfov_deg=45.0),
                    env_pixels=px, env_cdf=cdf, env_total_weight=total, name=f"displaced-spheres-l{level}")


def guided_room(count: int = 256, level: int = 4, seed: int = 2024, emission: float = 200.0) -> SceneDef:
    """Path-guiding workload: the displaced-spheres geometry (same seed, so the
    same meshes and materials) inside a half-closed room lit only by two
    0.2 x 0.2 emitters of radiance `emission`.

    Room: x in [-12, 12], y in [0, 9], z in [-12, 12]; floor (the ground quad),
    ceiling, back, left and right walls, grey Lambertian 0.7; the front
    (z = +12, towards the camera) is open. No environment map, black
    background. The emitters sit 0.4 below the ceiling at (-5, 8.6, -4) and
    (5, 8.6, 3) and face up, so nothing but the ceiling sees them directly:
    every other surface is lit by light that has bounced at least once, which
    a BSDF-sampled path reaches only by chance and a learned guide can aim at.
    """
    base = displaced_spheres(count=count, level=level, seed=seed, env_size=(0, 0))
    mats = list(base.materials)
    wall = len(mats)
    mats.append(L.diffuse((0.7, 0.7, 0.7)))
    lamp = len(mats)
    mats.append(L.emissive((emission, emission, emission)))
    mats = np.array(mats, L.MATERIAL)
    x0, x1, y1, z0, z1 = -12.0, 12.0, 9.0, -12.0, 12.0
    prims = [base.primitives[0],
             L.quad((x0, y1, z0), (x1 - x0, 0, 0), (0, 0, z1 - z0), wall),   # ceiling
             L.quad((x0, 0, z0), (0, y1, 0), (x1 - x0, 0, 0), wall),         # back
             L.quad((x0, 0, z0), (0, 0, z1 - z0), (0, y1, 0), wall),         # left
             L.quad((x1, 0, z0), (0, y1, 0), (0, 0, z1 - z0), wall)]         # right
    s = 0.2
    for cx, cz in ((-5.0, -4.0), (5.0, 3.0)):
        # edge_u x edge_v = (0, s^2, 0): the emitting side faces +y.
        prims.append(L.quad((cx - s / 2, 8.6, cz - s / 2), (0, 0, s), (s, 0, 0), lamp))
    prims = np.array(prims, L.PRIMITIVE)
    return SceneDef(materials=mats, primitives=prims, lights=L.quad_lights(mats, prims), positions=base.positions,
                    vertex_attrs=base.vertex_attrs, triangles=base.triangles, bvh_nodes=None, camera=base.camera,
                    name=f"guided-room-l{level}")


def _random_rotations(rng, n):
    """Uniform random rotations (normalised Gaussian quaternions) as (n, 3, 3)."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
                     np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
                     np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], 1)


def instanced_field(num_meshes: int = 16, tri_range=(50_000, 500_000), num_instances: int = 4096,
                    extent=(100.0, 10.0, 100.0), seed: int = 5150, level: int = 4, env_size=(1024, 512)) -> SceneDef:
    """Two-level workload: `num_meshes` base meshes whose triangle counts are
    log-uniform in `tri_range`, each a cluster of displaced icospheres built
    with the displaced-spheres recipe (value-noise amplitude 0.05, the same
    material mix: 40% diffuse, 40% GGX metal, 20% rough glass), placed by
    `num_instances` seeded affine transforms: uniform random rotation, uniform
    scale U[0.5, 2], position uniform in an `extent` box (y from 0) above a
    ground quad. The BLASes are built per mesh on the device and the TLAS by
    LBVH (scene.meshes / scene.placements); the sky is the procedural one of
    the displaced-spheres scene.
    """
    rng = np.random.default_rng(seed)
    unit, faces = icosphere_unit(level)
    nv, nf = len(unit), len(faces)
    mats = [L.diffuse((0.5, 0.5, 0.5))]  # 0: ground
    pos_all, nrm_all, tri_all, meshes = [], [], [], []
    vbase = tbase = 0
    lo, hi = np.log(tri_range[0]), np.log(tri_range[1])
    for m in range(num_meshes):
        target = float(np.exp(rng.uniform(lo, hi)))
        k = max(1, int(round(target / nf)))
        kind = rng.uniform()
        if kind < 0.4:
            mats.append(L.diffuse(tuple(rng.uniform(0.1, 0.9, 3))))
        elif kind < 0.8:
            mats.append(L.metal(tuple(rng.uniform(0.5, 1.0, 3)), rng.uniform(0.05, 0.8)))
        else:
            mats.append(L.glass((1.0, 1.0, 1.0), rng.uniform(0.0, 0.3), 1.5))
        first = tbase
        spread = 0.6 * k ** (1.0 / 3.0)
        for s in range(k):
            r = rng.uniform(0.3, 0.6)
            c = rng.uniform(-spread, spread, 3)
            disp = 1.0 + 0.05 * (2.0 * value_noise3(unit, seed * 7919 + m * 1000 + s) - 1.0)
            p = c + unit * (r * disp)[:, None]
            pos_all.append(p)
            nrm_all.append(_vertex_normals(p, faces))
            t = np.zeros(nf, L.TRIANGLE)
            t["i0"], t["i1"], t["i2"] = faces[:, 0] + vbase, faces[:, 1] + vbase, faces[:, 2] + vbase
            t["material"] = len(mats) - 1
            tri_all.append(t)
            vbase += nv
            tbase += nf
        meshes.append((first, tbase - first))
    positions = np.zeros((vbase, 4), F32)
    positions[:, :3] = np.concatenate(pos_all)
    attrs = np.zeros(vbase, L.VERTEX_ATTR)
    attrs["normal"] = np.concatenate(nrm_all)
    rot = _random_rotations(rng, num_instances)
    scale = rng.uniform(0.5, 2.0, num_instances)
    xyz = rng.uniform((-extent[0] / 2, 0.0, -extent[2] / 2), (extent[0] / 2, extent[1], extent[2] / 2),
                      (num_instances, 3))
    o2w = np.zeros((num_instances, 3, 4), F32)
    o2w[:, :, :3] = rot * scale[:, None, None]
    o2w[:, :, 3] = xyz
    mesh = rng.integers(0, num_meshes, num_instances).astype(np.uint32)
    material = np.full(num_instances, 0xFFFFFFFF, np.uint32)
    recolour = rng.uniform(size=num_instances) < 0.1  # every tenth or so: a material override
    material[recolour] = rng.integers(1, len(mats), int(recolour.sum()))
    mats = np.array(mats, L.MATERIAL)
    g = 0.6 * max(extent[0], extent[2])
    prims = np.array([L.quad((-g, 0, -g), (0, 0, 2 * g), (2 * g, 0, 0), 0)], L.PRIMITIVE)
    w, h = env_size
    px, cdf, total = procedural_sky(w, h, (-0.4, 0.55, -0.7), 1.0e4, 0.5) if w > 0 else (None, None, 0.0)
    return SceneDef(materials=mats, primitives=prims, lights=L.quad_lights(mats, prims), positions=positions,
                    vertex_attrs=attrs, triangles=np.concatenate(tri_all), bvh_nodes=None,
                    camera=Camera(eye=(0.0, 0.35 * max(extent) + 5.0, 0.8 * max(extent)), look_at=(0.0, 2.0, 0.0),
                                  vfov_deg=45.0),
                    env_pixels=px, env_cdf=cdf, env_total_weight=total,
                    meshes=np.array(meshes, np.uint32), placements=(o2w, mesh, material),
                    name=f"instanced-field-{num_meshes}x{num_instances}")


BATCH_RESOLUTIONS = ((256, 256), (512, 512), (1024, 1024), (1920, 1080))
BATCH_SPP = (4, 8, 16, 32, 64)


def batch_workload(num_scenes: int = 64, tri_range=(10_000, 2_000_000), seed: int = 4096, level: int = 4,
                   resolutions=BATCH_RESOLUTIONS, spp_choices=BATCH_SPP, depth_range=(4, 12), env_size=(1024, 512)):
    """Uneven batch: `num_scenes` scenes of the displaced-spheres recipe whose
    triangle counts are log-uniform in `tri_range` (whole level-`level`
    icospheres), each with a resolution from `resolutions`, spp from
    `spp_choices` and bounces uniform in `depth_range`, all seeded. Returns
    [(SceneDef, width, height, spp, max_depth)]; the scenes share one sky."""
    rng = np.random.default_rng(seed)
    faces = 20 * 4 ** level
    w, h = env_size
    sky = procedural_sky(w, h, (-0.4, 0.55, -0.7), 1.0e4, 0.5) if w > 0 else (None, None, 0.0)
    out = []
    for i in range(num_scenes):
        tris = float(np.exp(rng.uniform(np.log(tri_range[0]), np.log(tri_range[1]))))
        count = max(1, int(round(tris / faces)))
        res = resolutions[int(rng.integers(len(resolutions)))]
        spp = int(spp_choices[int(rng.integers(len(spp_choices)))])
        depth = int(rng.integers(depth_range[0], depth_range[1] + 1))
        sc = displaced_spheres(count=count, level=level, seed=seed * 1000 + i, env_size=env_size, sky=sky)
        sc.name = f"batch-{i}-{len(sc.triangles)}"
        out.append((sc, res[0], res[1], spp, depth))
    return out
