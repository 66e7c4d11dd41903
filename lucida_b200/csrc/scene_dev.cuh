// Device-side scene: the SceneBlob arrays resident in HBM, the environment
// map with its CDF, and the closest-hit / any-hit queries the wavefront
// stages use (crates/core/src/scene.rs, bvh.rs, envmap.rs semantics).
#pragma once
#include "device_math.cuh"

namespace luc {

struct DevScene {
    const GpuMaterial* materials;
    const GpuPrimitive* prims;  // analytic primitives only
    uint32_t num_prims;
    const GpuLight* lights;
    uint32_t num_lights;
    const float4* positions;
    const GpuVertexAttr* attrs;
    const GpuTriangle* tris;
    uint32_t num_tris;
    const float4* nodes;  // GpuBvhNode as two float4 each
    uint32_t num_nodes;
    const float4* env_px;
    const float* env_cond;   // (w+1) per row
    const float* env_marg;   // h+1
    const float* env_row_sin;  // sin(((j+0.5)/h)*pi) per row, rounded as the reference rounds it
    uint32_t env_w, env_h;
    float env_total;
    const float* energy;  // 32x32 directional albedo table
    V3 background;
    uint32_t light_strategies;  // lights + (env ? 1 : 0)
    bool has_env;
};

// ---------------------------------------------------------------- environment
// envmap.rs:103-111
LUC_D void env_uv(V3 d, float& u, float& v) {
    float theta = dacos(clampf(d.y, -1.0f, 1.0f));
    float a = datan2(d.z, d.x);
    float r = fmodf(a, kTau);
    float phi = r < 0.0f ? r + kTau : r;
    u = phi / kTau;
    v = theta / kPi;
}
LUC_D void env_texel(const DevScene& s, float u, float v, uint32_t& i, uint32_t& j) {
    // (uv * dim) as i64, clamped to [0, dim-1] (envmap.rs:199-203)
    float fi = u * (float)s.env_w, fj = v * (float)s.env_h;
    long long ii = (fi != fi) ? 0 : (long long)fmaxf(fminf(fi, 9.0e18f), -9.0e18f);
    long long jj = (fj != fj) ? 0 : (long long)fmaxf(fminf(fj, 9.0e18f), -9.0e18f);
    ii = ii < 0 ? 0 : (ii > (long long)s.env_w - 1 ? (long long)s.env_w - 1 : ii);
    jj = jj < 0 ? 0 : (jj > (long long)s.env_h - 1 ? (long long)s.env_h - 1 : jj);
    i = (uint32_t)ii;
    j = (uint32_t)jj;
}
LUC_D V3 env_radiance(const DevScene& s, V3 d) {  // envmap.rs:188-196
    float u, v;
    env_uv(d, u, v);
    uint32_t i, j;
    env_texel(s, u, v, i, j);
    float4 p = __ldg(s.env_px + (size_t)j * s.env_w + i);
    return V3{p.x, p.y, p.z};
}
LUC_D float env_pdf_texel(const DevScene& s, uint32_t i, uint32_t j) {
    float st = __ldg(s.env_row_sin + j);
    if (st <= 0.0f) return 0.0f;
    float4 p = __ldg(s.env_px + (size_t)j * s.env_w + i);
    float weight = fmaxf(luminance(V3{p.x, p.y, p.z}), 0.0f) * st;
    float pdf_uv = weight / s.env_total * (float)(s.env_w * s.env_h);
    return pdf_uv / (2.0f * kPi * kPi * st);
}
LUC_D float env_pdf(const DevScene& s, V3 d) {  // envmap.rs:211-232
    float u, v;
    env_uv(d, u, v);
    uint32_t i, j;
    env_texel(s, u, v, i, j);
    return env_pdf_texel(s, i, j);
}
// envmap.rs:290-317: largest index with cdf <= x, then the fraction.
LUC_D void sample_cdf(const float* cdf, uint32_t n, float x, uint32_t& cell, float& frac) {
    uint32_t lo = 0, len = n;
    while (len > 0) {
        uint32_t half = len / 2, mid = lo + half;
        if (__ldg(cdf + mid) <= x) {
            lo = mid + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    cell = min(lo == 0 ? 0u : lo - 1u, n - 1u);
    float c0 = __ldg(cdf + cell), c1 = __ldg(cdf + cell + 1);
    float span = c1 - c0;
    frac = span > 0.0f ? clampf((x - c0) / span, 0.0f, 1.0f) : 0.0f;
}
struct EnvSample {
    V3 dir, rad;
    float pdf;
};
LUC_D EnvSample env_sample(const DevScene& s, float ux, float uy) {  // envmap.rs:235-275
    EnvSample bad{V3{0.0f, 1.0f, 0.0f}, splat(0.0f), 0.0f};
    uint32_t j, i;
    float dv, du;
    sample_cdf(s.env_marg, s.env_h, uy, j, dv);
    sample_cdf(s.env_cond + (size_t)j * (s.env_w + 1), s.env_w, ux, i, du);
    float u = ((float)i + du) / (float)s.env_w;
    float v = ((float)j + dv) / (float)s.env_h;
    float theta = v * kPi, phi = u * kTau;
    float st, ct, sp, cp;
    dsincos(theta, st, ct);
    dsincos(phi, sp, cp);
    V3 dir{st * cp, ct, st * sp};
    float rs = __ldg(s.env_row_sin + j);
    if (rs <= 0.0f) return bad;
    float4 p = __ldg(s.env_px + (size_t)j * s.env_w + i);
    V3 rad{p.x, p.y, p.z};
    float weight = fmaxf(luminance(rad), 0.0f) * rs;
    float pdf_uv = weight / s.env_total * (float)(s.env_w * s.env_h);
    float pdf = pdf_uv / (2.0f * kPi * kPi * rs);
    if (pdf <= 0.0f) return bad;
    return EnvSample{dir, rad, pdf};
}

// ---------------------------------------------------------------- geometry
LUC_D V3 vtx(const DevScene& s, uint32_t i) {
    float4 p = __ldg(s.positions + i);
    return V3{p.x, p.y, p.z};
}

// Hit record id encoding: triangle index, or analytic primitive | kAnalytic.
constexpr uint32_t kAnalytic = 0x80000000u;
constexpr uint32_t kMiss = 0xFFFFFFFFu;

// Closest hit over the BVH (bvh.rs:1045-1130): near-child-first with a
// 64-entry stack, ties resolved toward the later-tested triangle.
struct TravCount {
    uint32_t nodes = 0, tris = 0;
};
LUC_D bool bvh_closest(const DevScene& s, V3 o, V3 d, float tmin, float& closest, float& bu, float& bv,
                       uint32_t& btri, TravCount& tc) {
    if (s.num_nodes == 0) return false;
    V3 inv = safe_inv_dir(d);
    bool found = false;
    uint32_t stack[64];
    int sp = 0;
    uint32_t node = 0;
    for (;;) {
        float4 a = __ldg(s.nodes + 2 * node), b = __ldg(s.nodes + 2 * node + 1);
        uint32_t count = __float_as_uint(b.w), lf = __float_as_uint(a.w);
        tc.nodes++;
        if (count > 0) {
            tc.tris += count;
            for (uint32_t k = lf; k < lf + count; ++k) {
                GpuTriangle t = s.tris[k];
                float th, uh, vh;
                if (hit_triangle(vtx(s, t.i0), vtx(s, t.i1), vtx(s, t.i2), o, d, tmin, closest, th, uh, vh)) {
                    closest = th;
                    bu = uh;
                    bv = vh;
                    btri = k;
                    found = true;
                }
            }
        } else {
            uint32_t c0 = lf;
            float4 a0 = __ldg(s.nodes + 2 * c0), b0 = __ldg(s.nodes + 2 * c0 + 1);
            float4 a1 = __ldg(s.nodes + 2 * c0 + 2), b1 = __ldg(s.nodes + 2 * c0 + 3);
            V3 t0 = (V3{a0.x, a0.y, a0.z} - o) * inv, t1 = (V3{b0.x, b0.y, b0.z} - o) * inv;
            float e0 = fmaxf(max_elem(vmin(t0, t1)), tmin), x0 = fminf(min_elem(vmax(t0, t1)), closest);
            V3 u0 = (V3{a1.x, a1.y, a1.z} - o) * inv, u1 = (V3{b1.x, b1.y, b1.z} - o) * inv;
            float e1 = fmaxf(max_elem(vmin(u0, u1)), tmin), x1 = fminf(min_elem(vmax(u0, u1)), closest);
            bool h0 = e0 <= x0, h1 = e1 <= x1;
            if (h0 && h1) {
                uint32_t nearc = e0 <= e1 ? c0 : c0 + 1, farc = e0 <= e1 ? c0 + 1 : c0;
                if (sp < 64) stack[sp++] = farc;
                node = nearc;
                continue;
            } else if (h0) {
                node = c0;
                continue;
            } else if (h1) {
                node = c0 + 1;
                continue;
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    return found;
}

// Any hit within [tmin, tmax] (bvh.rs:1137-1193).
LUC_D bool bvh_any(const DevScene& s, V3 o, V3 d, float tmin, float tmax, TravCount& tc) {
    if (s.num_nodes == 0) return false;
    V3 inv = safe_inv_dir(d);
    uint32_t stack[64];
    int sp = 0;
    uint32_t node = 0;
    for (;;) {
        float4 a = __ldg(s.nodes + 2 * node), b = __ldg(s.nodes + 2 * node + 1);
        uint32_t count = __float_as_uint(b.w), lf = __float_as_uint(a.w);
        tc.nodes++;
        if (count > 0) {
            tc.tris += count;
            for (uint32_t k = lf; k < lf + count; ++k) {
                GpuTriangle t = s.tris[k];
                float th, uh, vh;
                if (hit_triangle(vtx(s, t.i0), vtx(s, t.i1), vtx(s, t.i2), o, d, tmin, tmax, th, uh, vh)) return true;
            }
        } else {
            uint32_t c0 = lf;
            float4 a0 = __ldg(s.nodes + 2 * c0), b0 = __ldg(s.nodes + 2 * c0 + 1);
            float4 a1 = __ldg(s.nodes + 2 * c0 + 2), b1 = __ldg(s.nodes + 2 * c0 + 3);
            V3 t0 = (V3{a0.x, a0.y, a0.z} - o) * inv, t1 = (V3{b0.x, b0.y, b0.z} - o) * inv;
            float e0 = fmaxf(max_elem(vmin(t0, t1)), tmin), x0 = fminf(min_elem(vmax(t0, t1)), tmax);
            V3 u0 = (V3{a1.x, a1.y, a1.z} - o) * inv, u1 = (V3{b1.x, b1.y, b1.z} - o) * inv;
            float e1 = fmaxf(max_elem(vmin(u0, u1)), tmin), x1 = fminf(min_elem(vmax(u0, u1)), tmax);
            bool h0 = e0 <= x0, h1 = e1 <= x1;
            if (h0) {
                if (h1 && sp < 64) stack[sp++] = c0 + 1;
                node = c0;
                continue;
            }
            if (h1) {
                node = c0 + 1;
                continue;
            }
        }
        if (sp == 0) return false;
        node = stack[--sp];
    }
}

// Scene::intersect (scene.rs:452-527): analytic primitives by brute force,
// then triangles bounded by the analytic hit. Returns the id (kMiss on miss).
LUC_D uint32_t closest_hit(const DevScene& s, V3 o, V3 d, float& t, float& u, float& v, TravCount& tc) {
    float best_t = kTMax;
    uint32_t id = kMiss;
    for (uint32_t i = 0; i < s.num_prims; ++i) {
        const GpuPrimitive& p = s.prims[i];
        float th;
        bool h = p.kind == PRIM_KIND_QUAD
                     ? hit_quad(ld3(p.position), ld3(p.edge_u), ld3(p.edge_v), ld3(p.normal), o, d, kTMin, best_t, th)
                     : hit_sphere(ld3(p.position), p.radius, o, d, kTMin, best_t, th);
        if (h) {
            best_t = th;
            id = i | kAnalytic;
        }
    }
    float bu = 0.0f, bv = 0.0f;
    uint32_t tri;
    if (bvh_closest(s, o, d, kTMin, best_t, bu, bv, tri, tc)) {
        id = tri;
    } else if (s.num_nodes == 0 && s.num_tris > 0) {
        // No BVH: brute force over every triangle (bvh.rs:975-997).
        for (uint32_t k = 0; k < s.num_tris; ++k) {
            GpuTriangle tr = s.tris[k];
            float th, uh, vh;
            if (hit_triangle(vtx(s, tr.i0), vtx(s, tr.i1), vtx(s, tr.i2), o, d, kTMin, best_t, th, uh, vh)) {
                best_t = th;
                bu = uh;
                bv = vh;
                id = k;
            }
        }
    }
    t = best_t;
    u = bu;
    v = bv;
    return id;
}

// Scene::occluded (scene.rs:577-606).
LUC_D bool occluded(const DevScene& s, V3 o, V3 d, float tmax, TravCount& tc) {
    for (uint32_t i = 0; i < s.num_prims; ++i) {
        const GpuPrimitive& p = s.prims[i];
        float th;
        bool h = p.kind == PRIM_KIND_QUAD
                     ? hit_quad(ld3(p.position), ld3(p.edge_u), ld3(p.edge_v), ld3(p.normal), o, d, kTMin, tmax, th)
                     : hit_sphere(ld3(p.position), p.radius, o, d, kTMin, tmax, th);
        if (h) return true;
    }
    if (s.num_nodes == 0) {
        for (uint32_t k = 0; k < s.num_tris; ++k) {
            GpuTriangle tr = s.tris[k];
            float th, uh, vh;
            if (hit_triangle(vtx(s, tr.i0), vtx(s, tr.i1), vtx(s, tr.i2), o, d, kTMin, tmax, th, uh, vh)) return true;
        }
        return false;
    }
    return bvh_any(s, o, d, kTMin, tmax, tc);
}

struct SurfaceHit {
    V3 position, normal, gnormal;
    bool front;
    uint32_t material;
    float light_area;
};
// scene.rs:405-435 (triangles) and :533-573 (analytic).
LUC_D SurfaceHit surface_hit(const DevScene& s, uint32_t id, float t, float u, float v, V3 o, V3 d) {
    SurfaceHit h;
    if (id & kAnalytic) {
        const GpuPrimitive& p = s.prims[id & ~kAnalytic];
        h.position = o + t * d;
        bool quad = p.kind == PRIM_KIND_QUAD;
        h.light_area = quad ? length(cross(ld3(p.edge_u), ld3(p.edge_v))) : 0.0f;
        V3 gn = quad ? ld3(p.normal) : (h.position - ld3(p.position)) / p.radius;
        h.front = dot(gn, d) < 0.0f;
        V3 oriented = h.front ? gn : -gn;
        h.normal = oriented;
        h.gnormal = oriented;
        h.material = p.material;
        return h;
    }
    GpuTriangle tr = s.tris[id];
    V3 p0 = vtx(s, tr.i0), p1 = vtx(s, tr.i1), p2 = vtx(s, tr.i2);
    float w = 1.0f - u - v;
    V3 n0 = ld3(s.attrs[tr.i0].normal), n1 = ld3(s.attrs[tr.i1].normal), n2 = ld3(s.attrs[tr.i2].normal);
    V3 shading = normalize_or(w * n0 + u * n1 + v * n2, V3{0.0f, 0.0f, 1.0f});
    V3 cr = cross(p1 - p0, p2 - p0);
    V3 geometric = normalize_or(cr, V3{0.0f, 0.0f, 1.0f});
    h.front = dot(geometric, d) < 0.0f;
    float flip = h.front ? 1.0f : -1.0f;
    h.position = o + t * d;
    h.normal = shading * flip;
    h.gnormal = geometric * flip;
    h.material = tr.material;
    h.light_area = 0.5f * length(cr);
    return h;
}

}  // namespace luc
