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
    const float4* tnodes;  // child-pair records, 4 float4 per internal node id
    const float4* soup;    // (p0, e1, e2) per triangle, leaf order
    uint32_t root_first, root_count;  // the root when it is itself a leaf
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

struct TravCount {
    uint32_t nodes = 0, tris = 0;
};

// Traversal layout, derived on the device from the GpuBvhNode tree:
//   * child-pair nodes: for each internal node, both children's boxes and
//     references in one 64-byte record (4 x float4), so descending never
//     re-reads the node it just tested and one record serves both slab tests;
//     a reference is (node id, 0) for an internal child or (first triangle,
//     count) for a leaf;
//   * a triangle soup in leaf order: (p0, p1 - p0, p2 - p0), the exact
//     values Möller–Trumbore computes from the indexed vertices, so the test is
//     bit-identical with three independent loads instead of four dependent ones.
struct TRef {
    uint32_t a, cnt;
};
constexpr uint32_t kNoNode = 0xFFFFFFFFu;

// Slab tests of both children of a child-pair node. The FMA form
// (b * inv - o * inv) differs from the reference's (b - o) * inv by a few
// ULPs; boxes are padded by 1e-6 relative (bvh.rs:100-111), far above that,
// so no hit is ever culled. Only the visiting order of equal-entry boxes can
// change, which matters solely for exactly tied triangle distances.
LUC_D void test_pair(const float4* __restrict__ tn, V3 oi, V3 inv, float tmin, float tmax, bool& h0, bool& h1,
                     float& e0, float& e1, TRef& r0, TRef& r1) {
    float4 a = __ldg(tn), b = __ldg(tn + 1), c = __ldg(tn + 2);
    uint4 r = __ldg(reinterpret_cast<const uint4*>(tn + 3));
    float lx = __fmaf_rn(a.x, inv.x, -oi.x), hx = __fmaf_rn(a.w, inv.x, -oi.x);
    float ly = __fmaf_rn(a.y, inv.y, -oi.y), hy = __fmaf_rn(b.x, inv.y, -oi.y);
    float lz = __fmaf_rn(a.z, inv.z, -oi.z), hz = __fmaf_rn(b.y, inv.z, -oi.z);
    e0 = fmaxf(fmaxf(fminf(lx, hx), fminf(ly, hy)), fmaxf(fminf(lz, hz), tmin));
    float x0 = fminf(fminf(fmaxf(lx, hx), fmaxf(ly, hy)), fminf(fmaxf(lz, hz), tmax));
    lx = __fmaf_rn(b.z, inv.x, -oi.x); hx = __fmaf_rn(c.y, inv.x, -oi.x);
    ly = __fmaf_rn(b.w, inv.y, -oi.y); hy = __fmaf_rn(c.z, inv.y, -oi.y);
    lz = __fmaf_rn(c.x, inv.z, -oi.z); hz = __fmaf_rn(c.w, inv.z, -oi.z);
    e1 = fmaxf(fmaxf(fminf(lx, hx), fminf(ly, hy)), fmaxf(fminf(lz, hz), tmin));
    float x1 = fminf(fminf(fmaxf(lx, hx), fmaxf(ly, hy)), fminf(fmaxf(lz, hz), tmax));
    h0 = e0 <= x0;
    h1 = e1 <= x1;
    r0 = TRef{r.x, r.y};
    r1 = TRef{r.z, r.w};
}

// Möller–Trumbore from (p0, e1, e2) (bvh.rs:930-968, same operation order).
LUC_D bool hit_soup(const float4* __restrict__ soup, uint32_t k, V3 o, V3 d, float tmin, float tmax, float& tout,
                    float& uout, float& vout) {
    float4 q0 = __ldg(soup + 3 * k), q1 = __ldg(soup + 3 * k + 1), q2 = __ldg(soup + 3 * k + 2);
    V3 p0{q0.x, q0.y, q0.z}, e1{q1.x, q1.y, q1.z}, e2{q2.x, q2.y, q2.z};
    V3 pv = cross(d, e2);
    float det = dot(e1, pv);
    if (fabsf(det) < 1.0e-12f) return false;
    float inv_det = 1.0f / det;
    V3 tv = o - p0;
    float u = dot(tv, pv) * inv_det;
    if (!(u >= 0.0f && u <= 1.0f)) return false;
    V3 qv = cross(tv, e1);
    float v = dot(d, qv) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return false;
    float t = dot(e2, qv) * inv_det;
    if (t < tmin || t > tmax) return false;
    tout = t;
    uout = u;
    vout = v;
    return true;
}

// Closest hit (bvh.rs:1045-1130 semantics: the nearest t wins; among exact
// ties the later-tested triangle). While-while traversal (Aila & Laine):
// descend internal nodes near-child-first, postponing the first leaf met so
// lanes of a warp run the node loop and the triangle loop together.
LUC_D bool bvh_closest(const DevScene& s, V3 o, V3 d, float tmin, float& closest, float& bu, float& bv,
                       uint32_t& btri, TravCount& tc) {
    if (s.num_nodes == 0) return false;
    const V3 inv = safe_inv_dir(d);
    const V3 oi = V3{o.x * inv.x, o.y * inv.y, o.z * inv.z};
    bool found = false;
    TRef stack[64];
    int sp = 0;
    TRef cur{0u, 0u}, leaf{0u, 0u};
    if (s.root_count > 0) {
        leaf = TRef{s.root_first, s.root_count};
        cur = TRef{kNoNode, 0u};
    }
    for (;;) {
        while (cur.a != kNoNode && cur.cnt == 0) {
            bool h0, h1;
            float e0, e1;
            TRef r0, r1;
            test_pair(s.tnodes + 4 * (size_t)cur.a, oi, inv, tmin, closest, h0, h1, e0, e1, r0, r1);
            tc.nodes++;
            if (h0 && h1) {
                bool first = e0 <= e1;
                if (sp < 64) stack[sp++] = first ? r1 : r0;
                cur = first ? r0 : r1;
            } else if (h0) {
                cur = r0;
            } else if (h1) {
                cur = r1;
            } else {
                cur = sp > 0 ? stack[--sp] : TRef{kNoNode, 0u};
            }
            if (cur.cnt > 0 && leaf.cnt == 0) {
                leaf = cur;
                cur = sp > 0 ? stack[--sp] : TRef{kNoNode, 0u};
            }
            if (__all_sync(__activemask(), leaf.cnt > 0)) break;
        }
        while (leaf.cnt > 0) {
            tc.tris += leaf.cnt;
            for (uint32_t k = leaf.a; k < leaf.a + leaf.cnt; ++k) {
                float th, uh, vh;
                if (hit_soup(s.soup, k, o, d, tmin, closest, th, uh, vh)) {
                    closest = th;
                    bu = uh;
                    bv = vh;
                    btri = k;
                    found = true;
                }
            }
            leaf.cnt = 0;
            if (cur.a != kNoNode && cur.cnt > 0) {
                leaf = cur;
                cur = sp > 0 ? stack[--sp] : TRef{kNoNode, 0u};
            }
        }
        if (cur.a == kNoNode) break;
    }
    return found;
}

// Any hit within [tmin, tmax] (bvh.rs:1137-1193).
LUC_D bool bvh_any(const DevScene& s, V3 o, V3 d, float tmin, float tmax, TravCount& tc) {
    if (s.num_nodes == 0) return false;
    const V3 inv = safe_inv_dir(d);
    const V3 oi = V3{o.x * inv.x, o.y * inv.y, o.z * inv.z};
    TRef stack[64];
    int sp = 0;
    TRef cur{0u, 0u}, leaf{0u, 0u};
    if (s.root_count > 0) {
        leaf = TRef{s.root_first, s.root_count};
        cur = TRef{kNoNode, 0u};
    }
    for (;;) {
        while (cur.a != kNoNode && cur.cnt == 0) {
            bool h0, h1;
            float e0, e1;
            TRef r0, r1;
            test_pair(s.tnodes + 4 * (size_t)cur.a, oi, inv, tmin, tmax, h0, h1, e0, e1, r0, r1);
            tc.nodes++;
            if (h0 && h1) {
                if (sp < 64) stack[sp++] = r1;
                cur = r0;
            } else if (h0) {
                cur = r0;
            } else if (h1) {
                cur = r1;
            } else {
                cur = sp > 0 ? stack[--sp] : TRef{kNoNode, 0u};
            }
            if (cur.cnt > 0 && leaf.cnt == 0) {
                leaf = cur;
                cur = sp > 0 ? stack[--sp] : TRef{kNoNode, 0u};
            }
            if (__all_sync(__activemask(), leaf.cnt > 0)) break;
        }
        while (leaf.cnt > 0) {
            tc.tris += leaf.cnt;
            for (uint32_t k = leaf.a; k < leaf.a + leaf.cnt; ++k) {
                float th, uh, vh;
                if (hit_soup(s.soup, k, o, d, tmin, tmax, th, uh, vh)) return true;
            }
            leaf.cnt = 0;
            if (cur.a != kNoNode && cur.cnt > 0) {
                leaf = cur;
                cur = sp > 0 ? stack[--sp] : TRef{kNoNode, 0u};
            }
        }
        if (cur.a == kNoNode) return false;
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
