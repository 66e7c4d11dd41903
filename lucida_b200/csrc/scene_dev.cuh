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
    // Compressed 8-wide tree collapsed from `nodes` (wide.cu); null when the
    // scene traverses the binary tree (instanced scenes, LUC_BINARY_BVH=1).
    const float4* wnodes;  // 5 float4 per wide node, root = node 0
    const float4* wsoup;   // (p0 | leaf-order index in p0.w, e1, e2) per triangle, wide-node order
    uint32_t num_wnodes;
    // Two-level scenes: the wide trees are the BLASes'; blas_wide maps a BLAS's
    // binary root (an instance row's blas_root) to its wide root.
    const uint32_t* blas_wide;
    uint32_t root_first, root_count;  // the root when it is itself a leaf
    // Instancing (instance.rs): GpuInstance rows appended after the analytic
    // primitives, in TLAS-leaf order; the TLAS's first node in `nodes`; the
    // distinct BLAS roots (for the reference's shadow-ray behaviour).
    const GpuInstance* inst;
    // Device-built instancing: the TLAS collapsed into the 8-wide format
    // (root = wide node 0; a leaf slot's entries in twsoup are primitive
    // indices, instance row = index - num_prims), null for the binary walk.
    const float4* twnodes;
    const uint32_t* twsoup;
    // Device-built instancing: world box of each instance row (lo.xyz, hi.xyz
    // in two float4), null otherwise; a ray enters an instance's BLAS only if
    // it crosses the box.
    const float4* inst_box;
    uint32_t num_instances, tlas_root;
    const uint32_t* blas_roots;
    uint32_t num_blas;
    bool reference_shadows;
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
// Radiance and pdf of the texel a direction falls in (one direction-to-texel
// mapping serves both): EnvMap::radiance and EnvMap::pdf, envmap.rs:188-232.
LUC_D V3 env_radiance_pdf(const DevScene& s, V3 d, float& pdf) {
    float u, v;
    env_uv(d, u, v);
    uint32_t i, j;
    env_texel(s, u, v, i, j);
    pdf = env_pdf_texel(s, i, j);
    float4 p = __ldg(s.env_px + (size_t)j * s.env_w + i);
    return V3{p.x, p.y, p.z};
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
// A triangle's bounds padded as Aabb::pad does (bvh.rs:100-111): per axis
// 1e-6 * (1 + max(|lo|, |hi|)) outwards. Every box of the binary tree is a
// union of these.
LUC_D void padded_tri_box(float4 a, float4 b, float4 c, float lo[3], float hi[3]) {
    lo[0] = fminf(fminf(fminf(INFINITY, a.x), b.x), c.x);
    lo[1] = fminf(fminf(fminf(INFINITY, a.y), b.y), c.y);
    lo[2] = fminf(fminf(fminf(INFINITY, a.z), b.z), c.z);
    hi[0] = fmaxf(fmaxf(fmaxf(-INFINITY, a.x), b.x), c.x);
    hi[1] = fmaxf(fmaxf(fmaxf(-INFINITY, a.y), b.y), c.y);
    hi[2] = fmaxf(fmaxf(fmaxf(-INFINITY, a.z), b.z), c.z);
    for (int k = 0; k < 3; ++k) {
        const float scale = 1.0f + fmaxf(fabsf(lo[k]), fabsf(hi[k]));
        const float p = 1.0e-6f * scale;
        lo[k] = lo[k] - p;
        hi[k] = hi[k] + p;
    }
}
LUC_D V3 vtx(const DevScene& s, uint32_t i) {
    float4 p = __ldg(s.positions + i);
    return V3{p.x, p.y, p.z};
}

// Hit record id encoding: triangle index, or analytic primitive | kAnalytic.
constexpr uint32_t kAnalytic = 0x80000000u;
constexpr uint32_t kMiss = 0xFFFFFFFFu;

struct TravCount {
    uint32_t nodes = 0, tris = 0;
    uint32_t blas = 0;  // two-level scenes: instances whose BLAS the walk entered
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
// The slab test of test_pair on one box (lo in b[0].xyz, hi in b[1].xyz).
LUC_D bool test_box(const float4* __restrict__ b, V3 oi, V3 inv, float tmin, float tmax) {
    const float4 lo = __ldg(b), hi = __ldg(b + 1);
    const float lx = __fmaf_rn(lo.x, inv.x, -oi.x), hx = __fmaf_rn(hi.x, inv.x, -oi.x);
    const float ly = __fmaf_rn(lo.y, inv.y, -oi.y), hy = __fmaf_rn(hi.y, inv.y, -oi.y);
    const float lz = __fmaf_rn(lo.z, inv.z, -oi.z), hz = __fmaf_rn(hi.z, inv.z, -oi.z);
    const float e = fmaxf(fmaxf(fminf(lx, hx), fminf(ly, hy)), fmaxf(fminf(lz, hz), tmin));
    const float x = fminf(fminf(fmaxf(lx, hx), fmaxf(ly, hy)), fminf(fmaxf(lz, hz), tmax));
    return e <= x;
}
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
// `root` is (node, 0) for an internal root or (first triangle, count) for a
// root that is itself a leaf.
LUC_D bool bvh_closest(const DevScene& s, TRef root, V3 o, V3 d, float tmin, float& closest, float& bu, float& bv,
                       uint32_t& btri, TravCount& tc) {
    const V3 inv = safe_inv_dir(d);
    const V3 oi = V3{o.x * inv.x, o.y * inv.y, o.z * inv.z};
    bool found = false;
    TRef stack[64];
    int sp = 0;
    TRef cur = root, leaf{0u, 0u};
    if (root.cnt > 0) {
        leaf = root;
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
LUC_D bool bvh_any(const DevScene& s, TRef root, V3 o, V3 d, float tmin, float tmax, TravCount& tc) {
    const V3 inv = safe_inv_dir(d);
    const V3 oi = V3{o.x * inv.x, o.y * inv.y, o.z * inv.z};
    TRef stack[64];
    int sp = 0;
    TRef cur = root, leaf{0u, 0u};
    if (root.cnt > 0) {
        leaf = root;
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

// ---------------------------------------------------------------- wide tree
// Node record (80 B, 5 x 16 B), built by wide.cu from the binary tree:
//   [0] origin p (3 x f32), exponent bytes ex | ey << 8 | ez << 16, internal
//       child mask << 24 (bit s: slot s holds an internal child);
//   [1] first internal child (wide node index), first triangle (wide soup
//       index), triangle count mask (nibble s: the low `count` bits set for
//       a leaf slot s of 1-4 triangles), unused;
//   [2] qlo.x of slots 0-7 (8 x u8), qlo.y; [3] qlo.z, qhi.x; [4] qhi.y, qhi.z.
// Child box of slot s on axis a: [p + qlo * 2^(e-127), p + qhi * 2^(e-127)],
// each plane at least one quantum outside the binary child's (padded) box.
// Internal children are stored contiguously in slot order; so are the leaf
// slots' triangles, so bit b of the count mask is triangle
// first + popc(count mask below b). Slots are assigned by octant: slot s
// holds the child lying towards corner s of the node (bit a set: the +a
// side). A ray whose direction has sign bits oct (bit a set: negative along
// a) meets the children roughly in ascending order of k = s ^ oct, the order
// in which the hit bits are stored and visited.
constexpr int kWideStack = 64;

// Byte j of word as an exact float (2^23 + byte, minus 2^23): one PRMT and
// one FADD per plane.
LUC_D float wide_q(uint32_t word, uint32_t j) {
    return __uint_as_float(__byte_perm(word, 0x4B000000u, 0x7440u | j)) - 8388608.0f;
}

// Bit s of an 8-bit mask to nibble s (0x1 in each set slot's nibble).
LUC_D uint32_t spread_nibbles(uint32_t x) {
    x = (x | (x << 12)) & 0x000F000Fu;
    x = (x | (x << 6)) & 0x03030303u;
    return (x | (x << 3)) & 0x11111111u;
}
// Bit i of an 8-bit mask to bit i ^ oct (branch-free: oct differs per lane).
LUC_D uint32_t xor_permute8(uint32_t x, uint32_t oct) {
    const uint32_t m1 = 0u - (oct & 1u), m2 = 0u - ((oct >> 1) & 1u), m4 = 0u - ((oct >> 2) & 1u);
    x ^= (x ^ (((x & 0x55u) << 1) | ((x >> 1) & 0x55u))) & m1;
    x ^= (x ^ (((x & 0x33u) << 2) | ((x >> 2) & 0x33u))) & m2;
    x ^= (x ^ (((x & 0x0Fu) << 4) | ((x >> 4) & 0x0Fu))) & m4;
    return x;
}

// Slab tests of the 8 child boxes of wide node `node`. Returns the node group
// (first child, internal mask << 8 | hit bits at positions slot ^ oct) and
// the triangle group (first triangle, mask of hit triangle bits, count mask).
LUC_D void wide_slabs(const float4 a, const uint4 b, const uint4 c, const uint4 d, const uint4 e, V3 o, V3 inv,
                      uint32_t oct, float tmin, float tmax, uint2& ng, uint3& tg);
LUC_D void wide_node(const float4* __restrict__ wn, uint32_t node, V3 o, V3 inv, uint32_t oct, float tmin,
                     float tmax, uint2& ng, uint3& tg) {
    const float4* q = wn + 5 * (size_t)node;
    wide_slabs(__ldg(q), __ldg(reinterpret_cast<const uint4*>(q + 1)), __ldg(reinterpret_cast<const uint4*>(q + 2)),
               __ldg(reinterpret_cast<const uint4*>(q + 3)), __ldg(reinterpret_cast<const uint4*>(q + 4)), o, inv,
               oct, tmin, tmax, ng, tg);
}
// The same node test with the top `kStage` nodes of the tree (the first
// levels: the builder numbers nodes level by level) read from a copy in
// shared memory, `stage`, and the rest from global memory.
template <int kStage>
LUC_D void wide_node_staged(const float4* __restrict__ wn, const float4* stage, uint32_t node, V3 o, V3 inv,
                            uint32_t oct, float tmin, float tmax, uint2& ng, uint3& tg) {
    if (kStage == 0) {
        wide_node(wn, node, o, inv, oct, tmin, tmax, ng, tg);
        return;
    }
    // Only the five loads branch; the slab tests run once for either source.
    float4 a;
    uint4 b, c, d, e;
    if (node < (uint32_t)kStage) {
        const float4* q = stage + 5 * node;
        a = q[0];
        b = *reinterpret_cast<const uint4*>(q + 1);
        c = *reinterpret_cast<const uint4*>(q + 2);
        d = *reinterpret_cast<const uint4*>(q + 3);
        e = *reinterpret_cast<const uint4*>(q + 4);
    } else {
        const float4* q = wn + 5 * (size_t)node;
        a = __ldg(q);
        b = __ldg(reinterpret_cast<const uint4*>(q + 1));
        c = __ldg(reinterpret_cast<const uint4*>(q + 2));
        d = __ldg(reinterpret_cast<const uint4*>(q + 3));
        e = __ldg(reinterpret_cast<const uint4*>(q + 4));
    }
    wide_slabs(a, b, c, d, e, o, inv, oct, tmin, tmax, ng, tg);
}
LUC_D void wide_slabs(const float4 a, const uint4 b, const uint4 c, const uint4 d, const uint4 e, V3 o, V3 inv,
                      uint32_t oct, float tmin, float tmax, uint2& ng, uint3& tg) {
    const uint32_t ew = __float_as_uint(a.w);
    const float sx = __uint_as_float((ew & 0xFFu) << 23) * inv.x;
    const float sy = __uint_as_float(((ew >> 8) & 0xFFu) << 23) * inv.y;
    const float sz = __uint_as_float(((ew >> 16) & 0xFFu) << 23) * inv.z;
    const float ox = (a.x - o.x) * inv.x, oy = (a.y - o.y) * inv.y, oz = (a.z - o.z) * inv.z;
    const uint32_t imask = ew >> 24;
    // Near plane: lo for a positive direction, hi for a negative one.
    const bool nx = inv.x < 0.0f, ny = inv.y < 0.0f, nz = inv.z < 0.0f;
    const uint32_t nx0 = nx ? d.z : c.x, nx1 = nx ? d.w : c.y, fx0 = nx ? c.x : d.z, fx1 = nx ? c.y : d.w;
    const uint32_t ny0 = ny ? e.x : c.z, ny1 = ny ? e.y : c.w, fy0 = ny ? c.z : e.x, fy1 = ny ? c.w : e.y;
    const uint32_t nz0 = nz ? e.z : d.x, nz1 = nz ? e.w : d.y, fz0 = nz ? d.x : e.z, fz1 = nz ? d.y : e.w;
    uint32_t hm = 0;  // hit slots, slot order
#pragma unroll
    for (uint32_t s = 0; s < 8; ++s) {
        const uint32_t j = s & 3u;
        const bool hi = s >= 4;
        const float tnx = __fmaf_rn(wide_q(hi ? nx1 : nx0, j), sx, ox), tfx = __fmaf_rn(wide_q(hi ? fx1 : fx0, j), sx, ox);
        const float tny = __fmaf_rn(wide_q(hi ? ny1 : ny0, j), sy, oy), tfy = __fmaf_rn(wide_q(hi ? fy1 : fy0, j), sy, oy);
        const float tnz = __fmaf_rn(wide_q(hi ? nz1 : nz0, j), sz, oz), tfz = __fmaf_rn(wide_q(hi ? fz1 : fz0, j), sz, oz);
        const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, tmin));
        const float tf = fminf(fminf(tfx, tfy), fminf(tfz, tmax));
        hm |= (tn <= tf ? 1u : 0u) << s;
    }
    // Leaf slots: their nibbles of the count mask; empty slots have none.
    ng = make_uint2(b.x, (imask << 8) | xor_permute8(hm & imask, oct));
    tg = make_uint3(b.y, (spread_nibbles(hm & ~imask) * 0xFu) & b.z, b.z);
}

// Closest hit (kAny = false) or any hit (kAny = true) through the wide tree
// whose root is wide node `root`. The triangle test and its operands are
// those of the binary traversal (hit_soup on the same (p0, e1, e2)), so the
// nearest hit is the same; only which of two exactly tied triangles wins can
// differ. The current node group descends into its nearest hit child,
// pushing the rest; a node's triangle group is tested right after the node,
// one triangle per step (after Ylitie, Karras and Laine 2017, compressed
// wide BVHs; their deferral of triangle groups while few lanes have one
// measured slower here).
// A walk's stack of node groups, kCap entries: the first kShared in shared
// memory, in this thread's column of a [kShared][kThreads] array (`col`
// points at row 0, so a warp's accesses at any depths fall in distinct bank
// pairs), the rest in local memory.
template <int kShared, int kThreads, int kCap>
struct GroupStack {
    uint32_t col = 0;  // shared-window address of this thread's row-0 entry
    uint2 deep[kCap > kShared ? kCap - kShared : 1];
    LUC_D void bind(uint2* p) { col = (uint32_t)__cvta_generic_to_shared(p); }
    LUC_D void put(int i, uint2 v) {
        if (kShared > 0 && i < kShared)
            asm("st.shared.v2.u32 [%0], {%1, %2};" ::"r"(col + (uint32_t)i * (uint32_t)(kThreads * 8)), "r"(v.x),
                "r"(v.y)
                : "memory");
        else
            deep[i - kShared] = v;
    }
    LUC_D uint2 get(int i) const {
        if (kShared > 0 && i < kShared) {
            uint2 v;
            asm("ld.shared.v2.u32 {%0, %1}, [%2];"
                : "=r"(v.x), "=r"(v.y)
                : "r"(col + (uint32_t)i * (uint32_t)(kThreads * 8))
                : "memory");
            return v;
        }
        return deep[i - kShared];
    }
};
template <int kCap>
using LocalStack = GroupStack<0, 1, kCap>;

// A resumable walk of one ray through a wide tree: begin() then step()
// until it reports the end. Used whole by wide_trace and one node at a time
// by kernels that refill finished lanes with new rays (k_extend_dyn): both
// visit the same nodes and triangles in the same order.
template <class Stack = LocalStack<kWideStack>>
struct WideWalkT {
    V3 o, d, inv;
    uint32_t oct, btri;
    float tmax, bu, bv;
    bool found;
    uint2 g;
    int sp;
    uint32_t steps;
    Stack stack;

    // This thread's shared-memory stack column (used when Stack keeps entries there).
    LUC_D void bind(uint2* shared_col, uint2*) { stack.bind(shared_col); }
    LUC_D void begin(uint32_t root, V3 o_, V3 d_, float tmax_) {
        o = o_;
        d = d_;
        inv = safe_inv_dir(d_);
        oct = (inv.x < 0.0f ? 1u : 0u) | (inv.y < 0.0f ? 2u : 0u) | (inv.z < 0.0f ? 4u : 0u);
        tmax = tmax_;
        bu = bv = 0.0f;
        btri = 0u;
        found = false;
        // A virtual parent whose only child (slot 0, internal) is the root.
        g = make_uint2(root, (1u << 8) | (1u << oct));
        sp = 0;
        steps = 0;
    }
    // One node visit and its triangles. True when the walk is over: the
    // stack is empty, or (kAny) a hit was found. Each node and triangle is
    // visited at most once per ray in a tree; the step limit only bounds the
    // walk should the arrays ever not form one.
    template <bool kAny, int kStage = 0>
    LUC_D bool step(const DevScene& s, float tmin, TravCount& tc, const float4* stage = nullptr) {
        if (g.y & 0xFFu) {
            const uint32_t k = __ffs(g.y & 0xFFu) - 1u;
            g.y &= ~(1u << k);
            const uint32_t slot = k ^ oct;
            const uint32_t child = g.x + __popc((g.y >> 8) & ((1u << slot) - 1u));
            if ((g.y & 0xFFu) && sp < kWideStack) stack.put(sp++, g);
            uint3 t;
            wide_node_staged<kStage>(s.wnodes, stage, child, o, inv, oct, tmin, tmax, g, t);
            tc.nodes++;
            while (t.y) {
                const uint32_t bit = __ffs(t.y) - 1u;
                t.y &= t.y - 1u;
                const uint32_t kt = t.x + __popc(t.z & ((1u << bit) - 1u));
                tc.tris++;
                float th, uh, vh;
                if (hit_soup(s.wsoup, kt, o, d, tmin, tmax, th, uh, vh)) {
                    found = true;
                    if (kAny) return true;
                    tmax = th;
                    bu = uh;
                    bv = vh;
                    btri = __float_as_uint(__ldg(s.wsoup + 3 * (size_t)kt).w);
                }
            }
        }
        if (!(g.y & 0xFFu)) {
            if (sp == 0) return true;
            g = stack.get(--sp);
        }
        return ++steps >= (1u << 24);
    }
};
using WideWalk = WideWalkT<>;

// Closest hit (kAny = false) or any hit (kAny = true) through the wide tree
// whose root is wide node `root`. The triangle test and its operands are
// those of the binary traversal (hit_soup on the same (p0, e1, e2)), so the
// nearest hit is the same; only which of two exactly tied triangles wins can
// differ. The current node group descends into its nearest hit child,
// pushing the rest; a node's triangle group is tested right after the node,
// one triangle per step (after Ylitie, Karras and Laine 2017, compressed
// wide BVHs; their deferral of triangle groups while few lanes have one
// measured slower here).
template <bool kAny>
LUC_D bool wide_trace(const DevScene& s, uint32_t root, V3 o, V3 d, float tmin, float& tmax, float& bu, float& bv,
                      uint32_t& btri, TravCount& tc) {
    // WideWalk's steps as one loop (kept separate: the compiler schedules
    // the uninterrupted loop better; the megakernel-vs-wavefront bit-exact
    // tests hold the two to the same visiting order).
    const V3 inv = safe_inv_dir(d);
    const uint32_t oct = (inv.x < 0.0f ? 1u : 0u) | (inv.y < 0.0f ? 2u : 0u) | (inv.z < 0.0f ? 4u : 0u);
    uint2 stack[kWideStack];
    int sp = 0;
    uint2 g = make_uint2(root, (1u << 8) | (1u << oct));
    bool found = false;
    for (uint32_t guard = 0; guard < (1u << 24); ++guard) {
        if (g.y & 0xFFu) {
            const uint32_t k = __ffs(g.y & 0xFFu) - 1u;
            g.y &= ~(1u << k);
            const uint32_t slot = k ^ oct;
            const uint32_t child = g.x + __popc((g.y >> 8) & ((1u << slot) - 1u));
            if ((g.y & 0xFFu) && sp < kWideStack) stack[sp++] = g;
            uint3 t;
            wide_node(s.wnodes, child, o, inv, oct, tmin, tmax, g, t);
            tc.nodes++;
            while (t.y) {
                const uint32_t bit = __ffs(t.y) - 1u;
                t.y &= t.y - 1u;
                const uint32_t kt = t.x + __popc(t.z & ((1u << bit) - 1u));
                tc.tris++;
                float th, uh, vh;
                if (hit_soup(s.wsoup, kt, o, d, tmin, tmax, th, uh, vh)) {
                    if (kAny) return true;
                    tmax = th;
                    bu = uh;
                    bv = vh;
                    btri = __float_as_uint(__ldg(s.wsoup + 3 * (size_t)kt).w);
                    found = true;
                }
            }
        }
        if (!(g.y & 0xFFu)) {
            if (sp == 0) break;
            g = stack[--sp];
        }
    }
    return found;
}

// ---------------------------------------------------------------- instancing
// Root reference of the subtree at node i: (i, 0) if internal, else its leaf.
LUC_D TRef node_ref(const DevScene& s, uint32_t i) {
    float4 a = __ldg(s.nodes + 2 * (size_t)i), b = __ldg(s.nodes + 2 * (size_t)i + 1);
    uint32_t count = __float_as_uint(b.w);
    return count ? TRef{__float_as_uint(a.w), count} : TRef{i, 0u};
}
// Instance::transform_ray (instance.rs:119-125) through the stored rows:
// ((r.x*p.x + r.y*p.y) + r.z*p.z) (+ t), the order glam sums the columns in.
LUC_D V3 inst_point(const GpuInstance& g, V3 p) {
    return V3{((g.inv_row0[0] * p.x + g.inv_row0[1] * p.y) + g.inv_row0[2] * p.z) + g.inv_translation[0],
              ((g.inv_row1[0] * p.x + g.inv_row1[1] * p.y) + g.inv_row1[2] * p.z) + g.inv_translation[1],
              ((g.inv_row2[0] * p.x + g.inv_row2[1] * p.y) + g.inv_row2[2] * p.z) + g.inv_translation[2]};
}
LUC_D V3 inst_vector(const GpuInstance& g, V3 v) {
    return V3{(g.inv_row0[0] * v.x + g.inv_row0[1] * v.y) + g.inv_row0[2] * v.z,
              (g.inv_row1[0] * v.x + g.inv_row1[1] * v.y) + g.inv_row1[2] * v.z,
              (g.inv_row2[0] * v.x + g.inv_row2[1] * v.y) + g.inv_row2[2] * v.z};
}
// Instance::transform_normal (instance.rs:137-141): transpose of the stored
// 3x3 times n, normalised (or +z).
LUC_D V3 inst_normal(const GpuInstance& g, V3 n) {
    V3 t{(g.inv_row0[0] * n.x + g.inv_row1[0] * n.y) + g.inv_row2[0] * n.z,
         (g.inv_row0[1] * n.x + g.inv_row1[1] * n.y) + g.inv_row2[1] * n.z,
         (g.inv_row0[2] * n.x + g.inv_row1[2] * n.y) + g.inv_row2[2] * n.z};
    return normalize_or(t, V3{0.0f, 0.0f, 1.0f});
}

// A resumable walk of one ray through a two-level scene whose BLASes have
// wide trees: the TLAS's child pairs and, for each instance whose world box
// the ray enters, that instance's wide BLAS with the ray in object space.
// One step is one TLAS pair test, one instance (its box test and, on a hit,
// the entry into its BLAS) or one BLAS node visit, so kernels can walk a
// warp's rays in lock step and refill finished lanes. The order is
// instances_closest's (kAny = false: nearer pair child first, a leaf's
// instances in order, each BLAS walked whole before the next) or
// instances_any's (kAny: first child first; ends at the first hit), so the
// results are theirs.
template <bool kAny>
struct InstWalk {
    V3 o, d, inv, oi;  // the world ray
    float tmax, bu, bv;
    uint32_t btri, binst;
    bool found, in_blas, tlas_done;
    TRef cur;          // TLAS position: a child pair (cnt == 0) or a leaf's instances
    uint32_t next;     // the leaf's next instance
    uint32_t inst_k;   // the instance whose BLAS is being walked
    int sp;
    uint32_t steps;
    TRef stack[32];
    WideWalk w;

    LUC_D void bind(uint2*, uint2*) {}  // local-memory stacks only
    LUC_D void enter(const DevScene& s, TRef r) {
        cur = r;
        next = r.a;
    }
    LUC_D void begin(const DevScene& s, V3 o_, V3 d_, float tmax_) {
        o = o_;
        d = d_;
        inv = safe_inv_dir(d_);
        oi = V3{o.x * inv.x, o.y * inv.y, o.z * inv.z};
        tmax = tmax_;
        bu = bv = 0.0f;
        btri = binst = 0u;
        found = in_blas = tlas_done = false;
        sp = 0;
        steps = 0;
        enter(s, node_ref(s, s.tlas_root));
    }
    // The TLAS walk moves to the next subtree on its stack (or ends).
    LUC_D void pop(const DevScene& s) {
        if (sp == 0) tlas_done = true;
        else enter(s, stack[--sp]);
    }
    // True when the walk is over (kAny: also at the first hit).
    LUC_D bool step(const DevScene& s, float tmin, TravCount& tc) {
        if (++steps >= (1u << 24)) return true;  // bounds a walk over arrays that do not form trees
        if (in_blas) {
            if (w.step<kAny>(s, tmin, tc)) {
                in_blas = false;
                if (w.found) {
                    found = true;
                    if (kAny) return true;
                    tmax = w.tmax;
                    bu = w.bu;
                    bv = w.bv;
                    btri = w.btri;
                    binst = inst_k;
                }
                return tlas_done;
            }
            return false;
        }
        if (tlas_done) return true;
        if (cur.cnt == 0) {
            bool h0, h1;
            float e0, e1;
            TRef r0, r1;
            test_pair(s.tnodes + 4 * (size_t)cur.a, oi, inv, tmin, tmax, h0, h1, e0, e1, r0, r1);
            tc.nodes++;
            if (h0 && h1) {
                const bool first = kAny || e0 <= e1;
                if (sp < 32) stack[sp++] = first ? r1 : r0;
                enter(s, first ? r0 : r1);
            } else if (h0) {
                enter(s, r0);
            } else if (h1) {
                enter(s, r1);
            } else {
                pop(s);
            }
            return tlas_done;
        }
        // A leaf: one instance per step.
        const uint32_t k = next - s.num_prims;
        ++next;
        if (!s.inst_box || test_box(s.inst_box + 2 * (size_t)k, oi, inv, tmin, tmax)) {
            const GpuInstance g = s.inst[k];
            tc.blas++;
            w.begin(__ldg(s.blas_wide + g.blas_root), inst_point(g, o), inst_vector(g, d), tmax);
            in_blas = true;
            inst_k = k;
        }
        if (next >= cur.a + cur.cnt) pop(s);
        return !in_blas && tlas_done;
    }
};

// The two-level walk when the TLAS has an 8-wide tree too (s.twnodes): a
// TLAS node visit and a BLAS node visit are the same wide-node test, on the
// world ray or the entered instance's object-space ray, so the lanes of a
// warp run them together whichever level each is in. A TLAS node's leaf
// slots (instances) are entered one per step, in slot order, before its
// internal children; each BLAS is walked whole before the next instance.
// Hits update the walk's nearest distance as they are found (kAny: the walk
// ends at the first).
constexpr int kTlasStack = 24;
template <bool kAny, class TStack = LocalStack<kTlasStack>, class BStack = LocalStack<kWideStack>>
struct InstWalkW {
    V3 o, d, inv, oi;   // world ray
    V3 bo, bd, binv;    // the entered instance's object-space ray
    uint32_t oct, boct;
    float tmax, bu, bv;
    uint32_t btri, binst, inst_k;
    bool found, in_blas;
    uint2 gt, gb;       // current node groups of the TLAS and the BLAS walks
    uint3 pend;         // TLAS leaf entries still to enter: (first, entry bits, count mask)
    int spt, spb;
    uint32_t steps;
    TStack stt;
    BStack stb;

    // This thread's shared-memory stack columns, BLAS walk and TLAS walk.
    LUC_D void bind(uint2* blas_col, uint2* tlas_col) {
        stb.bind(blas_col);
        stt.bind(tlas_col);
    }
    LUC_D void begin(const DevScene& s, V3 o_, V3 d_, float tmax_) {
        o = o_;
        d = d_;
        inv = safe_inv_dir(d_);
        oi = V3{o.x * inv.x, o.y * inv.y, o.z * inv.z};
        oct = (inv.x < 0.0f ? 1u : 0u) | (inv.y < 0.0f ? 2u : 0u) | (inv.z < 0.0f ? 4u : 0u);
        tmax = tmax_;
        bu = bv = 0.0f;
        btri = binst = inst_k = 0u;
        found = in_blas = false;
        gt = make_uint2(0u, (1u << 8) | (1u << oct));  // a virtual parent of TLAS wide node 0
        gb = make_uint2(0u, 0u);
        pend = make_uint3(0u, 0u, 0u);
        spt = spb = 0;
        steps = 0;
        boct = 0u;
    }
    // True when the walk is over (kAny: also at the first hit).
    LUC_D bool step(const DevScene& s, float tmin, TravCount& tc) {
        if (++steps >= (1u << 24)) return true;  // bounds a walk over arrays that do not form trees
        if (!in_blas && pend.y) {
            // Enter the next instance of the last TLAS node's leaf slots: its
            // world box, then (ray in object space) its BLAS's root box, which
            // a rotated instance's world box bounds loosely.
            const uint32_t bit = __ffs(pend.y) - 1u;
            pend.y &= pend.y - 1u;
            const uint32_t k = __ldg(s.twsoup + pend.x + __popc(pend.z & ((1u << bit) - 1u))) - s.num_prims;
            if (!s.inst_box || test_box(s.inst_box + 2 * (size_t)k, oi, inv, tmin, tmax)) {
                const GpuInstance g = s.inst[k];
                bo = inst_point(g, o);
                bd = inst_vector(g, d);
                binv = safe_inv_dir(bd);
                const V3 boi{bo.x * binv.x, bo.y * binv.y, bo.z * binv.z};
                if (test_box(s.nodes + 2 * (size_t)g.blas_root, boi, binv, tmin, tmax)) {
                    tc.blas++;
                    boct = (binv.x < 0.0f ? 1u : 0u) | (binv.y < 0.0f ? 2u : 0u) | (binv.z < 0.0f ? 4u : 0u);
                    gb = make_uint2(__ldg(s.blas_wide + g.blas_root), (1u << 8) | (1u << boct));
                    spb = 0;
                    in_blas = true;
                    inst_k = k;
                }
            }
            // Entered: its root is visited in this same step. Otherwise the
            // node's next instance, or its children once none is left.
            if (!in_blas && pend.y) return false;
        }
        uint2 g = in_blas ? gb : gt;
        if (g.y & 0xFFu) {
            const uint32_t oc = in_blas ? boct : oct;
            const uint32_t kk = __ffs(g.y & 0xFFu) - 1u;
            g.y &= ~(1u << kk);
            const uint32_t slot = kk ^ oc;
            const uint32_t child = g.x + __popc((g.y >> 8) & ((1u << slot) - 1u));
            if (g.y & 0xFFu) {
                if (in_blas) {
                    if (spb < kWideStack) stb.put(spb++, g);
                } else if (spt < kTlasStack) {
                    stt.put(spt++, g);
                }
            }
            uint3 t;
            wide_node(in_blas ? s.wnodes : s.twnodes, child, in_blas ? bo : o, in_blas ? binv : inv, oc, tmin, tmax,
                      g, t);
            tc.nodes++;
            if (!in_blas) {
                pend = t;
            } else {
                while (t.y) {
                    const uint32_t tb = __ffs(t.y) - 1u;
                    t.y &= t.y - 1u;
                    const uint32_t kt = t.x + __popc(t.z & ((1u << tb) - 1u));
                    tc.tris++;
                    float th, uh, vh;
                    if (hit_soup(s.wsoup, kt, bo, bd, tmin, tmax, th, uh, vh)) {
                        found = true;
                        if (kAny) return true;
                        tmax = th;
                        bu = uh;
                        bv = vh;
                        btri = __float_as_uint(__ldg(s.wsoup + 3 * (size_t)kt).w);
                        binst = inst_k;
                    }
                }
            }
        }
        if (!(g.y & 0xFFu)) {
            if (in_blas) {
                if (spb > 0) {
                    g = stb.get(--spb);
                } else {
                    in_blas = false;  // this instance is done: back to the TLAS walk
                    return !pend.y && !(gt.y & 0xFFu) && spt == 0;
                }
            } else if (spt > 0) {
                g = stt.get(--spt);
            } else {
                gt = g;
                return !pend.y;
            }
        }
        if (in_blas) gb = g;
        else gt = g;
        return false;
    }
};

// InstanceSet::intersect (instance.rs:342-421): walk the TLAS in world space
// with the child-pair records (near child first; leaves hold instance
// rows), and at each instance walk its BLAS with the ray in object space and
// the closest t so far — the transform keeps t, so one t_max serves both
// levels. The returned triangle index is absolute; `instance` indexes s.inst.
// kWide: the BLASes are walked through their wide trees (s.blas_wide).
template <int kWide>
LUC_D bool instances_closest(const DevScene& s, V3 o, V3 d, float tmin, float& closest, float& bu, float& bv,
                             uint32_t& btri, uint32_t& binst, TravCount& tc) {
    if (kWide && s.twnodes) {  // the 8-wide TLAS: the wavefront's walk, run whole
        InstWalkW<false> w;
        w.begin(s, o, d, closest);
        while (!w.step(s, tmin, tc)) {
        }
        if (w.found) {
            closest = w.tmax;
            bu = w.bu;
            bv = w.bv;
            btri = w.btri;
            binst = w.binst;
        }
        return w.found;
    }
    const V3 inv = safe_inv_dir(d);
    const V3 oi = V3{o.x * inv.x, o.y * inv.y, o.z * inv.z};
    bool found = false;
    TRef stack[32];
    int sp = 0;
    TRef cur = node_ref(s, s.tlas_root);
    for (;;) {
        if (cur.cnt == 0) {
            bool h0, h1;
            float e0, e1;
            TRef r0, r1;
            test_pair(s.tnodes + 4 * (size_t)cur.a, oi, inv, tmin, closest, h0, h1, e0, e1, r0, r1);
            tc.nodes++;
            if (h0 && h1) {
                bool first = e0 <= e1;
                if (sp < 32) stack[sp++] = first ? r1 : r0;
                cur = first ? r0 : r1;
                continue;
            } else if (h0) {
                cur = r0;
                continue;
            } else if (h1) {
                cur = r1;
                continue;
            }
        } else {
            for (uint32_t ii = cur.a; ii < cur.a + cur.cnt; ++ii) {
                const uint32_t k = ii - s.num_prims;
                if (s.inst_box && !test_box(s.inst_box + 2 * (size_t)k, oi, inv, tmin, closest)) continue;
                const GpuInstance g = s.inst[k];
                tc.blas++;
                const bool h = kWide ? wide_trace<false>(s, __ldg(s.blas_wide + g.blas_root), inst_point(g, o),
                                                         inst_vector(g, d), tmin, closest, bu, bv, btri, tc)
                                     : bvh_closest(s, node_ref(s, g.blas_root), inst_point(g, o), inst_vector(g, d),
                                                   tmin, closest, bu, bv, btri, tc);
                if (h) {
                    binst = k;
                    found = true;
                }
            }
        }
        if (sp == 0) break;
        cur = stack[--sp];
    }
    return found;
}

// Any hit through the two levels (the default for shadow rays).
template <int kWide>
LUC_D bool instances_any(const DevScene& s, V3 o, V3 d, float tmin, float tmax, TravCount& tc) {
    if (kWide && s.twnodes) {
        InstWalkW<true> w;
        w.begin(s, o, d, tmax);
        while (!w.step(s, tmin, tc)) {
        }
        return w.found;
    }
    const V3 inv = safe_inv_dir(d);
    const V3 oi = V3{o.x * inv.x, o.y * inv.y, o.z * inv.z};
    TRef stack[32];
    int sp = 0;
    TRef cur = node_ref(s, s.tlas_root);
    for (;;) {
        if (cur.cnt == 0) {
            bool h0, h1;
            float e0, e1;
            TRef r0, r1;
            test_pair(s.tnodes + 4 * (size_t)cur.a, oi, inv, tmin, tmax, h0, h1, e0, e1, r0, r1);
            tc.nodes++;
            if (h0 && h1) {
                if (sp < 32) stack[sp++] = r1;
                cur = r0;
                continue;
            } else if (h0) {
                cur = r0;
                continue;
            } else if (h1) {
                cur = r1;
                continue;
            }
        } else {
            for (uint32_t ii = cur.a; ii < cur.a + cur.cnt; ++ii) {
                if (s.inst_box && !test_box(s.inst_box + 2 * (size_t)(ii - s.num_prims), oi, inv, tmin, tmax))
                    continue;
                const GpuInstance g = s.inst[ii - s.num_prims];
                tc.blas++;
                float tm = tmax, bu, bv;
                uint32_t bt;
                if (kWide ? wide_trace<true>(s, __ldg(s.blas_wide + g.blas_root), inst_point(g, o), inst_vector(g, d),
                                             tmin, tm, bu, bv, bt, tc)
                          : bvh_any(s, node_ref(s, g.blas_root), inst_point(g, o), inst_vector(g, d), tmin, tmax, tc))
                    return true;
            }
        }
        if (sp == 0) return false;
        cur = stack[--sp];
    }
}

// Scene::intersect (scene.rs:452-527): analytic primitives by brute force,
// then triangles bounded by the analytic hit. Returns the id (kMiss on miss).
// In an instanced scene the instances replace the single-level triangle path
// (scene.rs:489-501) and `inst` receives the hit's instance (s.inst index).
// kInst selects the instanced code at compile time, so kernels launched for
// single-level scenes carry none of its registers; likewise kWide for the
// single-level tree: 1 wide tree only (scenes whose triangles have one), 0
// binary tree only, 2 whichever the scene has.
// The analytic-primitive half of Scene::intersect: brute force, nearest t
// below best_t (kTMax to start); id = primitive | kAnalytic on a hit.
LUC_D void analytic_closest(const DevScene& s, V3 o, V3 d, float& best_t, uint32_t& id) {
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
}

// Any hit among the analytic primitives in (kTMin, tmax): the first loop of
// Scene::occluded (scene.rs:577-606).
LUC_D bool analytic_any(const DevScene& s, V3 o, V3 d, float tmax) {
    for (uint32_t i = 0; i < s.num_prims; ++i) {
        const GpuPrimitive& p = s.prims[i];
        float th;
        bool h = p.kind == PRIM_KIND_QUAD
                     ? hit_quad(ld3(p.position), ld3(p.edge_u), ld3(p.edge_v), ld3(p.normal), o, d, kTMin, tmax, th)
                     : hit_sphere(ld3(p.position), p.radius, o, d, kTMin, tmax, th);
        if (h) return true;
    }
    return false;
}

template <bool kInst, int kWide = 2>
LUC_D uint32_t closest_hit(const DevScene& s, V3 o, V3 d, float& t, float& u, float& v, uint32_t& inst,
                           TravCount& tc) {
    float best_t = kTMax;
    uint32_t id = kMiss;
    analytic_closest(s, o, d, best_t, id);
    float bu = 0.0f, bv = 0.0f;
    uint32_t tri;
    inst = 0u;
    if (kInst) {
        const bool h = kWide == 1 || (kWide == 2 && s.blas_wide)
                           ? instances_closest<1>(s, o, d, kTMin, best_t, bu, bv, tri, inst, tc)
                           : instances_closest<0>(s, o, d, kTMin, best_t, bu, bv, tri, inst, tc);
        if (h) id = tri;
    } else if (kWide == 1) {
        if (s.wnodes && wide_trace<false>(s, 0u, o, d, kTMin, best_t, bu, bv, tri, tc)) id = tri;
    } else if (kWide == 2 && s.wnodes) {
        if (wide_trace<false>(s, 0u, o, d, kTMin, best_t, bu, bv, tri, tc)) id = tri;
    } else if (s.num_nodes > 0 && bvh_closest(s, TRef{s.root_count ? s.root_first : 0u, s.root_count}, o, d, kTMin,
                                              best_t, bu, bv, tri, tc)) {
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

// Scene::occluded (scene.rs:577-606). kWide as for closest_hit.
template <bool kInst, int kWide = 2>
LUC_D bool occluded(const DevScene& s, V3 o, V3 d, float tmax, TravCount& tc) {
    for (uint32_t i = 0; i < s.num_prims; ++i) {
        const GpuPrimitive& p = s.prims[i];
        float th;
        bool h = p.kind == PRIM_KIND_QUAD
                     ? hit_quad(ld3(p.position), ld3(p.edge_u), ld3(p.edge_v), ld3(p.normal), o, d, kTMin, tmax, th)
                     : hit_sphere(ld3(p.position), p.radius, o, d, kTMin, tmax, th);
        if (h) return true;
    }
    if (kInst) {
        const bool wide = kWide == 1 || (kWide == 2 && s.blas_wide);
        if (!s.reference_shadows) return wide ? instances_any<1>(s, o, d, kTMin, tmax, tc)
                                              : instances_any<0>(s, o, d, kTMin, tmax, tc);
        // The reference's shadow rays (scene.rs:577-606) test every mesh's
        // triangles untransformed, in object space.
        for (uint32_t b = 0; b < s.num_blas; ++b) {
            float tm = tmax, bu, bv;
            uint32_t bt;
            if (wide ? wide_trace<true>(s, __ldg(s.blas_wide + s.blas_roots[b]), o, d, kTMin, tm, bu, bv, bt, tc)
                     : bvh_any(s, node_ref(s, s.blas_roots[b]), o, d, kTMin, tmax, tc))
                return true;
        }
        return false;
    }
    if (kWide == 1 && !s.wnodes) return false;  // no triangles
    if (kWide != 1 && s.num_nodes == 0) {
        for (uint32_t k = 0; k < s.num_tris; ++k) {
            GpuTriangle tr = s.tris[k];
            float th, uh, vh;
            if (hit_triangle(vtx(s, tr.i0), vtx(s, tr.i1), vtx(s, tr.i2), o, d, kTMin, tmax, th, uh, vh)) return true;
        }
        return false;
    }
    if (kWide == 1 || (kWide == 2 && s.wnodes)) {
        float tm = tmax, bu, bv;
        uint32_t bt;
        return wide_trace<true>(s, 0u, o, d, kTMin, tm, bu, bv, bt, tc);
    }
    return bvh_any(s, TRef{s.root_count ? s.root_first : 0u, s.root_count}, o, d, kTMin, tmax, tc);
}

struct SurfaceHit {
    V3 position, normal, gnormal;
    bool front;
    uint32_t material;
    float light_area;
};
// scene.rs:405-435 (triangles) and :533-573 (analytic).
template <bool kInst>
LUC_D SurfaceHit surface_hit_t(const DevScene& s, uint32_t id, uint32_t inst, float t, float u, float v, V3 o, V3 d) {
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
    // Instanced (scene.rs:375-402): shade in object space with the object-space
    // direction, bring both normals back, then decide front and back in world
    // space; the position is the world ray at t, which the transform keeps.
    const bool instanced = kInst;
    GpuInstance g;
    V3 dl = d;
    if (instanced) {
        g = s.inst[inst];
        dl = inst_vector(g, d);
    }
    GpuTriangle tr = s.tris[id];
    V3 p0 = vtx(s, tr.i0), p1 = vtx(s, tr.i1), p2 = vtx(s, tr.i2);
    float w = 1.0f - u - v;
    V3 n0 = ld3(s.attrs[tr.i0].normal), n1 = ld3(s.attrs[tr.i1].normal), n2 = ld3(s.attrs[tr.i2].normal);
    V3 shading = normalize_or(w * n0 + u * n1 + v * n2, V3{0.0f, 0.0f, 1.0f});
    V3 cr = cross(p1 - p0, p2 - p0);
    V3 geometric = normalize_or(cr, V3{0.0f, 0.0f, 1.0f});
    h.front = dot(geometric, dl) < 0.0f;
    float flip = h.front ? 1.0f : -1.0f;
    h.normal = shading * flip;
    h.gnormal = geometric * flip;
    h.material = tr.material;
    if (instanced) {
        h.normal = inst_normal(g, h.normal);
        h.gnormal = inst_normal(g, h.gnormal);
        h.front = dot(h.gnormal, d) < 0.0f;
        flip = h.front ? 1.0f : -1.0f;
        h.normal = h.normal * flip;
        h.gnormal = h.gnormal * flip;
        if (g.material != 0xFFFFFFFFu) h.material = g.material;
        h.position = o + t * d;
        h.light_area = 0.0f;
        return h;
    }
    h.position = o + t * d;
    h.light_area = 0.5f * length(cr);
    return h;
}
LUC_D SurfaceHit surface_hit(const DevScene& s, uint32_t id, uint32_t inst, float t, float u, float v, V3 o, V3 d) {
    return s.num_instances ? surface_hit_t<true>(s, id, inst, t, u, v, o, d)
                           : surface_hit_t<false>(s, id, inst, t, u, v, o, d);
}

}  // namespace luc
