// ORACLE — test infrastructure only (see oracle_core.hpp). Restates
// crates/core/src/instance.rs (transforms, world bounds, the two-level
// closest hit) and the instanced paths of crates/core/src/scene.rs
// (build_instances :252-345, shade_instanced_triangle :375-402,
// intersect_counting :452-501, occluded :577-606).
#include "oracle_scene.hpp"

namespace oracle {

Vec3 affine_point(const Affine& a, Vec3 p) {
    float r[3];
    for (int i = 0; i < 3; ++i) r[i] = ((a.m[i][0] * p.x + a.m[i][1] * p.y) + a.m[i][2] * p.z) + a.m[i][3];
    return Vec3(r[0], r[1], r[2]);
}
Vec3 affine_vector(const Affine& a, Vec3 v) {
    float r[3];
    for (int i = 0; i < 3; ++i) r[i] = (a.m[i][0] * v.x + a.m[i][1] * v.y) + a.m[i][2] * v.z;
    return Vec3(r[0], r[1], r[2]);
}

Affine affine_inverse(const Affine& a) {
    const float(*m)[4] = a.m;
    float c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    float c01 = m[0][2] * m[2][1] - m[0][1] * m[2][2];
    float c02 = m[0][1] * m[1][2] - m[0][2] * m[1][1];
    float c10 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
    float c11 = m[0][0] * m[2][2] - m[0][2] * m[2][0];
    float c12 = m[0][2] * m[1][0] - m[0][0] * m[1][2];
    float c20 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    float c21 = m[0][1] * m[2][0] - m[0][0] * m[2][1];
    float c22 = m[0][0] * m[1][1] - m[0][1] * m[1][0];
    float det = (m[0][0] * c00 + m[0][1] * c10) + m[0][2] * c20;
    Affine r;
    const float c[3][3] = {{c00, c01, c02}, {c10, c11, c12}, {c20, c21, c22}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = c[i][j] / det;
    for (int i = 0; i < 3; ++i)
        r.m[i][3] = -((r.m[i][0] * m[0][3] + r.m[i][1] * m[1][3]) + r.m[i][2] * m[2][3]);
    return r;
}

Affine instance_world_to_object(const GpuInstance& g) {
    Affine a;
    for (int j = 0; j < 3; ++j) {
        a.m[0][j] = g.inv_row0[j];
        a.m[1][j] = g.inv_row1[j];
        a.m[2][j] = g.inv_row2[j];
    }
    for (int i = 0; i < 3; ++i) a.m[i][3] = g.inv_translation[i];
    return a;
}

GpuInstance pack_instance(const Affine& w, uint32_t blas_root, uint32_t material) {
    GpuInstance g;
    std::memset(&g, 0, sizeof(g));
    for (int j = 0; j < 3; ++j) {
        g.inv_row0[j] = w.m[0][j];
        g.inv_row1[j] = w.m[1][j];
        g.inv_row2[j] = w.m[2][j];
        g.inv_translation[j] = w.m[j][3];
    }
    g.blas_root = blas_root;
    g.kind = PRIM_KIND_INSTANCE;
    g.material = material;
    return g;
}

Vec3 instance_point(const GpuInstance& g, Vec3 p) { return affine_point(instance_world_to_object(g), p); }
Vec3 instance_vector(const GpuInstance& g, Vec3 v) { return affine_vector(instance_world_to_object(g), v); }
Vec3 instance_normal(const GpuInstance& g, Vec3 n) {
    // transpose(W_3x3) * n: component i is (row0[i]*n.x + row1[i]*n.y) + row2[i]*n.z.
    float r[3];
    for (int i = 0; i < 3; ++i) r[i] = (g.inv_row0[i] * n.x + g.inv_row1[i] * n.y) + g.inv_row2[i] * n.z;
    return Vec3(r[0], r[1], r[2]).normalize_or(Vec3(0, 0, 1));
}

Aabb instance_world_bounds(const GpuInstance& g, const Aabb& ob) {
    Affine to_world = affine_inverse(instance_world_to_object(g));
    Aabb out;
    for (int i = 0; i < 8; ++i) {
        Vec3 c((i & 1) == 0 ? ob.min.x : ob.max.x, (i & 2) == 0 ? ob.min.y : ob.max.y,
               (i & 4) == 0 ? ob.min.z : ob.max.z);
        out.grow_point(affine_point(to_world, c));
    }
    out.pad();
    return out;
}

static inline void tri_pos_flat(const GpuTriangle& t, const float* pos, Vec3& a, Vec3& b, Vec3& c) {
    a = Vec3(pos[4 * t.i0], pos[4 * t.i0 + 1], pos[4 * t.i0 + 2]);
    b = Vec3(pos[4 * t.i1], pos[4 * t.i1 + 1], pos[4 * t.i1 + 2]);
    c = Vec3(pos[4 * t.i2], pos[4 * t.i2 + 1], pos[4 * t.i2 + 2]);
}

static const size_t FLAT_STACK = 64;

bool flat_bvh_intersect(const GpuBvhNode* nodes, uint32_t root, const GpuTriangle* tris, const float* pos,
                        const Ray& ray, float tmin, float tmax, TraversalStats& st, TriHit& out) {
    Vec3 inv = safe_inv_dir(ray.dir);
    bool found = false;
    float closest = tmax;
    uint32_t stack[FLAT_STACK];
    size_t sp = 0;
    uint32_t node = root;
    for (;;) {
        const GpuBvhNode& n = nodes[node];
        st.node_visits += 1;
        if (n.count > 0) {
            for (uint32_t k = n.left_first; k < n.left_first + n.count; ++k) {
                Vec3 a, b, c;
                tri_pos_flat(tris[k], pos, a, b, c);
                st.triangle_tests += 1;
                float t, u, v;
                if (intersect_triangle(a, b, c, ray, tmin, closest, t, u, v)) {
                    closest = t;
                    out = TriHit{t, u, v, k};
                    found = true;
                }
            }
        } else {
            uint32_t c0 = n.left_first, c1 = c0 + 1;
            float d0, d1;
            bool h0 = node_aabb(nodes[c0]).hit(ray.origin, inv, tmin, closest, d0);
            bool h1 = node_aabb(nodes[c1]).hit(ray.origin, inv, tmin, closest, d1);
            if (h0 && h1) {
                uint32_t nearc = d0 <= d1 ? c0 : c1, farc = d0 <= d1 ? c1 : c0;
                if (sp < FLAT_STACK) stack[sp++] = farc;
                node = nearc;
                continue;
            } else if (h0) {
                node = c0;
                continue;
            } else if (h1) {
                node = c1;
                continue;
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    return found;
}

bool flat_bvh_occluded(const GpuBvhNode* nodes, uint32_t root, const GpuTriangle* tris, const float* pos,
                       const Ray& ray, float tmin, float tmax) {
    Vec3 inv = safe_inv_dir(ray.dir);
    uint32_t stack[FLAT_STACK];
    size_t sp = 0;
    uint32_t node = root;
    for (;;) {
        const GpuBvhNode& n = nodes[node];
        if (n.count > 0) {
            for (uint32_t k = n.left_first; k < n.left_first + n.count; ++k) {
                Vec3 a, b, c;
                tri_pos_flat(tris[k], pos, a, b, c);
                float t, u, v;
                if (intersect_triangle(a, b, c, ray, tmin, tmax, t, u, v)) return true;
            }
        } else {
            uint32_t c0 = n.left_first, c1 = c0 + 1;
            float d;
            bool h0 = node_aabb(nodes[c0]).hit(ray.origin, inv, tmin, tmax, d);
            bool h1 = node_aabb(nodes[c1]).hit(ray.origin, inv, tmin, tmax, d);
            if (h0) {
                if (h1 && sp < FLAT_STACK) stack[sp++] = c1;
                node = c0;
                continue;
            }
            if (h1) {
                node = c1;
                continue;
            }
        }
        if (sp == 0) return false;
        node = stack[--sp];
    }
}

// instance.rs:342-421. The TLAS walk tests every node's own box (the root
// included), descends left first and stacks the right child (32 entries, a
// push dropped when full); leaves index the instance rows directly.
bool Scene::intersect_instances(const Ray& ray, float tmin, float tmax, TraversalStats& st, TriHit& best,
                                uint32_t& best_instance) const {
    if (instances.empty() || flat_nodes.empty()) return false;
    const uint32_t prim_base = (uint32_t)primitives.size();
    Vec3 inv = safe_inv_dir(ray.dir);
    float closest = tmax;
    bool found = false;
    uint32_t stack[32];
    size_t sp = 0;
    uint32_t node = tlas_root;
    for (;;) {
        const GpuBvhNode& n = flat_nodes[node];
        st.node_visits += 1;
        float entry;
        if (node_aabb(n).hit(ray.origin, inv, tmin, closest, entry)) {
            if (n.count > 0) {
                for (uint32_t ii = n.left_first; ii < n.left_first + n.count; ++ii) {
                    const GpuInstance& g = instances[ii - prim_base];
                    Ray local{instance_point(g, ray.origin), instance_vector(g, ray.dir)};
                    TriHit h;
                    if (flat_bvh_intersect(flat_nodes.data(), g.blas_root, triangles.data(), positions.data(), local,
                                           tmin, closest, st, h)) {
                        closest = h.t;
                        best = h;
                        best_instance = ii - prim_base;
                        found = true;
                    }
                }
            } else {
                uint32_t l = n.left_first;
                if (sp + 1 < 32) stack[sp++] = l + 1;
                node = l;
                continue;
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    return found;
}

// The two-level any-hit: the same TLAS walk, returning at the first blocker.
bool Scene::occluded_instances(const Ray& ray, float tmin, float tmax) const {
    if (instances.empty() || flat_nodes.empty()) return false;
    const uint32_t prim_base = (uint32_t)primitives.size();
    Vec3 inv = safe_inv_dir(ray.dir);
    uint32_t stack[32];
    size_t sp = 0;
    uint32_t node = tlas_root;
    for (;;) {
        const GpuBvhNode& n = flat_nodes[node];
        float entry;
        if (node_aabb(n).hit(ray.origin, inv, tmin, tmax, entry)) {
            if (n.count > 0) {
                for (uint32_t ii = n.left_first; ii < n.left_first + n.count; ++ii) {
                    const GpuInstance& g = instances[ii - prim_base];
                    Ray local{instance_point(g, ray.origin), instance_vector(g, ray.dir)};
                    if (flat_bvh_occluded(flat_nodes.data(), g.blas_root, triangles.data(), positions.data(), local,
                                          tmin, tmax))
                        return true;
                }
            } else {
                uint32_t l = n.left_first;
                if (sp + 1 < 32) stack[sp++] = l + 1;
                node = l;
                continue;
            }
        }
        if (sp == 0) return false;
        node = stack[--sp];
    }
}

// scene.rs:375-402
Hit Scene::shade_instanced_triangle(const TriHit& th, uint32_t instance, const Ray& ray) const {
    const GpuInstance& g = instances[instance];
    Ray local{instance_point(g, ray.origin), instance_vector(g, ray.dir)};
    Hit h = shade_triangle(th, local);
    h.normal = instance_normal(g, h.normal);
    h.geometric_normal = instance_normal(g, h.geometric_normal);
    h.position = ray.origin + th.t * ray.dir;
    h.front_face = h.geometric_normal.dot(ray.dir) < 0.0f;
    float flip = h.front_face ? 1.0f : -1.0f;
    h.normal = h.normal * flip;
    h.geometric_normal = h.geometric_normal * flip;
    if (g.material != 0xFFFFFFFFu) h.material = g.material;
    h.light_area = 0.0f;
    return h;
}

// scene.rs:252-345
void Scene::build_instances(const std::vector<std::pair<uint32_t, uint32_t>>& mesh_ranges,
                            const std::vector<Placement>& placements) {
    struct BlasInfo {
        uint32_t node_offset;
        Aabb bounds;
    };
    std::vector<BlasInfo> blas;
    flat_nodes.clear();
    for (const auto& r : mesh_ranges) {
        uint32_t first = r.first, count = r.second;
        std::vector<GpuTriangle> tris(triangles.begin() + first, triangles.begin() + first + count);
        Bvh b = Bvh::build(tris, positions);
        b.compact_primitives(tris);
        std::copy(tris.begin(), tris.end(), triangles.begin() + first);
        Aabb bounds;
        for (const GpuTriangle& t : tris) bounds.grow(triangle_bounds(t, positions.data()));
        uint32_t node_offset = (uint32_t)flat_nodes.size();
        for (GpuBvhNode n : b.nodes) {
            if (n.count == 0) n.left_first += node_offset;
            else n.left_first += first;
            flat_nodes.push_back(n);
        }
        blas.push_back(BlasInfo{node_offset, bounds});
    }
    std::vector<GpuInstance> inst;
    std::vector<Aabb> world;
    for (const Placement& p : placements) {
        GpuInstance g = pack_instance(affine_inverse(p.object_to_world), blas[p.mesh].node_offset, p.material);
        inst.push_back(g);
        world.push_back(instance_world_bounds(g, blas[p.mesh].bounds));
    }
    Bvh tlas = Bvh::build_over_bounds(world);
    tlas_root = (uint32_t)flat_nodes.size();
    const uint32_t prim_base = (uint32_t)primitives.size();
    for (GpuBvhNode n : tlas.nodes) {
        if (n.count == 0) n.left_first += tlas_root;
        else n.left_first += prim_base;
        flat_nodes.push_back(n);
    }
    instances.clear();
    for (uint32_t i : tlas.prim_indices) instances.push_back(inst[i]);
    bvh = Bvh();  // the single-level tree stays empty, as in the reference
}

void Scene::build_instances_lbvh(const std::vector<std::pair<uint32_t, uint32_t>>& mesh_ranges,
                                 const std::vector<Placement>& placements) {
    struct BlasInfo {
        uint32_t node_offset;
        Aabb bounds;
    };
    std::vector<BlasInfo> blas;
    flat_nodes.clear();
    for (const auto& r : mesh_ranges) {
        uint32_t first = r.first, count = r.second;
        std::vector<GpuTriangle> tris(triangles.begin() + first, triangles.begin() + first + count);
        Bvh b = lbvh_build(tris, positions, 4).tree;
        b.compact_primitives(tris);
        std::copy(tris.begin(), tris.end(), triangles.begin() + first);
        Aabb bounds;
        for (const GpuTriangle& t : tris) bounds.grow(triangle_bounds(t, positions.data()));
        uint32_t node_offset = (uint32_t)flat_nodes.size();
        for (GpuBvhNode n : b.nodes) {
            if (n.count == 0) n.left_first += node_offset;
            else n.left_first += first;
            flat_nodes.push_back(n);
        }
        blas.push_back(BlasInfo{node_offset, bounds});
    }
    std::vector<GpuInstance> inst;
    std::vector<Aabb> world;
    for (const Placement& p : placements) {
        GpuInstance g = pack_instance(affine_inverse(p.object_to_world), blas[p.mesh].node_offset, p.material);
        inst.push_back(g);
        world.push_back(instance_world_bounds(g, blas[p.mesh].bounds));
    }
    Bvh tlas = lbvh_build_over_bounds(world, 4).tree;
    tlas_root = (uint32_t)flat_nodes.size();
    const uint32_t prim_base = (uint32_t)primitives.size();
    for (GpuBvhNode n : tlas.nodes) {
        if (n.count == 0) n.left_first += tlas_root;
        else n.left_first += prim_base;
        flat_nodes.push_back(n);
    }
    instances.clear();
    for (uint32_t i : tlas.prim_indices) instances.push_back(inst[i]);
    bvh = Bvh();
}

}  // namespace oracle
