// ORACLE — test infrastructure only (see oracle_core.hpp). Restates
// crates/core/src/{scene,bvh,lbvh,integrator,denoise,mesh,scenes}.rs.
#pragma once
#include "oracle_core.hpp"
#include <string>

namespace oracle {

// ---------------------------------------------------------------- bvh.rs Aabb
struct Aabb {  // bvh.rs:45-157
    Vec3 min = Vec3::splat(INFINITY), max = Vec3::splat(-INFINITY);
    void grow_point(Vec3 p) { min = min.min(p); max = max.max(p); }
    void grow(const Aabb& o) { min = min.min(o.min); max = max.max(o.max); }
    bool is_empty() const { return min.x > max.x; }
    float surface_area() const {
        if (is_empty()) return 0.0f;
        Vec3 d = max - min;
        return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x);
    }
    Vec3 centroid() const { return (min + max) * 0.5f; }
    void pad() {  // bvh.rs:100-111
        if (is_empty()) return;
        const float RELATIVE = 1.0e-6f;
        for (int a = 0; a < 3; ++a) {
            float scale = 1.0f + fmax_(std::fabs(min[a]), std::fabs(max[a]));
            float p = RELATIVE * scale;
            min.at(a) = min[a] - p;
            max.at(a) = max[a] + p;
        }
    }
    // bvh.rs:139-150 — returns entry distance or NaN-free "no hit" via bool.
    bool hit(Vec3 o, Vec3 inv, float tmin, float tmax, float& entry_out) const {
        Vec3 t0 = (min - o) * inv;
        Vec3 t1 = (max - o) * inv;
        Vec3 n = t0.min(t1), f = t0.max(t1);
        float entry = fmax_(n.max_element(), tmin);
        float exit = fmin_(f.min_element(), tmax);
        entry_out = entry;
        return entry <= exit;
    }
};
inline Vec3 safe_inv_dir(Vec3 d) {  // bvh.rs:165-178
    const float BIG = 1.0e16f, SMALL = 1.0f / BIG;
    auto g = [&](float v) { return std::fabs(v) > SMALL ? 1.0f / v : std::copysign(BIG, v); };
    return Vec3(g(d.x), g(d.y), g(d.z));
}
inline Aabb node_aabb(const GpuBvhNode& n) {
    Aabb b;
    b.min = Vec3::from(n.bounds_min);
    b.max = Vec3::from(n.bounds_max);
    return b;
}
Aabb triangle_bounds(const GpuTriangle& t, const float* positions4);

struct TraversalStats {
    uint32_t node_visits = 0, triangle_tests = 0;
};
struct TriHit {
    float t, u, v;
    uint32_t triangle;
};

// bvh.rs:930-968
inline bool intersect_triangle(Vec3 p0, Vec3 p1, Vec3 p2, const Ray& ray, float tmin, float tmax,
                               float& t_out, float& u_out, float& v_out) {
    Vec3 e1 = p1 - p0, e2 = p2 - p0;
    Vec3 pv = ray.dir.cross(e2);
    float det = e1.dot(pv);
    if (std::fabs(det) < 1.0e-12f) return false;
    float inv_det = 1.0f / det;
    Vec3 tv = ray.origin - p0;
    float u = tv.dot(pv) * inv_det;
    if (!(u >= 0.0f && u <= 1.0f)) return false;
    Vec3 qv = tv.cross(e1);
    float v = ray.dir.dot(qv) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return false;
    float t = e2.dot(qv) * inv_det;
    if (t < tmin || t > tmax) return false;
    t_out = t;
    u_out = u;
    v_out = v;
    return true;
}

struct Bvh {
    std::vector<GpuBvhNode> nodes;
    std::vector<uint32_t> prim_indices;
    bool empty() const { return nodes.empty(); }
    static Bvh build(const std::vector<GpuTriangle>& tris, const std::vector<float>& pos4);
    static Bvh build_over_bounds(const std::vector<Aabb>& bounds);
    float sah_cost() const;
    void compact_primitives(std::vector<GpuTriangle>& tris);
    bool intersect(const GpuTriangle* tris, const float* pos4, const Ray& ray, float tmin,
                   float tmax, TraversalStats& st, TriHit& out) const;
    bool occluded(const GpuTriangle* tris, const float* pos4, const Ray& ray, float tmin,
                  float tmax) const;
    std::vector<std::string> validate(size_t triangle_count) const;
};
bool brute_force_intersect(const GpuTriangle* tris, size_t n, const float* pos4, const Ray& ray,
                           float tmin, float tmax, TriHit& out);

// ---------------------------------------------------------------- lbvh.rs
uint32_t expand_bits(uint32_t v);
uint32_t morton3d(Vec3 p);
Vec3 lbvh_normalise(Vec3 p, const Aabb& b);
int32_t longest_common_prefix(const uint32_t* codes, int64_t n, int32_t i, int32_t j);
// Every stage of Lbvh::build_with_leaf_size, exposed for stage-by-stage diffs.
struct LbvhStages {
    std::vector<Aabb> tri_bounds;
    Aabb centroid_bounds;
    std::vector<uint32_t> codes;         // input order
    std::vector<uint32_t> order;         // sorted permutation (stable by (code, index))
    std::vector<uint32_t> sorted_codes;
    std::vector<uint32_t> karras;        // 2 per internal node (left, right), ids in [0, 2n-1)
    std::vector<uint32_t> parent;        // 2n-1, u32::MAX for root
    std::vector<Aabb> node_bounds;       // 2n-1
    std::vector<uint32_t> subtree_size;  // n-1
    Bvh tree;                            // relaid out, collapsed <= max_leaf
};
LbvhStages lbvh_build(const std::vector<GpuTriangle>& tris, const std::vector<float>& pos4,
                      size_t max_leaf);
// Lbvh over arbitrary boxes (TLAS over instance bounds).
LbvhStages lbvh_build_over_bounds(const std::vector<Aabb>& bounds, size_t max_leaf);

// ---------------------------------------------------------------- scene.rs
static const float T_MAX = 1.0e30f;
static const float T_MIN = 1.0e-4f;

struct Hit {
    float t;
    uint32_t steps;
    Vec3 position, normal, geometric_normal;
    bool front_face;
    uint32_t material;
    float light_area;
};

// ---------------------------------------------------------------- instance.rs
// A 3x4 affine transform, row-major: m[i][3] is the translation.
struct Affine {
    float m[3][4];
};
// glam's Mat4::transform_point3 / transform_vector3 sum the columns in order:
// per component ((m[i][0]*p.x + m[i][1]*p.y) + m[i][2]*p.z) (+ m[i][3]).
Vec3 affine_point(const Affine& a, Vec3 p);
Vec3 affine_vector(const Affine& a, Vec3 v);
// The inverse of an affine transform by the adjugate: each entry of the 3x3 is
// its cofactor expression divided by the determinant (IEEE division, no
// reciprocal), the translation is -(inverse 3x3 . t). The device computes the
// same expression; glam's 4x4 inverse (used by the reference) agrees to
// rounding.
Affine affine_inverse(const Affine& a);
Affine instance_world_to_object(const GpuInstance& g);
GpuInstance pack_instance(const Affine& w2o, uint32_t blas_root, uint32_t material);  // gpu_layout.rs:513-529
Vec3 instance_point(const GpuInstance& g, Vec3 p);    // Instance::transform_ray, origin
Vec3 instance_vector(const GpuInstance& g, Vec3 v);   // Instance::transform_ray, direction (not normalised)
Vec3 instance_normal(const GpuInstance& g, Vec3 n);   // Instance::transform_normal (instance.rs:137-141)

bool intersect_sphere(const GpuPrimitive& s, const Ray& r, float tmin, float tmax, float& t);
bool intersect_quad(const GpuPrimitive& q, const Ray& r, float tmin, float tmax, float& t);

struct Scene {
    std::vector<GpuMaterial> materials;
    std::vector<GpuPrimitive> primitives;
    std::vector<float> positions;  // 4 floats per vertex
    std::vector<GpuVertexAttr> vertex_attrs;
    std::vector<GpuTriangle> triangles;
    std::vector<GpuLight> lights;
    Bvh bvh;  // single-level BVH over `triangles` (compacted: prim_indices is identity)
    // Instancing (instance.rs; scene.rs:252-345), in the upload's form: the
    // instance rows in TLAS-leaf order (appended to the primitives on upload),
    // the flattened node array (every BLAS, then the TLAS) and the TLAS root.
    // `primitives` keeps the analytic primitives only.
    std::vector<GpuInstance> instances;
    std::vector<GpuBvhNode> flat_nodes;
    uint32_t tlas_root = 0;
    // Shadow rays in an instanced scene: true = the reference's behaviour
    // (scene.rs:577-606 tests the analytic primitives and then every triangle
    // untransformed, in object space); false = the two-level any-hit.
    bool reference_instance_shadows = false;
    struct Placement {
        Affine object_to_world;
        uint32_t mesh, material;
    };
    EnvMap env;
    Vec3 background;
    Camera camera;

    uint32_t light_strategy_count() const {
        return (uint32_t)lights.size() + (env.is_empty() ? 0u : 1u);
    }
    void finalize();  // build SAH BVH, compact, build lights (scene.rs:227-230)
    void finalize_with_lbvh();
    bool intersect(const Ray& ray, Hit& out) const;
    bool occluded(const Ray& ray, float tmax) const;
    Hit shade_triangle(const TriHit& h, const Ray& ray) const;
    // scene.rs:252-345 with a binned-SAH BLAS per mesh range and a binned-SAH
    // TLAS over the instances' world bounds.
    void build_instances(const std::vector<std::pair<uint32_t, uint32_t>>& mesh_ranges,
                         const std::vector<Placement>& placements);
    // The device-built variant (no reference counterpart): an LBVH per mesh
    // range and an LBVH TLAS over the instances' world bounds, flattened the
    // same way.
    void build_instances_lbvh(const std::vector<std::pair<uint32_t, uint32_t>>& mesh_ranges,
                              const std::vector<Placement>& placements);
    // InstanceSet::intersect (instance.rs:342-421) over the flattened arrays.
    bool intersect_instances(const Ray& ray, float tmin, float tmax, TraversalStats& st, TriHit& tri,
                             uint32_t& instance) const;
    bool occluded_instances(const Ray& ray, float tmin, float tmax) const;
    Hit shade_instanced_triangle(const TriHit& h, uint32_t instance, const Ray& ray) const;  // scene.rs:375-402
};
// World bounds of a BLAS box under an instance: the eight corners through the
// forward transform (the inverse of the stored world-to-object), then padded
// (Instance::world_bounds, instance.rs:98-113).
Aabb instance_world_bounds(const GpuInstance& g, const Aabb& object_bounds);
// Bvh::intersect / occluded (bvh.rs:1045-1193) over a flattened node array
// from an arbitrary root (absolute child and triangle indices).
bool flat_bvh_intersect(const GpuBvhNode* nodes, uint32_t root, const GpuTriangle* tris, const float* pos4,
                        const Ray& ray, float tmin, float tmax, TraversalStats& st, TriHit& out);
bool flat_bvh_occluded(const GpuBvhNode* nodes, uint32_t root, const GpuTriangle* tris, const float* pos4,
                       const Ray& ray, float tmin, float tmax);

// ---------------------------------------------------------------- integrator.rs
struct GuideSample {
    Vec3 albedo, normal;
    float depth = 0.0f, steps = 0.0f;
};
GpuUniforms build_uniforms(const Scene& s, uint32_t width, uint32_t height, uint32_t spp,
                           uint32_t max_depth, uint32_t frame_seed, uint32_t sample_offset,
                           uint32_t sampling, uint32_t sampler);
Vec3 radiance_with_guide(const Scene& scene, Ray ray, Sampler& rng, uint32_t max_depth,
                         uint32_t mode, GuideSample& guide);
// Per-pixel sum of the `samples_per_launch` sample radiances in sample order
// (the quantity both `render_pixel` and RESOLVE accumulate), plus the summed
// guides and the squared-radiance sum. Pixels [row0, row1) of the image.
struct PixelSums {
    Vec3 radiance, radiance_sq, albedo, normal;
    float depth;
};
void render_sums(const Scene& s, const GpuUniforms& u, uint32_t threads, std::vector<PixelSums>& out,
                 uint32_t row0, uint32_t row1, uint32_t band = 32);
Vec3 trace_sample(const Scene& s, const GpuUniforms& u, uint32_t x, uint32_t y, uint32_t k, uint64_t& sig);

// ---------------------------------------------------------------- denoise.rs
struct DenoiseParams {
    uint32_t iterations = 4;
    float sigma_normal = 64.0f, sigma_depth = 0.08f, sigma_luminance = 4.0f, sigma_albedo = 0.1f;
};
void denoise(const std::vector<Vec3>& film, const std::vector<Vec3>& albedo,
             const std::vector<Vec3>& normal, const std::vector<float>& depth, uint32_t w,
             uint32_t h, const DenoiseParams& p, std::vector<Vec3>& out);

// ---------------------------------------------------------------- mesh.rs / scenes.rs
struct MeshBuilder {
    std::vector<Vec3> positions, normals;
    std::vector<Vec2> uvs;
    std::vector<uint32_t> indices;  // 3 per triangle
    uint32_t push_vertex(Vec3 p, Vec3 n, Vec2 uv) {
        positions.push_back(p);
        normals.push_back(n);
        uvs.push_back(uv);
        return (uint32_t)positions.size() - 1;
    }
    void append_to(Scene& s, uint32_t material) const;
};
MeshBuilder mesh_quad(Vec3 origin, Vec3 eu, Vec3 ev);
MeshBuilder icosphere(Vec3 center, float radius, uint32_t levels);
GpuMaterial mat_diffuse(Vec3 c);
GpuMaterial mat_glass(Vec3 tint, float roughness, float ior);
GpuMaterial mat_glossy(Vec3 c, float roughness);
GpuMaterial mat_metal(Vec3 c, float roughness);
GpuMaterial mat_conductor(Vec3 eta, Vec3 k, float roughness);
GpuMaterial mat_emissive(Vec3 e);
GpuPrimitive prim_sphere(Vec3 c, float r, uint32_t m);
GpuPrimitive prim_quad(Vec3 o, Vec3 eu, Vec3 ev, uint32_t m);
bool scene_by_name(const std::string& name, Scene& out);

}  // namespace oracle
