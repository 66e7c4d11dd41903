// ORACLE — test infrastructure only (see oracle_core.hpp). Restates
// crates/core/src/mesh.rs, the material/primitive constructors of
// crates/core/src/gpu_layout.rs:76-245 and the built-in scenes of
// crates/core/src/scenes.rs. The scenes are pinned against the reference's
// packed scene fixtures by tests/test_oracle_fixtures.py.
#include "oracle_scene.hpp"
#include <map>

namespace oracle {

static GpuMaterial zero_mat() {
    GpuMaterial m;
    std::memset(&m, 0, sizeof(m));
    return m;
}
GpuMaterial mat_diffuse(Vec3 c) {  // gpu_layout.rs:77-84
    GpuMaterial m = zero_mat();
    c.to(m.base_color);
    m.roughness = 1.0f;
    m.ior = 1.5f;
    return m;
}
GpuMaterial mat_glass(Vec3 tint, float roughness, float ior) {  // :96-104
    GpuMaterial m = zero_mat();
    tint.to(m.base_color);
    m.roughness = roughness;
    m.ior = ior;
    m.transmission = 1.0f;
    return m;
}
GpuMaterial mat_glossy(Vec3 c, float roughness) {  // :108-115
    GpuMaterial m = zero_mat();
    c.to(m.base_color);
    m.roughness = roughness;
    m.ior = 1.5f;
    return m;
}
GpuMaterial mat_metal(Vec3 c, float roughness) {  // :119-127
    GpuMaterial m = zero_mat();
    c.to(m.base_color);
    m.metallic = 1.0f;
    m.roughness = roughness;
    m.ior = 1.5f;
    return m;
}
GpuMaterial mat_conductor(Vec3 eta, Vec3 k, float roughness) {  // :131-144
    GpuMaterial m = zero_mat();
    fresnel_conductor(1.0f, eta, k).to(m.base_color);
    m.metallic = 1.0f;
    m.roughness = roughness;
    m.ior = 1.5f;
    eta.to(m.eta);
    k.to(m.k);
    return m;
}
GpuMaterial mat_emissive(Vec3 e) {  // :152-168
    GpuMaterial m = zero_mat();
    e.to(m.emissive);
    m.roughness = 1.0f;
    m.ior = 1.0f;
    return m;
}
GpuPrimitive prim_sphere(Vec3 c, float r, uint32_t mat) {  // :214-222
    GpuPrimitive p;
    std::memset(&p, 0, sizeof(p));
    c.to(p.position);
    p.radius = r;
    p.kind = PRIM_KIND_SPHERE;
    p.material = mat;
    return p;
}
GpuPrimitive prim_quad(Vec3 o, Vec3 eu, Vec3 ev, uint32_t mat) {  // :229-239
    GpuPrimitive p;
    std::memset(&p, 0, sizeof(p));
    o.to(p.position);
    eu.to(p.edge_u);
    p.kind = PRIM_KIND_QUAD;
    ev.to(p.edge_v);
    p.material = mat;
    eu.cross(ev).normalize().to(p.normal);
    return p;
}

// mesh.rs:47-68
void MeshBuilder::append_to(Scene& s, uint32_t material) const {
    uint32_t base = (uint32_t)(s.positions.size() / 4);
    for (size_t i = 0; i < positions.size(); ++i) {
        Vec3 p = positions[i];
        s.positions.insert(s.positions.end(), {p.x, p.y, p.z, 0.0f});
        GpuVertexAttr a;
        std::memset(&a, 0, sizeof(a));
        normals[i].to(a.normal);
        a.uv[0] = uvs[i].x;
        a.uv[1] = uvs[i].y;
        s.vertex_attrs.push_back(a);
    }
    for (size_t t = 0; t + 2 < indices.size(); t += 3)
        s.triangles.push_back(GpuTriangle{base + indices[t], base + indices[t + 1], base + indices[t + 2], material});
}

// mesh.rs:96-106
MeshBuilder mesh_quad(Vec3 origin, Vec3 eu, Vec3 ev) {
    Vec3 n = eu.cross(ev).normalize();
    MeshBuilder m;
    m.push_vertex(origin, n, Vec2(0, 0));
    m.push_vertex(origin + eu, n, Vec2(1, 0));
    m.push_vertex(origin + eu + ev, n, Vec2(1, 1));
    m.push_vertex(origin + ev, n, Vec2(0, 1));
    m.indices = {0, 1, 2, 0, 2, 3};
    return m;
}

// mesh.rs:171-244
MeshBuilder icosphere(Vec3 center, float radius, uint32_t levels) {
    float t = (1.0f + std::sqrt(5.0f)) / 2.0f;
    Vec3 base[12] = {Vec3(-1, t, 0), Vec3(1, t, 0),  Vec3(-1, -t, 0), Vec3(1, -t, 0),
                     Vec3(0, -1, t), Vec3(0, 1, t),  Vec3(0, -1, -t), Vec3(0, 1, -t),
                     Vec3(t, 0, -1), Vec3(t, 0, 1),  Vec3(-t, 0, -1), Vec3(-t, 0, 1)};
    static const uint32_t F[20][3] = {{0, 11, 5}, {0, 5, 1},  {0, 1, 7},   {0, 7, 10}, {0, 10, 11},
                                      {1, 5, 9},  {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                                      {3, 9, 4},  {3, 4, 2},  {3, 2, 6},   {3, 6, 8},  {3, 8, 9},
                                      {4, 9, 5},  {2, 4, 11}, {6, 2, 10},  {8, 6, 7},  {9, 8, 1}};
    std::vector<Vec3> unit;
    for (auto& v : base) unit.push_back(v.normalize());
    std::vector<uint32_t> faces;
    for (auto& f : F) faces.insert(faces.end(), {f[0], f[1], f[2]});
    for (uint32_t lv = 0; lv < levels; ++lv) {
        std::map<std::pair<uint32_t, uint32_t>, uint32_t> cache;
        std::vector<uint32_t> next;
        next.reserve(faces.size() * 4);
        auto midpoint = [&](uint32_t a, uint32_t b) {
            auto key = a < b ? std::make_pair(a, b) : std::make_pair(b, a);
            auto it = cache.find(key);
            if (it != cache.end()) return it->second;
            Vec3 m = ((unit[a] + unit[b]) * 0.5f).normalize();
            unit.push_back(m);
            uint32_t i = (uint32_t)unit.size() - 1;
            cache[key] = i;
            return i;
        };
        for (size_t k = 0; k < faces.size(); k += 3) {
            uint32_t f0 = faces[k], f1 = faces[k + 1], f2 = faces[k + 2];
            uint32_t a = midpoint(f0, f1);
            uint32_t b = midpoint(f1, f2);
            uint32_t c = midpoint(f2, f0);
            next.insert(next.end(), {f0, a, c, f1, b, a, f2, c, b, a, b, c});
        }
        faces = std::move(next);
    }
    MeshBuilder m;
    for (const Vec3& u : unit) {
        Vec2 uv(0.5f + std::atan2(u.z, u.x) / TAU, 0.5f - std::asin(u.y) / PI);
        m.push_vertex(center + u * radius, u, uv);
    }
    m.indices = faces;
    return m;
}

// scenes.rs:56-160
static Scene cornell_box() {
    const float S = 555.0f;
    Scene s;
    s.materials = {mat_diffuse(Vec3(0.725f, 0.710f, 0.680f)), mat_diffuse(Vec3(0.630f, 0.065f, 0.050f)),
                   mat_diffuse(Vec3(0.140f, 0.450f, 0.091f)), mat_emissive(Vec3(18.4f, 15.6f, 8.0f)),
                   mat_diffuse(Vec3::splat(0.800f)),          mat_diffuse(Vec3(0.200f, 0.380f, 0.800f))};
    s.primitives = {
        prim_quad(Vec3(), Vec3(0, 0, S), Vec3(S, 0, 0), 0),
        prim_quad(Vec3(0, S, 0), Vec3(S, 0, 0), Vec3(0, 0, S), 0),
        prim_quad(Vec3(0, 0, S), Vec3(0, S, 0), Vec3(S, 0, 0), 0),
        prim_quad(Vec3(S, 0, 0), Vec3(0, 0, S), Vec3(0, S, 0), 1),
        prim_quad(Vec3(), Vec3(0, S, 0), Vec3(0, 0, S), 2),
        prim_quad(Vec3(213.0f, S - 0.1f, 227.0f), Vec3(130, 0, 0), Vec3(0, 0, 105), 3),
        prim_sphere(Vec3(185, 120, 175), 120.0f, 4),
        prim_sphere(Vec3(370, 90, 350), 90.0f, 5),
    };
    s.camera = Camera::make(Vec3(278, 278, -800), Vec3(278, 278, 0), 37.0f);
    s.background = Vec3();
    s.finalize();
    return s;
}

// scenes.rs:174-210
static Scene cornell_mesh() {
    Scene s = cornell_box();
    std::vector<GpuPrimitive> prims = std::move(s.primitives);
    s.primitives.clear();
    for (const GpuPrimitive& p : prims)
        if (p.kind == PRIM_KIND_QUAD)
            mesh_quad(Vec3::from(p.position), Vec3::from(p.edge_u), Vec3::from(p.edge_v)).append_to(s, p.material);
    uint32_t mats[2] = {4, 5};
    int k = 0;
    for (const GpuPrimitive& p : prims) {
        if (p.kind == PRIM_KIND_QUAD) continue;
        if (k >= 2) break;
        icosphere(Vec3::from(p.position), p.radius, 4).append_to(s, mats[k++]);
    }
    s.finalize();
    return s;
}

// scenes.rs:276-313
static Scene furnace_test() {
    Scene s;
    const int N = 5;
    for (int i = 0; i < N; ++i) {
        float r = (float)i / (float)(N - 1);
        s.materials.push_back(mat_metal(Vec3::splat(1.0f), r));
        float x = ((float)i - (float)(N - 1) * 0.5f) * 2.4f;
        s.primitives.push_back(prim_sphere(Vec3(x, 0, 0), 1.0f, (uint32_t)i));
    }
    s.camera = Camera::make(Vec3(0, 0.8f, -12.0f), Vec3(), 45.0f);
    s.background = Vec3::splat(1.0f);
    s.finalize();
    return s;
}

// scenes.rs:331-385
static Scene metal_sweep() {
    Scene s;
    const int N = 6;
    s.materials.push_back(mat_diffuse(Vec3::splat(0.35f)));
    const Vec3 CU_ETA(0.200438f, 0.924033f, 1.102212f), CU_K(3.9124f, 2.44753f, 2.13764f);
    const Vec3 AU_ETA(0.143245f, 0.375346f, 1.442386f), AU_K(3.98312f, 2.385704f, 1.603575f);
    for (int row = 0; row < 2; ++row) {
        Vec3 eta = row == 0 ? CU_ETA : AU_ETA, k = row == 0 ? CU_K : AU_K;
        for (int i = 0; i < N; ++i) {
            float t = (float)i / (float)(N - 1);
            float roughness = 0.02f + 0.78f * t * t;
            s.materials.push_back(mat_conductor(eta, k, roughness));
            float x = ((float)(N - 1) * 0.5f - (float)i) * 2.3f;
            s.primitives.push_back(prim_sphere(Vec3(x, 1.0f, (float)row * 2.6f), 1.0f,
                                               (uint32_t)s.materials.size() - 1));
        }
    }
    s.primitives.push_back(prim_quad(Vec3(-40, 0, -40), Vec3(0, 0, 80), Vec3(80, 0, 0), 0));
    s.camera = Camera::make(Vec3(0, 3.4f, -13.0f), Vec3(0, 1.0f, 1.3f), 40.0f);
    s.background = Vec3::splat(0.75f);
    s.finalize();
    return s;
}

// scenes.rs:415-511
static Scene mis_scene() {
    Scene s;
    s.materials.push_back(mat_diffuse(Vec3::splat(0.25f)));
    Vec3 eye(0.0f, 3.0f, -8.5f);
    float light_y = 5.4f, light_z = 1.2f, depth = 1.5f;
    float rough[4] = {0.045f, 0.09f, 0.18f, 0.35f};
    for (int i = 0; i < 4; ++i) {
        s.materials.push_back(mat_metal(Vec3::splat(0.85f), rough[i]));
        Vec3 centre(0.0f, 0.62f * (float)i, 0.6f + (float)i * 1.9f);
        Vec3 to_camera = (eye - centre).normalize();
        Vec3 to_light = (Vec3(0.0f, light_y, light_z) - centre).normalize();
        Vec3 n = (to_camera + to_light).normalize();
        Vec3 eu(0.0f, -depth * n.z, depth * n.y);
        Vec3 ev(10.0f, 0.0f, 0.0f);
        Vec3 origin = centre - 0.5f * eu - 0.5f * ev;
        s.primitives.push_back(prim_quad(origin, eu, ev, (uint32_t)s.materials.size() - 1));
    }
    const float POWER = 46.0f;
    float hw[4] = {0.055f, 0.16f, 0.46f, 1.15f};
    for (int j = 0; j < 4; ++j) {
        float x = 3.7f - (float)j * 2.45f;
        float area = 4.0f * hw[j] * hw[j];
        s.materials.push_back(mat_emissive(Vec3::splat(POWER / area)));
        s.primitives.push_back(prim_quad(Vec3(x - hw[j], light_y, light_z - hw[j]), Vec3(2.0f * hw[j], 0, 0),
                                         Vec3(0, 0, 2.0f * hw[j]), (uint32_t)s.materials.size() - 1));
    }
    s.primitives.push_back(prim_quad(Vec3(-16, -3, 10.5f), Vec3(0, 16, 0), Vec3(32, 0, 0), 0));
    s.camera = Camera::make(eye, Vec3(0.0f, 1.35f, 3.4f), 42.0f);
    s.background = Vec3::splat(0.015f);
    s.finalize();
    return s;
}

// scenes.rs:547-644
static Scene glass_box() {
    const float S = 555.0f;
    Scene s;
    s.materials = {mat_diffuse(Vec3(0.725f, 0.710f, 0.680f)),
                   mat_diffuse(Vec3(0.630f, 0.065f, 0.050f)),
                   mat_diffuse(Vec3(0.140f, 0.450f, 0.091f)),
                   mat_emissive(Vec3(30.0f, 26.0f, 18.0f)),
                   mat_glass(Vec3::splat(1.0f), 0.0f, 1.5f),
                   mat_glass(Vec3::splat(1.0f), 0.0f, 2.42f),
                   mat_glass(Vec3::splat(1.0f), 0.25f, 1.5f),
                   mat_glass(Vec3(0.35f, 0.75f, 0.55f), 0.02f, 1.5f)};
    s.primitives = {
        prim_quad(Vec3(), Vec3(0, 0, S), Vec3(S, 0, 0), 0),
        prim_quad(Vec3(0, S, 0), Vec3(S, 0, 0), Vec3(0, 0, S), 0),
        prim_quad(Vec3(0, 0, S), Vec3(0, S, 0), Vec3(S, 0, 0), 0),
        prim_quad(Vec3(S, 0, 0), Vec3(0, 0, S), Vec3(0, S, 0), 1),
        prim_quad(Vec3(), Vec3(0, S, 0), Vec3(0, 0, S), 2),
        prim_quad(Vec3(163.0f, S - 0.1f, 177.0f), Vec3(230, 0, 0), Vec3(0, 0, 205), 3),
        prim_quad(Vec3(60, 40, 430), Vec3(0, 300, 0), Vec3(230, 0, 0), 7),
        prim_sphere(Vec3(150, 110, 160), 110.0f, 4),
        prim_sphere(Vec3(390, 95, 140), 95.0f, 5),
        prim_sphere(Vec3(300, 85, 330), 85.0f, 6),
    };
    s.camera = Camera::make(Vec3(278, 278, -800), Vec3(278, 278, 0), 37.0f);
    s.background = Vec3();
    s.finalize();
    return s;
}

// scenes.rs:660-718
static Scene sunset() {
    Scene s;
    s.materials = {mat_diffuse(Vec3(0.38f, 0.35f, 0.30f)), mat_diffuse(Vec3::splat(0.78f)),
                   mat_metal(Vec3(0.95f, 0.93f, 0.88f), 0.06f), mat_glass(Vec3::splat(1.0f), 0.0f, 1.5f)};
    s.primitives = {prim_quad(Vec3(-40, 0, -40), Vec3(80, 0, 0), Vec3(0, 0, 80), 0),
                    prim_sphere(Vec3(-2.4f, 1, 0), 1.0f, 1), prim_sphere(Vec3(0, 1, 0), 1.0f, 2),
                    prim_sphere(Vec3(2.4f, 1, 0), 1.0f, 3)};
    s.env = procedural_sky(256, 128, Vec3(-0.45f, 0.22f, -0.86f), 6000.0f, 1.0f);
    s.camera = Camera::make(Vec3(0, 1.6f, 7.5f), Vec3(0, 0.9f, 0), 42.0f);
    s.background = Vec3();
    s.finalize();
    return s;
}

// scenes.rs:733-812: forty-nine placements of one icosphere (rotation about
// y and non-uniform scale), one BLAS under a TLAS.
static Scene instance_forest() {
    Scene s;
    s.materials = {mat_diffuse(Vec3(0.34f, 0.32f, 0.29f)), mat_glossy(Vec3(0.70f, 0.35f, 0.25f), 0.35f),
                   mat_metal(Vec3(0.95f, 0.80f, 0.40f), 0.18f)};
    s.primitives = {prim_quad(Vec3(-30, 0, -30), Vec3(60, 0, 0), Vec3(0, 0, 60), 0)};
    icosphere(Vec3(), 0.5f, 2).append_to(s, 1);
    uint32_t tri_count = (uint32_t)s.triangles.size();
    Rng rng(0x1057, 0, 0);
    std::vector<Scene::Placement> placements;
    for (int gx = 0; gx < 7; ++gx) {
        for (int gz = 0; gz < 7; ++gz) {
            float jx = rng.next_f32() - 0.5f;
            float x = ((float)gx * 1.6f - 4.8f) + jx * 0.5f;
            float jz = rng.next_f32() - 0.5f;
            float z = ((float)gz * 1.6f - 4.8f) + jz * 0.5f;
            float sx = 0.7f + rng.next_f32() * 0.7f;
            float sy = 0.5f + rng.next_f32() * 1.1f;
            float sz = 0.7f + rng.next_f32() * 0.7f;
            float spin = rng.next_f32() * TAU;
            float y = 0.5f * sy;
            // translation * rotation_y(spin) * scale: the products are exact
            // (every other term is a zero), leaving these columns.
            float sn = std::sin(spin), cs = std::cos(spin);
            Affine m;
            float rows[3][4] = {{cs * sx, 0.0f, sn * sz, x}, {0.0f, sy, 0.0f, y}, {-sn * sx, 0.0f, cs * sz, z}};
            std::memcpy(m.m, rows, sizeof(rows));
            uint32_t material = (gx + gz) % 3 == 0 ? 2u : 0xFFFFFFFFu;
            placements.push_back(Scene::Placement{m, 0u, material});
        }
    }
    s.env = procedural_sky(256, 128, Vec3(-0.4f, 0.35f, -0.85f), 6000.0f, 1.0f);
    s.camera = Camera::make(Vec3(0, 3.2f, -11.0f), Vec3(0, 0.7f, 0), 40.0f);
    s.background = Vec3();
    s.build_instances({{0u, tri_count}}, placements);
    s.lights = build_lights(s.materials, s.primitives, s.triangles, s.positions);
    return s;
}

bool scene_by_name(const std::string& name, Scene& out) {
    if (name == "instance-forest") {
        out = instance_forest();
        return true;
    }
    if (name == "cornell-box") out = cornell_box();
    else if (name == "cornell-mesh") out = cornell_mesh();
    else if (name == "furnace-test") out = furnace_test();
    else if (name == "metal-sweep") out = metal_sweep();
    else if (name == "mis-scene") out = mis_scene();
    else if (name == "glass-box") out = glass_box();
    else if (name == "sunset") out = sunset();
    else return false;
    return true;
}

}  // namespace oracle
