// ORACLE — test infrastructure only (see oracle_core.hpp). Restates
// crates/core/src/scene.rs (intersection) and crates/core/src/integrator.rs.
#include "oracle_scene.hpp"
#include <atomic>
#include <thread>

namespace oracle {

int g_libm_mode = 0;
thread_local uint64_t* g_path_sig = nullptr;
static inline bool sig_bool(uint32_t kind, bool b) {
    sig_event(kind, b ? 1 : 0);
    return b;
}

// scene.rs:76-97
bool intersect_sphere(const GpuPrimitive& s, const Ray& ray, float tmin, float tmax, float& out) {
    Vec3 center = Vec3::from(s.position);
    Vec3 oc = ray.origin - center;
    float a = ray.dir.dot(ray.dir);
    float h = oc.dot(ray.dir);
    float c = oc.dot(oc) - s.radius * s.radius;
    float disc = h * h - a * c;
    if (disc < 0.0f) return false;
    float sd = std::sqrt(disc);
    float t = (-h - sd) / a;
    if (t < tmin || t > tmax) {
        t = (-h + sd) / a;
        if (t < tmin || t > tmax) return false;
    }
    out = t;
    return true;
}

// scene.rs:120-148
bool intersect_quad(const GpuPrimitive& q, const Ray& ray, float tmin, float tmax, float& out) {
    Vec3 origin = Vec3::from(q.position), eu = Vec3::from(q.edge_u), ev = Vec3::from(q.edge_v);
    Vec3 normal = Vec3::from(q.normal);
    float denom = normal.dot(ray.dir);
    if (std::fabs(denom) < 1.0e-8f) return false;
    float t = (normal.dot(origin) - normal.dot(ray.origin)) / denom;
    if (t < tmin || t > tmax) return false;
    Vec3 p = ray.origin + t * ray.dir;
    Vec3 d = p - origin;
    Vec3 n_raw = eu.cross(ev);
    Vec3 w = n_raw / n_raw.dot(n_raw);
    float a = w.dot(d.cross(ev));
    float b = w.dot(eu.cross(d));
    if (!(a >= 0.0f && a <= 1.0f) || !(b >= 0.0f && b <= 1.0f)) return false;
    out = t;
    return true;
}

void Scene::finalize() {  // scene.rs:227-239, 352-365
    bvh = Bvh::build(triangles, positions);
    bvh.compact_primitives(triangles);
    lights = build_lights(materials, primitives, triangles, positions);
}
void Scene::finalize_with_lbvh() {
    bvh = lbvh_build(triangles, positions, 4).tree;
    bvh.compact_primitives(triangles);
    lights = build_lights(materials, primitives, triangles, positions);
}

// scene.rs:405-435
Hit Scene::shade_triangle(const TriHit& h, const Ray& ray) const {
    const GpuTriangle& tri = triangles[h.triangle];
    const float* P = positions.data();
    Vec3 p0(P[4 * tri.i0], P[4 * tri.i0 + 1], P[4 * tri.i0 + 2]);
    Vec3 p1(P[4 * tri.i1], P[4 * tri.i1 + 1], P[4 * tri.i1 + 2]);
    Vec3 p2(P[4 * tri.i2], P[4 * tri.i2 + 1], P[4 * tri.i2 + 2]);
    float w = 1.0f - h.u - h.v;
    auto attr = [&](uint32_t i) { return Vec3::from(vertex_attrs[i].normal); };
    Vec3 shading = (w * attr(tri.i0) + h.u * attr(tri.i1) + h.v * attr(tri.i2)).normalize_or(Vec3(0, 0, 1));
    Vec3 cr = (p1 - p0).cross(p2 - p0);
    Vec3 geometric = cr.normalize_or(Vec3(0, 0, 1));
    bool front = geometric.dot(ray.dir) < 0.0f;
    float flip = front ? 1.0f : -1.0f;
    Hit out;
    out.t = h.t;
    out.steps = 0;
    out.position = ray.origin + h.t * ray.dir;
    out.normal = shading * flip;
    out.geometric_normal = geometric * flip;
    out.front_face = front;
    out.material = tri.material;
    out.light_area = 0.5f * cr.length();
    return out;
}

// scene.rs:452-573 (single-level path)
bool Scene::intersect(const Ray& ray, Hit& out) const {
    TraversalStats st;
    float best_t = T_MAX;
    int64_t best = -1;
    for (size_t i = 0; i < primitives.size(); ++i) {
        const GpuPrimitive& p = primitives[i];
        float t;
        bool h = p.kind == PRIM_KIND_QUAD ? intersect_quad(p, ray, T_MIN, best_t, t)
                                          : intersect_sphere(p, ray, T_MIN, best_t, t);
        if (h) {
            best_t = t;
            best = (int64_t)i;
        }
    }
    TriHit th;
    if (!instances.empty()) {
        // Instances instead of the single-level path (scene.rs:489-501).
        uint32_t inst = 0;
        if (intersect_instances(ray, T_MIN, best_t, st, th, inst)) {
            sig_event(1, ((uint64_t)inst + 1) << 32 | th.triangle);
            out = shade_instanced_triangle(th, inst, ray);
            out.steps = st.node_visits;
            return true;
        }
    } else {
        bool tri_hit = bvh.empty()
                           ? brute_force_intersect(triangles.data(), triangles.size(), positions.data(), ray,
                                                   T_MIN, best_t, th)
                           : bvh.intersect(triangles.data(), positions.data(), ray, T_MIN, best_t, st, th);
        if (tri_hit) {
            sig_event(1, th.triangle);
            out = shade_triangle(th, ray);
            out.steps = st.node_visits;
            return true;
        }
    }
    if (best < 0) return sig_event(1, ~0ull), false;
    sig_event(1, (1ull << 62) | (uint64_t)best);
    const GpuPrimitive& prim = primitives[best];
    Vec3 position = ray.origin + best_t * ray.dir;
    bool quad = prim.kind == PRIM_KIND_QUAD;
    float la = quad ? Vec3::from(prim.edge_u).cross(Vec3::from(prim.edge_v)).length() : 0.0f;
    Vec3 gn = quad ? Vec3::from(prim.normal) : (position - Vec3::from(prim.position)) / prim.radius;
    bool front = gn.dot(ray.dir) < 0.0f;
    Vec3 oriented = front ? gn : -gn;
    out.t = best_t;
    out.steps = st.node_visits;
    out.position = position;
    out.normal = oriented;
    out.geometric_normal = oriented;
    out.front_face = front;
    out.material = prim.material;
    out.light_area = la;
    return true;
}

// scene.rs:577-606
bool Scene::occluded(const Ray& ray, float tmax) const {
    for (const GpuPrimitive& p : primitives) {
        float t;
        bool h = p.kind == PRIM_KIND_QUAD ? intersect_quad(p, ray, T_MIN, tmax, t)
                                          : intersect_sphere(p, ray, T_MIN, tmax, t);
        if (h) return sig_bool(2, true);
    }
    if (!instances.empty() && !reference_instance_shadows) return sig_bool(2, occluded_instances(ray, T_MIN, tmax));
    if (bvh.empty()) {
        TriHit th;
        return sig_bool(2, brute_force_intersect(triangles.data(), triangles.size(), positions.data(), ray,
                                                 T_MIN, tmax, th));
    }
    return sig_bool(2, bvh.occluded(triangles.data(), positions.data(), ray, T_MIN, tmax));
}

// integrator.rs:153-178
GpuUniforms build_uniforms(const Scene& s, uint32_t width, uint32_t height, uint32_t spp,
                           uint32_t max_depth, uint32_t frame_seed, uint32_t sample_offset,
                           uint32_t sampling, uint32_t sampler) {
    GpuUniforms u;
    std::memset(&u, 0, sizeof(u));
    u.width = width;
    u.height = height;
    u.sample_offset = sample_offset;
    u.samples_per_launch = spp;
    u.max_depth = max_depth;
    u.frame_seed = frame_seed;
    u.num_primitives = (uint32_t)s.primitives.size();
    u.num_triangles = (uint32_t)s.triangles.size();
    u.num_bvh_nodes = (uint32_t)s.bvh.nodes.size();
    u.num_lights = (uint32_t)s.lights.size();
    u.sampling_mode = sampling;
    s.background.to(u.background);
    u.env_width = s.env.width;
    u.env_height = s.env.height;
    u.env_total_weight = s.env.total_weight;
    u.sampler_kind = sampler;
    s.camera.write_uniforms(u, (float)width / (float)height);
    return u;
}

// integrator.rs:418-532
static Vec3 direct_light(const Scene& scene, const Surface& surf, const Hit& hit, Vec3 wo,
                         Sampler& rng, uint32_t mode) {
    float u_select = rng.next_f32();
    Vec2 u_area = rng.next_vec2();
    uint32_t n_lights = (uint32_t)scene.lights.size();
    uint32_t total = scene.light_strategy_count();
    if (total == 0) return Vec3();
    uint32_t pick = std::min(f2u(u_select * (float)total), total - 1);
    sig_event(5, pick);
    Vec3 wi_world, radiance;
    float distance, pdf;
    if (pick < n_lights) {
        // light::sample_lights (light.rs:173-221) with u_select = cell centre
        float u_light = ((float)pick + 0.5f) / (float)n_lights;
        size_t n = scene.lights.size();
        size_t index = std::min<size_t>(f2usize(u_light * (float)n), n - 1);
        const GpuLight& light = scene.lights[index];
        // sample_light_point (light.rs:144-164)
        Vec3 o = Vec3::from(light.origin), eu = Vec3::from(light.edge_u), ev = Vec3::from(light.edge_v);
        Vec3 point;
        if (light.kind == LIGHT_KIND_TRIANGLE) {
            float su = std::sqrt(u_area.x);
            float b1 = 1.0f - su;
            float b2 = u_area.y * su;
            point = o + b1 * eu + b2 * ev;
        } else {
            point = o + u_area.x * eu + u_area.y * ev;
        }
        Vec3 ln = Vec3::from(light.normal);
        Vec3 to_light = point - hit.position;
        float dist_sq = to_light.length_squared();
        if (dist_sq <= 0.0f) return Vec3();
        float dist = std::sqrt(dist_sq);
        Vec3 wi = to_light / dist;
        float cos_light = ln.dot(-wi);
        if (cos_light <= MIN_COS_LIGHT) return Vec3();
        float pdf_area = 1.0f / ((float)n * light.area);
        float lpdf = pdf_area * dist_sq / cos_light;
        if (!std::isfinite(lpdf) || lpdf <= 0.0f) return Vec3();
        float scale = (float)n_lights / (float)total;
        wi_world = wi;
        radiance = Vec3::from(scene.materials[light.material].emissive);
        distance = dist;
        pdf = lpdf * scale;
    } else {
        EnvSample es = scene.env.sample(u_area);
        if (es.pdf <= 0.0f) return Vec3();
        wi_world = es.direction;
        radiance = es.radiance;
        distance = INFINITY;
        pdf = es.pdf / (float)total;
    }
    if (pdf <= 0.0f) return Vec3();
    Vec3 wi = to_local(wi_world, hit.normal);
    if (wi.z == 0.0f || (wi.z < 0.0f && surf.transmission <= 0.0f)) return Vec3();
    Vec3 f = surface_eval(surf, wo, wi);
    if (f.max_element() <= 0.0f) return Vec3();
    float mis = 1.0f;
    if (mode == LUC_SAMPLING_MIS) mis = power_heuristic(pdf, surface_pdf(surf, wo, wi));
    if (mis <= 0.0f) return Vec3();
    Vec3 origin = offset_ray_origin(hit.position, wi.z < 0.0f ? -hit.geometric_normal : hit.geometric_normal);
    // light::unoccluded (light.rs:327-333)
    if (scene.occluded(Ray{origin, wi_world}, distance * (1.0f - 1.0e-3f))) return Vec3();
    return f * std::fabs(wi.z) * radiance * (mis / pdf);
}

// integrator.rs:209-403
Vec3 radiance_with_guide(const Scene& scene, Ray ray, Sampler& rng, uint32_t max_depth, uint32_t mode,
                         GuideSample& guide) {
    Vec3 radiance;
    Vec3 throughput = Vec3::splat(1.0f);
    float prev_bsdf_pdf = 0.0f;
    Vec3 prev_position = ray.origin;
    for (uint32_t depth = 0; depth < max_depth; ++depth) {
        Hit hit;
        if (!scene.intersect(ray, hit)) {
            const EnvMap& env = scene.env;
            if (!env.is_empty()) {
                Vec3 l = env.radiance(ray.dir);
                float weight;
                if (depth == 0) {
                    weight = 1.0f;
                } else if (mode == LUC_SAMPLING_BSDF) {
                    weight = 1.0f;
                } else if (mode == LUC_SAMPLING_NEE) {
                    weight = 0.0f;
                } else {
                    uint32_t total = std::max(scene.light_strategy_count(), 1u);
                    float pdf_env = env.pdf(ray.dir) / (float)total;
                    weight = power_heuristic(prev_bsdf_pdf, pdf_env);
                }
                if (weight > 0.0f) radiance += throughput * l * weight;
            } else {
                radiance += throughput * scene.background;
            }
            break;
        }
        const GpuMaterial& m = scene.materials[hit.material];
        Vec3 emissive = Vec3::from(m.emissive);
        if (hit.front_face && emissive.max_element() > 0.0f) {
            float weight;
            if (depth == 0) {
                weight = 1.0f;
            } else if (mode == LUC_SAMPLING_BSDF) {
                weight = 1.0f;
            } else if (mode == LUC_SAMPLING_NEE) {
                weight = 0.0f;
            } else {
                uint32_t n = (uint32_t)scene.lights.size();
                uint32_t total = scene.light_strategy_count();
                float pdf_light = light_pdf_from_geometry(n, hit.light_area, hit.geometric_normal,
                                                          prev_position, hit.position) *
                                  ((float)n / (float)std::max(total, 1u));
                weight = power_heuristic(prev_bsdf_pdf, pdf_light);
            }
            if (weight > 0.0f) radiance += throughput * emissive * weight;
        }
        Surface surf = Surface::from_material(m, hit.front_face);
        if (depth == 0) {
            guide.albedo = (surf.diffuse_albedo + surf.f0 + emissive).max(Vec3::splat(1.0e-3f));
            guide.normal = hit.normal;
            guide.depth = hit.t;
            guide.steps = (float)hit.steps;
        }
        Vec3 wo = to_local(-ray.dir, hit.normal);
        if (wo.z <= 0.0f) {
            sig_event(8, 0);
            break;
        }
        bool has_env = !scene.env.is_empty();
        if ((mode == LUC_SAMPLING_NEE || mode == LUC_SAMPLING_MIS) && depth + 1 < max_depth &&
            (!scene.lights.empty() || has_env)) {
            Vec3 dl = direct_light(scene, surf, hit, wo, rng, mode);
            sig_event(6, dl.max_element() > 0.0f);
            radiance += throughput * dl;
        }
        float u_lobe = rng.next_f32();
        Vec2 u = rng.next_vec2();
        BsdfSample smp = surface_sample(surf, wo, u_lobe, u);
        if (!smp.valid()) break;
        throughput *= smp.weight;
        if (throughput.max_element() <= 0.0f) {
            sig_event(7, 0);
            break;
        }
        prev_bsdf_pdf = smp.pdf;
        prev_position = hit.position;
        Vec3 dir = to_world(smp.wi, hit.normal);
        ray = Ray{offset_ray_origin(hit.position, smp.wi.z < 0.0f ? -hit.geometric_normal : hit.geometric_normal),
                  dir};
    }
    return radiance;
}

// integrator.rs:536-589 and the 32-row band scheduler of :635-699. Sums are
// kept (not multiplied by 1/spp) so the caller can compare against an
// accumulator.
void render_sums(const Scene& s, const GpuUniforms& u, uint32_t threads, std::vector<PixelSums>& out,
                 uint32_t row0, uint32_t row1, uint32_t band) {
    const uint32_t BAND = band == 0 ? 32 : band;
    out.assign((size_t)u.width * (row1 - row0), PixelSums{});
    uint32_t rows = row1 - row0;
    uint32_t num_bands = (rows + BAND - 1) / BAND;
    std::atomic<uint32_t> next{0};
    uint32_t mode = u.sampling_mode == 0 ? LUC_SAMPLING_BSDF : (u.sampling_mode == 1 ? LUC_SAMPLING_NEE : LUC_SAMPLING_MIS);
    uint32_t kind = u.sampler_kind == LUC_SAMPLER_SOBOL ? LUC_SAMPLER_SOBOL : LUC_SAMPLER_INDEPENDENT;
    auto worker = [&] {
        for (;;) {
            uint32_t b = next.fetch_add(1);
            if (b >= num_bands) break;
            uint32_t y0 = row0 + b * BAND, y1 = std::min(row1, y0 + BAND);
            for (uint32_t y = y0; y < y1; ++y) {
                for (uint32_t x = 0; x < u.width; ++x) {
                    uint32_t pixel = y * u.width + x;
                    PixelSums ps{};
                    for (uint32_t k = 0; k < u.samples_per_launch; ++k) {
                        Sampler rng(kind, u.frame_seed, pixel, u.sample_offset + k);
                        Vec2 puv = rng.next_vec2();
                        Vec2 luv = rng.next_vec2();
                        Ray ray = generate_ray(u, x, y, puv, luv);
                        GuideSample g;
                        Vec3 r = radiance_with_guide(s, ray, rng, u.max_depth, mode, g);
                        ps.radiance += r;
                        ps.radiance_sq += r * r;
                        ps.albedo += g.albedo;
                        ps.normal += g.normal;
                        ps.depth = ps.depth + g.depth;
                    }
                    out[(size_t)(y - row0) * u.width + x] = ps;
                }
            }
        }
    };
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
}

// One sample (pixel x, y; sample index k of the uniforms' range) traced as
// render_sums traces it, with its path signature (g_path_sig events).
Vec3 trace_sample(const Scene& s, const GpuUniforms& u, uint32_t x, uint32_t y, uint32_t k, uint64_t& sig) {
    uint32_t mode = u.sampling_mode == 0 ? LUC_SAMPLING_BSDF : (u.sampling_mode == 1 ? LUC_SAMPLING_NEE : LUC_SAMPLING_MIS);
    uint32_t kind = u.sampler_kind == LUC_SAMPLER_SOBOL ? LUC_SAMPLER_SOBOL : LUC_SAMPLER_INDEPENDENT;
    uint32_t pixel = y * u.width + x;
    Sampler rng(kind, u.frame_seed, pixel, u.sample_offset + k);
    Vec2 puv = rng.next_vec2();
    Vec2 luv = rng.next_vec2();
    Ray ray = generate_ray(u, x, y, puv, luv);
    GuideSample g;
    sig = 0;
    g_path_sig = &sig;
    Vec3 r = radiance_with_guide(s, ray, rng, u.max_depth, mode, g);
    g_path_sig = nullptr;
    return r;
}

}  // namespace oracle
