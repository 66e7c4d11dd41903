// ORACLE — test infrastructure only (see oracle_core.hpp). A C ABI over the
// restatement so tests/ (through oracle/__init__.py) can drive it with ctypes.
#include "oracle_scene.hpp"
#include <atomic>
#include <thread>

using namespace oracle;

namespace {
struct LbvhHandle {
    LbvhStages s;
};
enum Which {
    W_MATERIALS = 0, W_PRIMITIVES, W_LIGHTS, W_POSITIONS, W_ATTRS, W_TRIANGLES, W_BVH_NODES,
    W_BVH_PRIMS, W_ENV_PIXELS, W_ENV_COND, W_ENV_MARG
};
}  // namespace

extern "C" {

void* orc_scene_builtin(const char* name) {
    Scene* s = new Scene();
    if (!scene_by_name(name, *s)) {
        delete s;
        return nullptr;
    }
    return s;
}

// Assemble a scene from the upload arrays. `bvh_kind`: 0 = binned SAH (what
// Scene::finalize does), 1 = the CPU LBVH. `lights` may be null, in which case
// build_lights runs after compaction exactly as Scene::finalize does; when
// given, it is used verbatim (the light list does not depend on triangle order).
void* orc_scene_from_arrays(const GpuMaterial* mats, uint32_t nm, const GpuPrimitive* prims, uint32_t np,
                            const GpuLight* lights, uint32_t nl, const float* pos4, uint32_t nv,
                            const GpuVertexAttr* attrs, const GpuTriangle* tris, uint32_t nt,
                            const float* env_px, uint32_t env_w, uint32_t env_h, const float* env_cond,
                            const float* env_marg, float env_total, const float* background, int bvh_kind) {
    Scene* s = new Scene();
    s->materials.assign(mats, mats + nm);
    s->primitives.assign(prims, prims + np);
    s->positions.assign(pos4, pos4 + 4 * (size_t)nv);
    s->vertex_attrs.assign(attrs, attrs + nv);
    s->triangles.assign(tris, tris + nt);
    if (env_w > 0 && env_px) {
        s->env.width = env_w;
        s->env.height = env_h;
        s->env.pixels.assign(env_px, env_px + 4 * (size_t)env_w * env_h);
        s->env.conditional.assign(env_cond, env_cond + (size_t)(env_w + 1) * env_h);
        s->env.marginal.assign(env_marg, env_marg + env_h + 1);
        s->env.total_weight = env_total;
    }
    s->background = background ? Vec3::from(background) : Vec3();
    if (!s->triangles.empty() && bvh_kind != 2) {  // 2: the caller supplies the tree (orc_scene_set_instancing)
        if (bvh_kind == 1) s->bvh = lbvh_build(s->triangles, s->positions, 4).tree;
        else s->bvh = Bvh::build(s->triangles, s->positions);
        s->bvh.compact_primitives(s->triangles);
    }
    if (lights) s->lights.assign(lights, lights + nl);
    else s->lights = build_lights(s->materials, s->primitives, s->triangles, s->positions);
    return s;
}

// Instanced scene in the upload's form: the last `num_instances` primitives
// are GpuInstance rows in TLAS-leaf order, `nodes` the flattened BLAS + TLAS
// array, `tlas_root` the TLAS's first node.
void orc_scene_set_instancing(void* h, const GpuBvhNode* nodes, uint32_t nn, uint32_t num_instances,
                              uint32_t tlas_root) {
    Scene* s = (Scene*)h;
    size_t na = s->primitives.size() - num_instances;
    s->instances.resize(num_instances);
    if (num_instances) std::memcpy(s->instances.data(), s->primitives.data() + na, num_instances * sizeof(GpuInstance));
    s->primitives.resize(na);
    s->flat_nodes.assign(nodes, nodes + nn);
    s->tlas_root = tlas_root;
    s->bvh = Bvh();
}
// out3: instance count, analytic primitive count, TLAS root.
void orc_scene_instancing(void* h, uint32_t* out3) {
    Scene* s = (Scene*)h;
    out3[0] = (uint32_t)s->instances.size();
    out3[1] = (uint32_t)s->primitives.size();
    out3[2] = s->tlas_root;
}
// Device-built instancing restated (Scene::build_instances_lbvh): mesh
// ranges of the scene's (object-space) triangles and placements given by
// row-major 3x4 object-to-world transforms.
void orc_scene_build_instances_lbvh(void* h, const uint32_t* first, const uint32_t* count, uint32_t nm,
                                    const float* o2w, const uint32_t* mesh, const uint32_t* material, uint32_t n) {
    Scene* s = (Scene*)h;
    std::vector<std::pair<uint32_t, uint32_t>> ranges;
    for (uint32_t m = 0; m < nm; ++m) ranges.push_back({first[m], count[m]});
    std::vector<Scene::Placement> pl(n);
    for (uint32_t i = 0; i < n; ++i) {
        std::memcpy(pl[i].object_to_world.m, o2w + 12 * (size_t)i, 48);
        pl[i].mesh = mesh[i];
        pl[i].material = material[i];
    }
    s->build_instances_lbvh(ranges, pl);
}
void orc_scene_set_reference_shadows(void* h, int on) { ((Scene*)h)->reference_instance_shadows = on != 0; }

// Instance maths (instance.rs): affine inverse of a row-major 3x4; pack an
// instance from a world-to-object transform; transform n points (mode 0),
// vectors (1) or normals (2); world bounds of a box (6 floats: min, max).
void orc_affine_inverse(const float* in12, float* out12) {
    Affine a;
    std::memcpy(a.m, in12, sizeof(a.m));
    Affine r = affine_inverse(a);
    std::memcpy(out12, r.m, sizeof(r.m));
}
void orc_pack_instance(const float* w2o12, uint32_t blas_root, uint32_t material, GpuInstance* out) {
    Affine a;
    std::memcpy(a.m, w2o12, sizeof(a.m));
    *out = pack_instance(a, blas_root, material);
}
void orc_instance_transform(const GpuInstance* g, int mode, const float* in3, uint32_t n, float* out3) {
    for (uint32_t i = 0; i < n; ++i) {
        Vec3 v = Vec3::from(in3 + 3 * i);
        Vec3 r = mode == 0 ? instance_point(*g, v) : mode == 1 ? instance_vector(*g, v) : instance_normal(*g, v);
        r.to(out3 + 3 * i);
    }
}
void orc_instance_world_bounds(const GpuInstance* g, const float* box6, float* out6) {
    Aabb b;
    b.min = Vec3::from(box6);
    b.max = Vec3::from(box6 + 3);
    Aabb w = instance_world_bounds(*g, b);
    w.min.to(out6);
    w.max.to(out6 + 3);
}

void orc_scene_set_camera(void* h, const float* eye, const float* at, const float* up, float vfov,
                          float aperture, float focus) {
    Scene* s = (Scene*)h;
    s->camera.eye = Vec3::from(eye);
    s->camera.look_at = Vec3::from(at);
    s->camera.up = Vec3::from(up);
    s->camera.vfov_deg = vfov;
    s->camera.aperture = aperture;
    s->camera.focus_distance = focus;
}
void orc_scene_get_camera(void* h, float* out10) {
    Scene* s = (Scene*)h;
    s->camera.eye.to(out10);
    s->camera.look_at.to(out10 + 3);
    s->camera.up.to(out10 + 6);
    out10[9] = s->camera.vfov_deg;
}
void orc_scene_get_misc(void* h, float* bg3, float* env_total, uint32_t* env_wh) {
    Scene* s = (Scene*)h;
    s->background.to(bg3);
    *env_total = s->env.total_weight;
    env_wh[0] = s->env.width;
    env_wh[1] = s->env.height;
}
void orc_scene_free(void* h) { delete (Scene*)h; }

size_t orc_scene_count(void* h, int which) {
    Scene* s = (Scene*)h;
    switch (which) {
        case W_MATERIALS: return s->materials.size();
        case W_PRIMITIVES: return s->primitives.size() + s->instances.size();
        case W_LIGHTS: return s->lights.size();
        case W_POSITIONS: return s->positions.size() / 4;
        case W_ATTRS: return s->vertex_attrs.size();
        case W_TRIANGLES: return s->triangles.size();
        case W_BVH_NODES: return s->instances.empty() ? s->bvh.nodes.size() : s->flat_nodes.size();
        case W_BVH_PRIMS: return s->bvh.prim_indices.size();
        case W_ENV_PIXELS: return s->env.pixels.size() / 4;
        case W_ENV_COND: return s->env.conditional.size();
        case W_ENV_MARG: return s->env.marginal.size();
    }
    return 0;
}
void orc_scene_copy(void* h, int which, void* dst) {
    Scene* s = (Scene*)h;
    auto cp = [&](const void* src, size_t bytes) { if (bytes) std::memcpy(dst, src, bytes); };
    switch (which) {
        case W_MATERIALS: cp(s->materials.data(), s->materials.size() * sizeof(GpuMaterial)); break;
        case W_PRIMITIVES:
            cp(s->primitives.data(), s->primitives.size() * sizeof(GpuPrimitive));
            if (!s->instances.empty())
                std::memcpy((char*)dst + s->primitives.size() * sizeof(GpuPrimitive), s->instances.data(),
                            s->instances.size() * sizeof(GpuInstance));
            break;
        case W_LIGHTS: cp(s->lights.data(), s->lights.size() * sizeof(GpuLight)); break;
        case W_POSITIONS: cp(s->positions.data(), s->positions.size() * 4); break;
        case W_ATTRS: cp(s->vertex_attrs.data(), s->vertex_attrs.size() * sizeof(GpuVertexAttr)); break;
        case W_TRIANGLES: cp(s->triangles.data(), s->triangles.size() * sizeof(GpuTriangle)); break;
        case W_BVH_NODES:
            if (s->instances.empty()) cp(s->bvh.nodes.data(), s->bvh.nodes.size() * sizeof(GpuBvhNode));
            else cp(s->flat_nodes.data(), s->flat_nodes.size() * sizeof(GpuBvhNode));
            break;
        case W_BVH_PRIMS: cp(s->bvh.prim_indices.data(), s->bvh.prim_indices.size() * 4); break;
        case W_ENV_PIXELS: cp(s->env.pixels.data(), s->env.pixels.size() * 4); break;
        case W_ENV_COND: cp(s->env.conditional.data(), s->env.conditional.size() * 4); break;
        case W_ENV_MARG: cp(s->env.marginal.data(), s->env.marginal.size() * 4); break;
    }
}

void orc_build_uniforms(void* h, uint32_t w, uint32_t ht, uint32_t spp, uint32_t depth, uint32_t seed,
                        uint32_t offset, uint32_t sampling, uint32_t sampler, GpuUniforms* out) {
    *out = build_uniforms(*(Scene*)h, w, ht, spp, depth, seed, offset, sampling, sampler);
}

// Per pixel of rows [row0, row1): 13 floats — radiance sum (3), squared
// radiance sum (3), albedo sum (3), normal sum (3), depth sum (1).
void orc_render_sums(void* h, const GpuUniforms* u, uint32_t threads, uint32_t row0, uint32_t row1, uint32_t band,
                     float* out) {
    std::vector<PixelSums> ps;
    render_sums(*(Scene*)h, *u, threads, ps, row0, row1, band);
    for (size_t i = 0; i < ps.size(); ++i) {
        float* o = out + 13 * i;
        ps[i].radiance.to(o);
        ps[i].radiance_sq.to(o + 3);
        ps[i].albedo.to(o + 6);
        ps[i].normal.to(o + 9);
        o[12] = ps[i].depth;
    }
}

// render_sums over an explicit list of image rows (each row one work item,
// handed to `threads` workers through an atomic counter): a bounded sample
// of a frame spread over its whole height. Output rows in list order.
void orc_render_row_list(void* h, const GpuUniforms* u, uint32_t threads, const uint32_t* rows, uint32_t nrows,
                         float* out) {
    const Scene& s = *(Scene*)h;
    std::atomic<uint32_t> next{0};
    auto worker = [&] {
        std::vector<PixelSums> ps;
        for (;;) {
            uint32_t i = next.fetch_add(1);
            if (i >= nrows) break;
            render_sums(s, *u, 1, ps, rows[i], rows[i] + 1, 1);
            for (uint32_t x = 0; x < u->width; ++x) {
                float* o = out + 13 * ((size_t)i * u->width + x);
                ps[x].radiance.to(o);
                ps[x].radiance_sq.to(o + 3);
                ps[x].albedo.to(o + 6);
                ps[x].normal.to(o + 9);
                o[12] = ps[x].depth;
            }
        }
    };
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
}

// Render-time transcendental rounding: 0 = glibc f32 (the reference), 1 =
// double evaluation rounded once (the CUDA integrator's). Call between renders.
void orc_set_libm_mode(int mode) { g_libm_mode = mode ? 1 : 0; }
int orc_get_libm_mode(void) { return g_libm_mode; }

// Every sample of the listed pixels traced on its own: radiance (3 floats)
// and path signature per (pixel, sample), pixel-major. Threads split pixels.
void orc_sample_traces(void* h, const GpuUniforms* u, const uint32_t* pixels, uint32_t n, uint32_t threads,
                       float* rad_out, uint64_t* sig_out) {
    const Scene& s = *(Scene*)h;
    const uint32_t spp = u->samples_per_launch;
    std::atomic<uint32_t> next{0};
    auto worker = [&] {
        for (;;) {
            uint32_t i = next.fetch_add(1);
            if (i >= n) break;
            uint32_t x = pixels[i] % u->width, y = pixels[i] / u->width;
            for (uint32_t k = 0; k < spp; ++k) {
                uint64_t sig;
                Vec3 r = trace_sample(s, *u, x, y, k, sig);
                r.to(rad_out + 3 * ((size_t)i * spp + k));
                sig_out[(size_t)i * spp + k] = sig;
            }
        }
    };
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& t : pool) t.join();
}

// Closest hit for a batch of rays (origin3, dir3): t, material, front_face,
// position3, normal3, geometric_normal3, light_area -> 12 floats (u32 bits
// stored as float bit patterns for material/front_face). Miss: t = -1.
void orc_intersect_batch(void* h, const float* rays6, uint32_t n, float* out12) {
    Scene* s = (Scene*)h;
    for (uint32_t i = 0; i < n; ++i) {
        Ray r{Vec3::from(rays6 + 6 * i), Vec3::from(rays6 + 6 * i + 3)};
        Hit hit;
        float* o = out12 + 12 * i;
        if (!s->intersect(r, hit)) {
            std::memset(o, 0, 48);
            o[0] = -1.0f;
            continue;
        }
        o[0] = hit.t;
        o[1] = from_bits(hit.material);
        o[2] = from_bits(hit.front_face ? 1u : 0u);
        hit.position.to(o + 3);
        hit.normal.to(o + 6);
        o[9] = hit.geometric_normal.x;
        o[10] = hit.geometric_normal.y;
        o[11] = hit.geometric_normal.z;
    }
}

// ---- samplers
uint32_t orc_pcg_hash(uint32_t x) { return pcg_hash(x); }
uint32_t orc_hash_u32(uint32_t x) { return hash_u32(x); }
uint32_t orc_owen_scramble(uint32_t x, uint32_t seed) { return owen_scramble(x, seed); }
uint32_t orc_sobol(uint32_t index, uint32_t dim) { return sobol(index, dim); }
float orc_sobol_sample(uint32_t index, uint32_t dim, uint32_t seed) { return sobol_sample(index, dim, seed); }
// `pattern` is a string of 'f' (next_f32) and 'v' (next_vec2) draws; the
// outputs are written in draw order (a 'v' writes two floats).
void orc_sampler_stream(uint32_t kind, uint32_t frame_seed, uint32_t pixel, uint32_t sample,
                        const char* pattern, float* out) {
    Sampler s(kind, frame_seed, pixel, sample);
    size_t k = 0;
    for (const char* p = pattern; *p; ++p) {
        if (*p == 'f') {
            out[k++] = s.next_f32();
        } else {
            Vec2 v = s.next_vec2();
            out[k++] = v.x;
            out[k++] = v.y;
        }
    }
}
void orc_energy_table(float* out) {
    const float* t = energy_table();
    std::memcpy(out, t, sizeof(float) * ENERGY_TABLE_SIZE * ENERGY_TABLE_SIZE);
}

// ---- BSDF per function, for sampler/pdf tests and device-function diffs.
void orc_bsdf_eval_batch(const GpuMaterial* m, int front, const float* wo3, const float* wi3, uint32_t n,
                         float* f3, float* pdf) {
    Surface s = Surface::from_material(*m, front != 0);
    for (uint32_t i = 0; i < n; ++i) {
        Vec3 wo = Vec3::from(wo3 + 3 * i), wi = Vec3::from(wi3 + 3 * i);
        surface_eval(s, wo, wi).to(f3 + 3 * i);
        pdf[i] = surface_pdf(s, wo, wi);
    }
}
void orc_bsdf_sample_batch(const GpuMaterial* m, int front, const float* wo3, const float* u3, uint32_t n,
                           float* wi3, float* w3, float* pdf) {
    Surface s = Surface::from_material(*m, front != 0);
    for (uint32_t i = 0; i < n; ++i) {
        BsdfSample b = surface_sample(s, Vec3::from(wo3 + 3 * i), u3[3 * i], Vec2(u3[3 * i + 1], u3[3 * i + 2]));
        b.wi.to(wi3 + 3 * i);
        b.weight.to(w3 + 3 * i);
        pdf[i] = b.pdf;
    }
}
void orc_env_sample_batch(void* h, const float* u2, uint32_t n, float* dir3, float* rad3, float* pdf) {
    Scene* s = (Scene*)h;
    for (uint32_t i = 0; i < n; ++i) {
        EnvSample e = s->env.sample(Vec2(u2[2 * i], u2[2 * i + 1]));
        e.direction.to(dir3 + 3 * i);
        e.radiance.to(rad3 + 3 * i);
        pdf[i] = e.pdf;
    }
}
void orc_env_pdf_batch(void* h, const float* dir3, uint32_t n, float* pdf, float* rad3) {
    Scene* s = (Scene*)h;
    for (uint32_t i = 0; i < n; ++i) {
        pdf[i] = s->env.pdf(Vec3::from(dir3 + 3 * i));
        s->env.radiance(Vec3::from(dir3 + 3 * i)).to(rad3 + 3 * i);
    }
}
// envmap.rs:114-178 over caller pixels (4 floats per texel): conditional
// (w+1)*h, marginal h+1, returns total weight.
float orc_env_build(const float* px, uint32_t w, uint32_t h, float* cond, float* marg) {
    EnvMap e = EnvMap::build(w, h, std::vector<float>(px, px + 4 * (size_t)w * h));
    std::memcpy(cond, e.conditional.data(), e.conditional.size() * 4);
    std::memcpy(marg, e.marginal.data(), e.marginal.size() * 4);
    return e.total_weight;
}

// ---- BVH / LBVH
void* orc_lbvh_build(const GpuTriangle* tris, uint32_t nt, const float* pos4, uint32_t nv, uint32_t max_leaf) {
    LbvhHandle* h = new LbvhHandle();
    h->s = lbvh_build(std::vector<GpuTriangle>(tris, tris + nt), std::vector<float>(pos4, pos4 + 4 * (size_t)nv),
                      max_leaf);
    return h;
}
void* orc_lbvh_build_over_bounds(const float* boxes6, uint32_t n, uint32_t max_leaf) {
    std::vector<Aabb> b(n);
    for (uint32_t i = 0; i < n; ++i) {
        b[i].min = Vec3::from(boxes6 + 6 * i);
        b[i].max = Vec3::from(boxes6 + 6 * i + 3);
    }
    LbvhHandle* h = new LbvhHandle();
    h->s = lbvh_build_over_bounds(b, max_leaf);
    return h;
}
// field: 0 tri_bounds (6 floats each), 1 centroid_bounds (6), 2 codes, 3 order,
// 4 sorted_codes, 5 karras (2 per node), 6 parent, 7 node_bounds (6 each),
// 8 subtree_size, 9 nodes (8 words each), 10 prim_indices. Returns element
// count (words for u32 fields, boxes for box fields, nodes for 9).
size_t orc_lbvh_field(void* hh, int field, void* dst) {
    LbvhStages& s = ((LbvhHandle*)hh)->s;
    auto boxes = [&](const std::vector<Aabb>& v) {
        if (dst)
            for (size_t i = 0; i < v.size(); ++i) {
                v[i].min.to((float*)dst + 6 * i);
                v[i].max.to((float*)dst + 6 * i + 3);
            }
        return v.size();
    };
    auto words = [&](const std::vector<uint32_t>& v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * 4);
        return v.size();
    };
    switch (field) {
        case 0: return boxes(s.tri_bounds);
        case 1: return boxes(std::vector<Aabb>{s.centroid_bounds});
        case 2: return words(s.codes);
        case 3: return words(s.order);
        case 4: return words(s.sorted_codes);
        case 5: return words(s.karras);
        case 6: return words(s.parent);
        case 7: return boxes(s.node_bounds);
        case 8: return words(s.subtree_size);
        case 9:
            if (dst && !s.tree.nodes.empty()) std::memcpy(dst, s.tree.nodes.data(), s.tree.nodes.size() * 32);
            return s.tree.nodes.size();
        case 10: return words(s.tree.prim_indices);
    }
    return 0;
}
float orc_lbvh_sah_cost(void* hh) { return ((LbvhHandle*)hh)->s.tree.sah_cost(); }
void orc_lbvh_free(void* hh) { delete (LbvhHandle*)hh; }

uint32_t orc_morton3d(float x, float y, float z) { return morton3d(Vec3(x, y, z)); }
uint32_t orc_expand_bits(uint32_t v) { return expand_bits(v); }
int32_t orc_lcp(const uint32_t* codes, int64_t n, int32_t i, int32_t j) { return longest_common_prefix(codes, n, i, j); }

// SAH tree over triangles; writes nodes (n_nodes*32 bytes) and prim indices
// when the destinations are non-null; returns node count.
void* orc_sah_build(const GpuTriangle* tris, uint32_t nt, const float* pos4, uint32_t nv) {
    Bvh* b = new Bvh(Bvh::build(std::vector<GpuTriangle>(tris, tris + nt),
                                std::vector<float>(pos4, pos4 + 4 * (size_t)nv)));
    return b;
}
size_t orc_bvh_nodes(void* h, GpuBvhNode* dst) {
    Bvh* b = (Bvh*)h;
    if (dst && !b->nodes.empty()) std::memcpy(dst, b->nodes.data(), b->nodes.size() * 32);
    return b->nodes.size();
}
size_t orc_bvh_prims(void* h, uint32_t* dst) {
    Bvh* b = (Bvh*)h;
    if (dst && !b->prim_indices.empty()) std::memcpy(dst, b->prim_indices.data(), b->prim_indices.size() * 4);
    return b->prim_indices.size();
}
float orc_bvh_sah_cost(void* h) { return ((Bvh*)h)->sah_cost(); }
int orc_bvh_validate(void* h, uint32_t tc) { return (int)((Bvh*)h)->validate(tc).size(); }
void orc_bvh_free(void* h) { delete (Bvh*)h; }
float orc_nodes_sah_cost(const GpuBvhNode* nodes, uint32_t n) {
    Bvh b;
    b.nodes.assign(nodes, nodes + n);
    return b.sah_cost();
}

// Stable ascending sort of (key, value) pairs by (key, original position):
// the order `order.sort_by_key(|&i| (codes[i], i))` produces (lbvh.rs:458-460).
void orc_sort_pairs(const uint32_t* keys, const uint32_t* vals, uint32_t n, uint32_t* ko, uint32_t* vo) {
    std::vector<uint32_t> idx(n);
    for (uint32_t i = 0; i < n; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
    for (uint32_t i = 0; i < n; ++i) {
        ko[i] = keys[idx[i]];
        vo[i] = vals[idx[i]];
    }
}

// ---- denoiser: film/albedo/normal 3 floats per pixel, depth 1.
void orc_denoise(const float* film, const float* albedo, const float* normal, const float* depth, uint32_t w,
                 uint32_t h, uint32_t iterations, float sn, float sd, float sl, float sa, float* out) {
    size_t n = (size_t)w * h;
    std::vector<Vec3> f(n), a(n), nn(n), o;
    std::vector<float> d(depth, depth + n);
    for (size_t i = 0; i < n; ++i) {
        f[i] = Vec3::from(film + 3 * i);
        a[i] = Vec3::from(albedo + 3 * i);
        nn[i] = Vec3::from(normal + 3 * i);
    }
    DenoiseParams p;
    p.iterations = iterations;
    p.sigma_normal = sn;
    p.sigma_depth = sd;
    p.sigma_luminance = sl;
    p.sigma_albedo = sa;
    denoise(f, a, nn, d, w, h, p, o);
    for (size_t i = 0; i < n; ++i) o[i].to(out + 3 * i);
}

// ---- meshes
// Icosphere into caller buffers: positions (4 floats), normals (3), uvs (2),
// indices (3 per triangle). Returns vertex count; call with null buffers to
// size them (triangles = 20 * 4^levels).
uint32_t orc_icosphere(float cx, float cy, float cz, float radius, uint32_t levels, float* pos4, float* nrm3,
                       float* uv2, uint32_t* idx3) {
    MeshBuilder m = icosphere(Vec3(cx, cy, cz), radius, levels);
    if (pos4)
        for (size_t i = 0; i < m.positions.size(); ++i) {
            m.positions[i].to(pos4 + 4 * i);
            pos4[4 * i + 3] = 0.0f;
            m.normals[i].to(nrm3 + 3 * i);
            uv2[2 * i] = m.uvs[i].x;
            uv2[2 * i + 1] = m.uvs[i].y;
        }
    if (idx3) std::memcpy(idx3, m.indices.data(), m.indices.size() * 4);
    return (uint32_t)m.positions.size();
}

float orc_glibc_sinf(float x) { return std::sin(x); }
float orc_glibc_cosf(float x) { return std::cos(x); }
void orc_transcendental_batch(int fn, const float* x, const float* y, uint32_t n, float* out) {
    for (uint32_t i = 0; i < n; ++i) {
        switch (fn) {
            case 0: out[i] = std::sin(x[i]); break;
            case 1: out[i] = std::cos(x[i]); break;
            case 2: out[i] = std::acos(x[i]); break;
            case 3: out[i] = std::atan2(x[i], y[i]); break;
            case 4: out[i] = std::exp(x[i]); break;
            case 5: out[i] = std::pow(x[i], y[i]); break;
            case 6: out[i] = std::asin(x[i]); break;
            case 7: out[i] = std::tan(x[i]); break;
        }
    }
}

}  // extern "C"
