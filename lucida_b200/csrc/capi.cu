// The C ABI of liblucida_cuda.so (include/luc_cuda.h): context, scene
// residency, and the render(scene, camera, spp, bounces) entry point.
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "ctx.cuh"

using namespace luc;

int32_t luc_fail(luc_ctx* c, int32_t code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}
int32_t luc_cuda_fail(luc_ctx* c, cudaError_t e, const char* what) {
    int32_t code = e == cudaErrorMemoryAllocation ? LUC_ERR_OUT_OF_MEMORY : LUC_ERR_LAUNCH;
    return luc_fail(c, code, std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

// The white-Fresnel single-scattering GGX directional albedo table that the
// Turquin compensation interpolates (crates/core/src/bsdf.rs:1210-1225,
// 760-777): 32x32 entries over (roughness, sqrt(cos_o)), each a 128x128
// midpoint quadrature over the VNDF sampler's unit square, summed in double.
// Computed once per context on the host, with the same f32 operations (and
// the same libm) the reference's CPU build uses, so the GPU interpolates the
// identical table.
std::vector<float> energy_table_host() {
    const float PI = 3.14159265358979323846f;
    auto alpha_of = [](float r) { return std::fmax(r * r, 2.0e-3f); };
    auto lambda = [](float a, float ct) {
        float c = std::fabs(ct);
        if (c >= 1.0f) return 0.0f;
        float c2 = c * c;
        float tan2 = (1.0f - c2) / std::fmax(c2, 1.0e-12f);
        return 0.5f * (-1.0f + std::sqrt(1.0f + a * a * tan2));
    };
    auto ggx = [&](float a, float c) {
        if (c <= 0.0f) return 0.0f;
        float a2 = a * a, c2 = c * c, s2 = std::fmax(1.0f - c2, 0.0f), den = a2 * c2 + s2;
        return a2 / (PI * den * den);
    };
    std::vector<float> t(32 * 32);
    for (int ri = 0; ri < 32; ++ri) {
        float roughness = (float)ri / 31.0f;
        float a = alpha_of(roughness);
        for (int ci = 0; ci < 32; ++ci) {
            float rm = (float)ci / 31.0f;
            float mu = std::fmax(rm * rm, 1.0e-4f);
            float st = std::sqrt(std::fmax(1.0f - mu * mu, 0.0f));
            float wo[3] = {st, 0.0f, mu};
            double sum = 0.0;
            for (int i = 0; i < 128; ++i) {
                for (int j = 0; j < 128; ++j) {
                    float ux = ((float)i + 0.5f) / 128.0f, uy = ((float)j + 0.5f) / 128.0f;
                    // sample_ggx_vndf (bsdf.rs:187-216)
                    float vx = a * wo[0], vy = a * wo[1], vz = wo[2];
                    float il = 1.0f / std::sqrt(((vx * vx) + (vy * vy)) + (vz * vz));
                    vx = vx * il; vy = vy * il; vz = vz * il;
                    float lensq = vx * vx + vy * vy;
                    float t1x = 1.0f, t1y = 0.0f, t1z = 0.0f;
                    if (lensq > 0.0f) {
                        float sl = std::sqrt(lensq);
                        t1x = -vy / sl; t1y = vx / sl; t1z = 0.0f / sl;
                    }
                    float t2x = vy * t1z - t1y * vz, t2y = vz * t1x - t1z * vx, t2z = vx * t1y - t1x * vy;
                    float r = std::sqrt(ux);
                    float phi = 2.0f * PI * uy;
                    float p1 = r * std::cos(phi);
                    float p2 = r * std::sin(phi);
                    float s = 0.5f * (1.0f + vz);
                    p2 = (1.0f - s) * std::sqrt(std::fmax(1.0f - p1 * p1, 0.0f)) + s * p2;
                    float q = std::sqrt(std::fmax(1.0f - p1 * p1 - p2 * p2, 0.0f));
                    float nx = p1 * t1x + p2 * t2x + q * vx, ny = p1 * t1y + p2 * t2y + q * vy,
                          nz = p1 * t1z + p2 * t2z + q * vz;
                    float mx = a * nx, my = a * ny, mz = std::fmax(nz, 0.0f);
                    float im = 1.0f / std::sqrt(((mx * mx) + (my * my)) + (mz * mz));
                    mx = mx * im; my = my * im; mz = mz * im;
                    // reflect (bsdf.rs:699-701) and specular::sample_single (488-511)
                    float dm = ((wo[0] * mx) + (wo[1] * my)) + (wo[2] * mz);
                    float k2 = 2.0f * dm;
                    float wiz = -wo[2] + k2 * mz;
                    if (wiz <= 0.0f) continue;
                    float g1 = 1.0f / (1.0f + lambda(a, mu));
                    float pdf = g1 * ggx(a, mz) / (4.0f * mu);
                    if (pdf <= 0.0f) continue;
                    float g2 = 1.0f / (1.0f + lambda(a, mu) + lambda(a, wiz));
                    float f = 1.0f + (1.0f - 1.0f) * 0.0f;  // white Schlick: F == 1
                    sum += (double)(f * (g2 / g1));
                }
            }
            t[ri * 32 + ci] = (float)(sum / (128.0 * 128.0));
        }
    }
    return t;
}

const std::vector<float>& energy_table_cached() {
    static std::vector<float> t = energy_table_host();
    return t;
}

}  // namespace

extern "C" {

uint32_t luc_layout_version(void) { return LUC_LAYOUT_VERSION; }
uint32_t luc_sizeof(uint32_t which) {
    switch (which) {
        case 0: return sizeof(GpuMaterial);
        case 1: return sizeof(GpuPrimitive);
        case 2: return sizeof(GpuLight);
        case 3: return sizeof(GpuVertexAttr);
        case 4: return sizeof(GpuTriangle);
        case 5: return sizeof(GpuBvhNode);
        case 6: return sizeof(GpuAccum);
        case 7: return sizeof(GpuUniforms);
        case 8: return sizeof(GpuInstance);
    }
    return 0;
}

int32_t luc_create(int32_t device, luc_ctx** out) {
    if (!out) return LUC_ERR_VALIDATION;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return LUC_ERR_NO_DEVICE;
    if (device < 0 || device >= count) return LUC_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return LUC_ERR_NO_DEVICE;
    luc_ctx* c = new luc_ctx();
    c->device = device;
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    c->rs.num_sms = c->num_sms;
    query_occupancy(c->rs);
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return LUC_ERR_NO_DEVICE;
    }
    c->stream = c->own_stream;
    if (const char* b = std::getenv("LUC_PATH_BUDGET")) c->path_budget = std::strtoull(b, nullptr, 10);
    if (const char* g = std::getenv("LUC_NO_GRAPHS")) c->use_graphs = g[0] == '\0' || g[0] == '0';
    if (const char* g = std::getenv("LUC_BINARY_BVH")) c->use_wide = g[0] == '\0' || g[0] == '0';
    if (const char* g = std::getenv("LUC_GUIDE_TC")) c->rs.guide_tc = g[0] != '\0' && g[0] != '0';
    if (const char* w = std::getenv("LUC_WIDE_STAGE")) c->rs.wide_stage = std::atoi(w) == 73 ? 73 : 0;
    if (const char* sp = std::getenv("LUC_SPLIT_ESCAPES")) c->rs.split = sp[0] != '\0' && sp[0] != '0';
    if (const char* ic = std::getenv("LUC_INST_CULL")) c->inst_cull = ic[0] != '\0' && ic[0] != '0';
    const std::vector<float>& et = energy_table_cached();
    if (upload(c->energy, et.data(), et.size(), c->stream) != cudaSuccess ||
        luc_init_sobol_tables(c->stream) != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess) {
        cudaStreamDestroy(c->own_stream);
        delete c;
        return LUC_ERR_OUT_OF_MEMORY;
    }
    *out = c;
    return LUC_OK;
}

void luc_destroy(luc_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    DevBuf* bufs[] = {&c->materials, &c->prims,    &c->lights,   &c->positions, &c->attrs,     &c->tris,
                      &c->nodes,     &c->env_px,   &c->env_cond, &c->env_marg,  &c->env_row_sin, &c->energy,
                      &c->tnodes,    &c->soup,     &c->frame_word, &c->blas_roots, &c->wnodes,  &c->wsoup,
                      &c->wtasks,    &c->wctr,     &c->conv_scratch, &c->wroots, &c->blas_wide, &c->upload_scratch,
                      &c->pool,      &c->accum_tmp, &c->lb_tris, &c->lb_pos,    &c->lb_boxes,  &c->lb_keys,
                      &c->lb_vals,   &c->lb_keys2, &c->lb_vals2, &c->lb_hist,   &c->lb_karras, &c->lb_parent,
                      &c->lb_nbounds, &c->lb_subtree, &c->lb_flags, &c->lb_nodes, &c->lb_rank, &c->lb_misc,
                      &c->lb_icount, &c->lb_look, &c->lb_codes, &c->dn_in,  &c->dn_out,    &c->dn_a,      &c->dn_b,
                      &c->dn_dev,    &c->g_params, &c->g_m,     &c->g_v,       &c->g_grad,    &c->g_wbf,
                      &c->g_bias,    &c->g_misc,   &c->g_lobes, &c->g_rec,     &c->g_io,
                      &c->g_part,    &c->twnodes,  &c->twsoup};
    for (DevBuf* b : bufs) b->release();
    if (c->graph.exec) cudaGraphExecDestroy(c->graph.exec);
    c->graph.timer.release();
    if (c->side_stream) cudaStreamDestroy(c->side_stream);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->ev_ready) cudaEventDestroy(c->ev_ready);
    if (c->ev_done) cudaEventDestroy(c->ev_done);
    if (c->ev_up0) cudaEventDestroy(c->ev_up0);
    if (c->ev_up1) cudaEventDestroy(c->ev_up1);
    cudaStreamDestroy(c->own_stream);
    delete c;
}

const char* luc_last_error(const luc_ctx* c) { return c ? c->err.c_str() : "null context"; }

int32_t luc_set_tlas_leaf(luc_ctx* c, uint32_t max_leaf) {
    if (!c) return LUC_ERR_VALIDATION;
    if (max_leaf < 1 || max_leaf > 64) return luc_fail(c, LUC_ERR_VALIDATION, "tlas leaf size must be 1..64");
    c->tlas_leaf = max_leaf;
    return LUC_OK;
}

int32_t luc_debug_waits(luc_ctx* c, uint32_t mode, uint32_t limit) {
    if (!c) return LUC_ERR_VALIDATION;
    if (mode != LUC_DEBUG_NONE && mode != LUC_DEBUG_SORT_ORPHAN_TILE && mode != LUC_DEBUG_TC_NO_COMMIT)
        return luc_fail(c, LUC_ERR_VALIDATION, "debug waits: unknown mode");
    c->dbg_mode = mode;
    c->dbg_limit = limit;
    return LUC_OK;
}

int32_t luc_set_stream(luc_ctx* c, void* stream) {
    if (!c) return LUC_ERR_VALIDATION;
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return LUC_OK;
}

}  // extern "C"

// Mesh ranges for device-built instancing (luc_upload_meshes); null for a
// plain upload.
struct MeshSpec {
    const uint32_t* first;
    const uint32_t* count;
    uint32_t n;
};

namespace {

// Triangle validation on the device: the smallest index of a triangle whose
// vertex or material index is out of range (0xFFFFFFFF: none).
__global__ void k_validate_tris(const GpuTriangle* __restrict__ t, uint32_t n, uint32_t nv, uint32_t nm,
                                uint32_t* __restrict__ first_bad) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const GpuTriangle g = t[i];
        if (g.i0 >= nv || g.i1 >= nv || g.i2 >= nv || g.material >= nm) atomicMin(first_bad, i);
    }
}

// Vertex bounds on the device (the guide's default position box): min / max
// per axis as order-preserving integer keys (NaN skipped, -0 taken as +0).
__device__ __forceinline__ int float_key(float f) {
    const int b = __float_as_int(f == 0.0f ? 0.0f : f);
    return b >= 0 ? b : b ^ 0x7FFFFFFF;
}
__global__ void k_vertex_bounds(const float4* __restrict__ pos, uint32_t n, int* __restrict__ keys) {
    int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = pos[i];
        const float q[3] = {p.x, p.y, p.z};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (q[a] != q[a]) continue;
            const int k = float_key(q[a]);
            lo[a] = min(lo[a], k);
            hi[a] = max(hi[a], k);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = min(lo[a], __shfl_down_sync(0xFFFFFFFFu, lo[a], o));
            hi[a] = max(hi[a], __shfl_down_sync(0xFFFFFFFFu, hi[a], o));
        }
        if ((threadIdx.x & 31u) == 0) {
            atomicMin(keys + a, lo[a]);
            atomicMax(keys + 3 + a, hi[a]);
        }
    }
}
float key_float(int k) {
    const int b = k >= 0 ? k : k ^ 0x7FFFFFFF;
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

int32_t validate_tris_dev(luc_ctx* c, const GpuTriangle* t, uint32_t n, uint32_t nv, uint32_t nm) {
    if (n == 0) return LUC_OK;
    LUC_CUDA(c, c->upload_scratch.ensure(64), "alloc upload scratch");
    uint32_t* bad = c->upload_scratch.as<uint32_t>();
    LUC_CUDA(c, cudaMemsetAsync(bad, 0xFF, 4, c->stream), "clear validation word");
    k_validate_tris<<<(int)std::min<uint64_t>((n + 255) / 256, (uint64_t)c->num_sms * 8), 256, 0, c->stream>>>(
        t, n, nv, nm, bad);
    uint32_t h = 0;
    LUC_CUDA(c, cudaMemcpyAsync(&h, bad, 4, cudaMemcpyDeviceToHost, c->stream), "read validation word");
    LUC_CUDA(c, cudaStreamSynchronize(c->stream), "validate triangles");
    if (h != 0xFFFFFFFFu) return luc_fail(c, LUC_ERR_VALIDATION, "triangle " + std::to_string(h) + " indexes out of range");
    return LUC_OK;
}

}  // namespace

// The context's second stream (highest priority: a frame's deferred guide
// step must get its blocks ahead of the EXTEND blocks that would otherwise
// fill every SM) and the events that order work across the two streams.
static int32_t ensure_side_stream(luc_ctx* c) {
    if (!c->side_stream) {
        int lo_prio = 0, hi_prio = 0;
        cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
        LUC_CUDA(c, cudaStreamCreateWithPriority(&c->side_stream, cudaStreamNonBlocking, hi_prio), "create side stream");
    }
    for (cudaEvent_t* e : {&c->ev_fork, &c->ev_join, &c->ev_ready, &c->ev_done, &c->ev_up0, &c->ev_up1})
        if (!*e) LUC_CUDA(c, cudaEventCreateWithFlags(e, cudaEventDisableTiming), "create event");
    return LUC_OK;
}

static int32_t upload_scene(luc_ctx* c, const luc_scene_view* v, const MeshSpec* meshes) {
    if (!c || !v) return LUC_ERR_VALIDATION;
    cudaSetDevice(c->device);
    if (v->num_materials == 0 || !v->materials) return luc_fail(c, LUC_ERR_VALIDATION, "scene has no materials");
    if (v->num_primitives && !v->primitives) return luc_fail(c, LUC_ERR_VALIDATION, "null primitives");
    if (v->num_lights && !v->lights) return luc_fail(c, LUC_ERR_VALIDATION, "null lights");
    if (v->num_triangles && (!v->triangles || !v->positions || !v->vertex_attrs || v->num_vertices == 0))
        return luc_fail(c, LUC_ERR_VALIDATION, "triangles without positions/attributes");
    const uint32_t ni = v->num_instances, np_ = v->num_primitives;
    if (ni) {
        // Instanced scene (scene.rs:252-345 layout): instance rows appended
        // after the analytic primitives, BLAS nodes then TLAS nodes, the TLAS
        // from tlas_root on. The tree must come with the scene.
        if (v->num_bvh_nodes == 0 || v->tlas_root >= v->num_bvh_nodes)
            return luc_fail(c, LUC_ERR_VALIDATION, "instanced scene without its BLAS/TLAS nodes or a valid tlas_root");
        for (uint32_t i = 0; i < ni; ++i) {
            const GpuInstance& g = *reinterpret_cast<const GpuInstance*>(v->primitives + np_ + i);
            if (g.kind != PRIM_KIND_INSTANCE || g.blas_root >= v->tlas_root ||
                (g.material != 0xFFFFFFFFu && g.material >= v->num_materials))
                return luc_fail(c, LUC_ERR_VALIDATION, "instance " + std::to_string(i) + " has a bad tag, BLAS root or material");
        }
    }
    for (uint32_t i = 0; i < v->num_primitives; ++i)
        if (v->primitives[i].material >= v->num_materials || v->primitives[i].kind > PRIM_KIND_QUAD)
            return luc_fail(c, LUC_ERR_VALIDATION, "primitive " + std::to_string(i) + " has a bad kind or material");
    for (uint32_t i = 0; i < v->num_lights; ++i)
        if (v->lights[i].material >= v->num_materials)
            return luc_fail(c, LUC_ERR_VALIDATION, "light " + std::to_string(i) + " has a bad material");
    // Triangle indices are validated on the device, right after their upload
    // and before any kernel dereferences them (validate_tris_dev).
    for (uint32_t i = 0; i < v->num_bvh_nodes; ++i) {
        const GpuBvhNode& n = v->bvh_nodes[i];
        const bool tlas = ni && i >= v->tlas_root;
        // Children come after their parent (every builder here and in the
        // reference emits them so), which also rules out cycles; TLAS leaves
        // index instance rows, BLAS leaves triangles.
        bool bad = n.count == 0 ? (n.left_first <= i || (uint64_t)n.left_first + 1 >= v->num_bvh_nodes ||
                                   (ni && !tlas && n.left_first + 1 >= v->tlas_root))
                 : tlas ? (n.left_first < np_ || (uint64_t)n.left_first + n.count > (uint64_t)np_ + ni)
                        : (uint64_t)n.left_first + n.count > v->num_triangles;
        if (bad) return luc_fail(c, LUC_ERR_VALIDATION, "bvh node " + std::to_string(i) + " out of range");
    }
    if (v->env_width && (!v->env_pixels || !v->env_cdf || v->env_height == 0 ||
                         v->env_cdf_width < std::max(v->env_width, v->env_height) + 1))
        return luc_fail(c, LUC_ERR_VALIDATION, "environment map without pixels or a packed CDF");
    // Scene bounds (the guide's default position box): vertices (reduced on
    // the device after their upload, merged in at the end), spheres, quad
    // corners.
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    const bool vertex_bounds = v->num_vertices && v->num_triangles && !ni;
    {
        auto grow = [&](float x, float y, float z) {
            const float q[3] = {x, y, z};
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::min(lo[a], q[a]);
                hi[a] = std::max(hi[a], q[a]);
            }
        };
        if (ni && v->num_triangles) {  // instanced: the TLAS root's box (world space)
            const GpuBvhNode& r = v->bvh_nodes[v->tlas_root];
            grow(r.bounds_min[0], r.bounds_min[1], r.bounds_min[2]);
            grow(r.bounds_max[0], r.bounds_max[1], r.bounds_max[2]);
        }
        for (uint32_t i = 0; i < v->num_primitives; ++i) {
            const GpuPrimitive& p = v->primitives[i];
            const float* o = p.position;
            if (p.kind == PRIM_KIND_QUAD) {
                for (int k = 0; k < 4; ++k) {
                    float su = (k & 1) ? 1.0f : 0.0f, sv = (k & 2) ? 1.0f : 0.0f;
                    grow(o[0] + su * p.edge_u[0] + sv * p.edge_v[0], o[1] + su * p.edge_u[1] + sv * p.edge_v[1],
                         o[2] + su * p.edge_u[2] + sv * p.edge_v[2]);
                }
            } else {
                grow(o[0] - p.radius, o[1] - p.radius, o[2] - p.radius);
                grow(o[0] + p.radius, o[1] + p.radius, o[2] + p.radius);
            }
        }
    }
    cudaStream_t s = c->stream;
    c->has_scene = false;
    // Vertex attributes and the environment go up on the side stream, beside
    // the BVH build (nothing in it reads them), once the context's earlier
    // work is done with the buffers. Every return waits for those copies: the
    // caller may free its arrays once the upload returns.
    if (int32_t rc = ensure_side_stream(c)) return rc;
    const cudaStream_t side = c->side_stream;
    struct SideWait {
        cudaStream_t st;
        ~SideWait() { cudaStreamSynchronize(st); }
    } side_wait{side};
    LUC_CUDA(c, cudaEventRecord(c->ev_up0, s), "order uploads");
    LUC_CUDA(c, cudaStreamWaitEvent(side, c->ev_up0, 0), "order uploads");
    LUC_CUDA(c, upload(c->materials, v->materials, v->num_materials, s), "upload materials");
    LUC_CUDA(c, upload(c->prims, v->primitives, (size_t)np_ + ni, s), "upload primitives");
    std::vector<uint32_t> roots;
    for (uint32_t i = 0; i < ni; ++i) roots.push_back(reinterpret_cast<const GpuInstance*>(v->primitives + np_ + i)->blas_root);
    std::sort(roots.begin(), roots.end());
    roots.erase(std::unique(roots.begin(), roots.end()), roots.end());
    LUC_CUDA(c, upload(c->blas_roots, roots.data(), roots.size(), s), "upload blas roots");
    LUC_CUDA(c, upload(c->lights, v->lights, v->num_lights, s), "upload lights");
    LUC_CUDA(c, upload(c->positions, v->positions, 4 * (size_t)v->num_vertices, s), "upload positions");
    LUC_CUDA(c, upload(c->attrs, v->vertex_attrs, v->num_vertices, side), "upload vertex attrs");
    int bkeys[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
    if (vertex_bounds) {
        LUC_CUDA(c, c->upload_scratch.ensure(64), "alloc upload scratch");
        int* keys = c->upload_scratch.as<int>() + 4;
        LUC_CUDA(c, cudaMemcpyAsync(keys, bkeys, sizeof(bkeys), cudaMemcpyHostToDevice, s), "init bounds");
        k_vertex_bounds<<<(int)std::min<uint64_t>((v->num_vertices + 255) / 256, (uint64_t)c->num_sms * 4), 256, 0,
                          s>>>(c->positions.as<float4>(), v->num_vertices, keys);
        LUC_CUDA(c, cudaMemcpyAsync(bkeys, keys, sizeof(bkeys), cudaMemcpyDeviceToHost, s), "read bounds");
    }
    uint32_t num_nodes = v->num_bvh_nodes;
    c->num_meshes = 0;
    c->needs_instances = false;
    if (meshes) {
        // One BLAS per mesh now; the TLAS comes with luc_set_instances.
        LUC_CUDA(c, upload(c->lb_tris, v->triangles, v->num_triangles, s), "upload triangles");
        if (int32_t rv = validate_tris_dev(c, c->lb_tris.as<GpuTriangle>(), v->num_triangles, v->num_vertices,
                                           v->num_materials))
            return rv;
        int32_t rc = luc_build_blases(c, meshes->first, meshes->count, meshes->n, v->num_triangles, &num_nodes);
        if (rc) return rc;
        c->num_meshes = meshes->n;
        c->blas_nodes = num_nodes;
        c->inst_capacity = 0;
        c->needs_instances = true;
        c->host_prims.assign(v->primitives, v->primitives + np_);
    } else if (v->num_triangles && v->num_bvh_nodes == 0) {
        // No caller tree: build an LBVH on the device and reorder our copy of
        // the triangles into leaf order (Bvh::compact_primitives).
        LUC_CUDA(c, upload(c->lb_tris, v->triangles, v->num_triangles, s), "upload triangles");
        if (int32_t rv = validate_tris_dev(c, c->lb_tris.as<GpuTriangle>(), v->num_triangles, v->num_vertices,
                                           v->num_materials))
            return rv;
        int32_t rc = luc_triangle_boxes_device(c, c->lb_tris.as<GpuTriangle>(), c->positions.as<float4>(),
                                               v->num_triangles);
        if (rc) return rc;
        rc = luc_lbvh_device(c, v->num_triangles, &num_nodes);
        if (rc) return rc;
        LUC_CUDA(c, c->tris.ensure((size_t)v->num_triangles * sizeof(GpuTriangle)), "alloc triangles");
        rc = luc_gather_triangles(c, c->lb_tris.as<GpuTriangle>(), c->tris.as<GpuTriangle>(), c->lb_vals.as<uint32_t>(),
                                  v->num_triangles);
        if (rc) return rc;
        LUC_CUDA(c, c->nodes.ensure((size_t)num_nodes * sizeof(GpuBvhNode)), "alloc nodes");
        LUC_CUDA(c, cudaMemcpyAsync(c->nodes.p, c->lb_nodes.p, (size_t)num_nodes * sizeof(GpuBvhNode),
                                    cudaMemcpyDeviceToDevice, s), "copy nodes");
    } else {
        LUC_CUDA(c, upload(c->tris, v->triangles, v->num_triangles, s), "upload triangles");
        if (int32_t rv = validate_tris_dev(c, c->tris.as<GpuTriangle>(), v->num_triangles, v->num_vertices,
                                           v->num_materials))
            return rv;
        LUC_CUDA(c, upload(c->nodes, v->bvh_nodes, v->num_bvh_nodes, s), "upload bvh nodes");
    }
    // Environment: pixels, the packed CDF split into conditional rows and
    // the marginal, and the per-row sin(theta) the pdf divides by.
    // The rows are copied straight out of the caller's packed array (pitch
    // env_cdf_width floats): no host staging.
    std::vector<float> rsin;
    LUC_CUDA(c, upload(c->env_px, v->env_pixels, 4 * (size_t)v->env_width * v->env_height, side), "upload env");
    if (v->env_width) {
        const uint32_t w = v->env_width, h = v->env_height, cw = v->env_cdf_width;
        LUC_CUDA(c, c->env_cond.ensure((size_t)(w + 1) * h * sizeof(float)), "alloc env cdf");
        LUC_CUDA(c, cudaMemcpy2DAsync(c->env_cond.p, (w + 1) * sizeof(float), v->env_cdf, (size_t)cw * sizeof(float),
                                      (w + 1) * sizeof(float), h, cudaMemcpyHostToDevice, side),
                 "upload env cdf");
        LUC_CUDA(c, upload(c->env_marg, v->env_cdf + (size_t)h * cw, (size_t)h + 1, side), "upload env marginal");
        rsin.resize(h);
        const float PI = 3.14159265358979323846f;
        for (uint32_t j = 0; j < h; ++j) rsin[j] = std::sin(((float)j + 0.5f) / (float)h * PI);
    }
    LUC_CUDA(c, upload(c->env_row_sin, rsin.data(), rsin.size(), side), "upload env rows");
    c->wide_nodes = 0;
    if (v->num_triangles && num_nodes) {
        int32_t rc2 = luc_build_traversal(c, num_nodes, v->num_triangles);
        if (rc2) return rc2;
        if (c->use_wide && !ni && !meshes) {
            rc2 = luc_build_wide(c, num_nodes, v->num_triangles);
            if (rc2) return rc2;
        } else if (c->use_wide) {
            // Two-level scenes: one wide tree per BLAS; instances reach theirs
            // through blas_wide. Device-built TLASes (luc_set_instances) get
            // their own wide tree each frame; a caller's TLAS stays binary.
            const std::vector<uint32_t>& br = meshes ? c->host_mesh_root : roots;
            rc2 = luc_build_wide_roots(c, br.data(), (uint32_t)br.size(), true, num_nodes, v->num_triangles);
            if (rc2) return rc2;
        }
    }
    LUC_CUDA(c, cudaEventRecord(c->ev_up1, side), "join uploads");
    LUC_CUDA(c, cudaStreamWaitEvent(s, c->ev_up1, 0), "join uploads");
    LUC_CUDA(c, cudaStreamSynchronize(s), "scene upload");
    if (vertex_bounds)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], key_float(bkeys[a]));
            hi[a] = std::max(hi[a], key_float(bkeys[3 + a]));
        }
    for (int a = 0; a < 3; ++a) {
        c->scene_lo[a] = lo[a] <= hi[a] ? lo[a] : 0.0f;
        c->scene_hi[a] = lo[a] <= hi[a] ? hi[a] : 1.0f;
    }

    DevScene& d = c->scene;
    d.materials = c->materials.as<GpuMaterial>();
    d.prims = c->prims.as<GpuPrimitive>();
    d.num_prims = v->num_primitives;
    d.lights = c->lights.as<GpuLight>();
    d.num_lights = v->num_lights;
    d.positions = c->positions.as<float4>();
    d.attrs = c->attrs.as<GpuVertexAttr>();
    d.tris = c->tris.as<GpuTriangle>();
    d.num_tris = v->num_triangles;
    d.nodes = c->nodes.as<float4>();
    d.num_nodes = v->num_triangles ? num_nodes : 0;
    d.inst = reinterpret_cast<const GpuInstance*>(c->prims.as<GpuPrimitive>() + np_);
    d.inst_box = nullptr;  // caller-built instancing (SceneBlob layout): no per-instance boxes
    d.twnodes = nullptr;   // nor a wide TLAS
    d.twsoup = nullptr;
    d.num_instances = v->num_triangles ? ni : 0;
    d.tlas_root = v->tlas_root;
    d.blas_roots = c->blas_roots.as<uint32_t>();
    d.num_blas = (uint32_t)roots.size();
    d.reference_shadows = false;
    d.tnodes = c->tnodes.as<float4>();
    d.soup = c->soup.as<float4>();
    d.wnodes = c->wide_nodes ? c->wnodes.as<float4>() : nullptr;
    d.wsoup = c->wide_nodes ? c->wsoup.as<float4>() : nullptr;
    d.num_wnodes = c->wide_nodes;
    d.blas_wide = c->wide_nodes && (ni || meshes) ? c->blas_wide.as<uint32_t>() : nullptr;
    d.root_first = 0;
    d.root_count = 0;
    if (d.num_nodes) {
        GpuBvhNode root;
        LUC_CUDA(c, cudaMemcpy(&root, c->nodes.p, sizeof(root), cudaMemcpyDeviceToHost), "read root");
        if (root.count > 0) {
            d.root_first = root.left_first;
            d.root_count = root.count;
        }
    }
    d.env_px = c->env_px.as<float4>();
    d.env_cond = c->env_cond.as<float>();
    d.env_marg = c->env_marg.as<float>();
    d.env_row_sin = c->env_row_sin.as<float>();
    d.env_w = v->env_width;
    d.env_h = v->env_width ? v->env_height : 0;
    d.env_total = v->env_total_weight;
    d.energy = c->energy.as<float>();
    d.has_env = v->env_width > 0 && v->env_total_weight > 0.0f;  // EnvMap::is_empty
    d.light_strategies = v->num_lights + (d.has_env ? 1u : 0u);
    c->num_materials = v->num_materials;
    c->total_nodes = num_nodes;
    c->has_scene = true;
    return LUC_OK;
}

extern "C" {

int32_t luc_upload_scene(luc_ctx* c, const luc_scene_view* v) { return upload_scene(c, v, nullptr); }

int32_t luc_upload_meshes(luc_ctx* c, const luc_scene_view* v, const uint32_t* mesh_first, const uint32_t* mesh_count,
                          uint32_t num_meshes) {
    if (!c || !v || !mesh_first || !mesh_count || num_meshes == 0) return LUC_ERR_VALIDATION;
    if (v->num_instances || v->num_bvh_nodes)
        return luc_fail(c, LUC_ERR_VALIDATION, "luc_upload_meshes takes no instances and no tree");
    if (v->num_triangles == 0) return luc_fail(c, LUC_ERR_VALIDATION, "luc_upload_meshes needs triangles");
    uint64_t end = 0;
    for (uint32_t m = 0; m < num_meshes; ++m) {
        if (mesh_count[m] == 0 || mesh_first[m] < end || (uint64_t)mesh_first[m] + mesh_count[m] > v->num_triangles)
            return luc_fail(c, LUC_ERR_VALIDATION,
                            "mesh " + std::to_string(m) + ": ranges must be non-empty, ascending, disjoint and inside the triangles");
        end = (uint64_t)mesh_first[m] + mesh_count[m];
    }
    MeshSpec ms{mesh_first, mesh_count, num_meshes};
    return upload_scene(c, v, &ms);
}

}  // extern "C"

int32_t ensure_pool(luc_ctx* c, uint64_t paths, uint32_t max_depth) {
    RenderState& rs = c->rs;
    uint32_t ctrs = kCtrStride * (max_depth + 2);
    if (paths <= rs.capacity && ctrs <= rs.ctr_capacity) return LUC_OK;
    paths = std::max(paths, rs.capacity);
    ctrs = std::max(ctrs, rs.ctr_capacity);
    const size_t f4 = sizeof(float4);
    size_t bytes = paths * (11 * f4 + 8 * sizeof(uint32_t)) + ctrs * sizeof(uint32_t) + 20 * 256;
    LUC_CUDA(c, c->pool.ensure(bytes), "allocate path pool");
    char* p = (char*)c->pool.p;
    auto take = [&](size_t n) {
        char* r = p;
        p += (n + 255) & ~size_t(255);
        return r;
    };
    PathState& ps = rs.ps;
    ps.o_pdf = (float4*)take(paths * f4);
    ps.dir = (float4*)take(paths * f4);
    ps.thr = (float4*)take(paths * f4);
    ps.rad = (float4*)take(paths * f4);
    ps.prev = (float4*)take(paths * f4);
    ps.hit = (float4*)take(paths * f4);
    ps.galb = (float4*)take(paths * f4);
    ps.gnrm = (float4*)take(paths * f4);
    ps.sh_o = (float4*)take(paths * f4);
    ps.sh_d = (float4*)take(paths * f4);
    ps.sh_c = (float4*)take(paths * f4);
    ps.queue[0] = (uint32_t*)take(paths * 4);
    ps.queue[1] = (uint32_t*)take(paths * 4);
    ps.hinst = (uint32_t*)take(paths * 4);
    for (int k = 0; k < 3; ++k) ps.hitq[k] = (uint32_t*)take(paths * 4);
    ps.missq = (uint32_t*)take(paths * 4);
    ps.seg = (uint32_t*)take(paths * 4);
    ps.ctr = (uint32_t*)take(ctrs * 4);
    ps.stat = (unsigned long long*)take(8 * sizeof(unsigned long long));
    if ((size_t)(p - (char*)c->pool.p) > c->pool.bytes) return luc_fail(c, LUC_ERR_VALIDATION, "path pool carve");
    rs.capacity = paths;
    rs.ctr_capacity = ctrs;
    return LUC_OK;
}

extern "C" {

int32_t luc_render(luc_ctx* c, const GpuUniforms* u, uint32_t spp, uint32_t max_depth, uint32_t flags,
                   GpuAccum* out_host, void* out_dev) {
    if (!c || !u) return LUC_ERR_VALIDATION;
    cudaSetDevice(c->device);
    if (!c->has_scene) return luc_fail(c, LUC_ERR_VALIDATION, "no scene uploaded");
    if (c->needs_instances) return luc_fail(c, LUC_ERR_VALIDATION, "meshes uploaded but no instances set (luc_set_instances)");
    if (u->width == 0 || u->height == 0) return luc_fail(c, LUC_ERR_VALIDATION, "zero-sized image");
    if (spp == 0) return luc_fail(c, LUC_ERR_VALIDATION, "spp must be positive");
    if (max_depth == 0 || max_depth > 256) return luc_fail(c, LUC_ERR_VALIDATION, "max_depth must be in 1..=256");
    if ((out_host == nullptr) == (out_dev == nullptr))
        return luc_fail(c, LUC_ERR_VALIDATION, "exactly one of out_host / out_dev must be given");
    const uint32_t arch = flags & 0xFFu;
    if (arch != LUC_ARCH_WAVEFRONT && arch != LUC_ARCH_MEGAKERNEL)
        return luc_fail(c, LUC_ERR_VALIDATION, "unknown architecture");
    if (flags & ~(0xFFu | LUC_FLAG_NO_GUIDES | LUC_FLAG_PROFILE | LUC_FLAG_GUIDED | LUC_FLAG_REFERENCE_SHADOWS |
                  LUC_FLAG_MEASURE))
        return luc_fail(c, LUC_ERR_VALIDATION, "unknown render flag");
    const bool guided = (flags & LUC_FLAG_GUIDED) != 0;
    const bool mega = arch == LUC_ARCH_MEGAKERNEL;
    if (mega && guided) return luc_fail(c, LUC_ERR_VALIDATION, "the megakernel does not sample the learned guide");
    if (guided && !c->guide_ready)
        return luc_fail(c, LUC_ERR_VALIDATION, "LUC_FLAG_GUIDED needs luc_guide_init first");
    if (u->sampling_mode > 2 || u->sampler_kind > 1) return luc_fail(c, LUC_ERR_VALIDATION, "bad sampling mode");
    const uint64_t pixels = (uint64_t)u->width * u->height;
    if (pixels > 0xFFFFFFFFull) return luc_fail(c, LUC_ERR_VALIDATION, "image too large");
    cudaStream_t s = c->stream;

    GpuAccum* accum = (GpuAccum*)out_dev;
    if (out_host) {
        LUC_CUDA(c, c->accum_tmp.ensure(pixels * sizeof(GpuAccum)), "allocate accumulator");
        accum = c->accum_tmp.as<GpuAccum>();
        LUC_CUDA(c, cudaMemsetAsync(accum, 0, pixels * sizeof(GpuAccum), s), "clear accumulator");
    }
    uint64_t per_batch = std::max<uint64_t>(1, std::min<uint64_t>(spp, c->path_budget / pixels));
    int32_t rc = ensure_pool(c, per_batch * pixels, max_depth);
    if (rc) return rc;
    if (guided) {
        rc = luc_guide_prepare_frame(c, c->rs.capacity);
        if (rc) return rc;
        c->rs.ps.lobes = c->g_lobes.as<float4>();
        c->rs.ps.lobe_stride = c->rs.capacity;
        c->rs.ps.rec = c->g_rec.as<float4>();
        c->rs.ps.gmisc = c->g_misc.as<uint32_t>();
    }
    GuideTrain gt = guided ? luc_guide_train_state(c) : GuideTrain{};
    // A guided, trained, single-batch graph frame leaves its gradient step
    // to the start of the next guided frame, where it runs beside GENERATE
    // and the first EXTEND (which read neither the records nor the guide);
    // every other render, and every guide call, runs a pending step first.
    const bool one_batch = per_batch >= spp;
    const bool defer = guided && gt.train && c->guide_rec_cap && one_batch && c->use_graphs && !mega &&
                       !(flags & LUC_FLAG_PROFILE);
    if (!defer || !c->guide_pending)
        if (int32_t rc2 = luc_guide_flush(c)) return rc2;
    const bool pending = defer && c->guide_pending;
    gt.defer = defer;

    LUC_CUDA(c, c->frame_word.ensure(256), "allocate frame word");
    FrameParams fp{};
    fp.sbase = c->frame_word.as<uint32_t>();
    fp.pixels = (uint32_t)pixels;
    fp.width = u->width;
    fp.height = u->height;
    fp.frame_seed = u->frame_seed;
    fp.sampler_kind = u->sampler_kind;
    fp.sampling = u->sampling_mode;
    fp.max_depth = max_depth;
    fp.guides = (flags & LUC_FLAG_NO_GUIDES) ? 0u : 1u;
    fp.split = c->rs.split ? 1u : 0u;
    if (guided) {
        fp.guided = 1u;
        fp.rec_cap = c->guide_train ? c->guide_rec_cap : 0u;
        fp.guide = luc_guide_dev(c);
    }
    fp.lens_radius = u->lens_radius;
    fp.cam_origin = ld3(u->cam_origin);
    fp.cam_upper_left = ld3(u->cam_upper_left);
    fp.cam_horizontal = ld3(u->cam_horizontal);
    fp.cam_vertical = ld3(u->cam_vertical);
    DevScene sc = c->scene;
    sc.background = ld3(u->background);
    sc.reference_shadows = (flags & LUC_FLAG_REFERENCE_SHADOWS) != 0;

    c->stats = luc_render_stats{};
    c->rs.launches = 0;
    StageTimer timer;
    StageTimer* tp = (flags & LUC_FLAG_PROFILE) ? &timer : nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaMemsetAsync(c->rs.ps.stat, 0, 8 * sizeof(unsigned long long), s);
    cudaEventRecord(e0, s);
    if (mega) {
        // Batches of whole samples through the same pool as the wavefront:
        // one launch walks every path of the batch, then RESOLVE.
        for (uint32_t done = 0; done < spp;) {
            uint32_t n = (uint32_t)std::min<uint64_t>(per_batch, spp - done);
            fp.sample_base = u->sample_offset + done;
            LUC_CUDA(c, cudaMemcpyAsync(c->frame_word.p, &fp.sample_base, 4, cudaMemcpyHostToDevice, s),
                     "upload sample base");
            fp.batch_samples = n;
            fp.num_paths = (uint64_t)n * pixels;
            record_megakernel(c->rs, sc, fp, accum, s);
            c->rs.launches += 2;
            done += n;
            c->stats.paths += fp.num_paths;
        }
    } else if (one_batch && c->use_graphs) {
        // Single-batch frame: capture it once as a CUDA graph and replay it
        // while the frame parameters, scene, pool and accumulator repeat.
        // The sample offset reaches the kernels through the frame word, so
        // the graph (keyed on everything else) replays across offsets.
        fp.sample_base = 0;
        const uint32_t sbase = u->sample_offset;
        LUC_CUDA(c, cudaMemcpyAsync(c->frame_word.p, &sbase, 4, cudaMemcpyHostToDevice, s), "upload sample base");
        fp.batch_samples = spp;
        fp.num_paths = (uint64_t)spp * pixels;
        uint32_t lr_bits = 0;
        std::memcpy(&lr_bits, &gt.lr, 4);
        // The scene enters the key through the DevScene bytes (pointers,
        // counts, roots): the kernels read the arrays at run time, so a
        // re-upload into the same buffers replays the graph unchanged.
        const uint64_t extra[10] = {(uint64_t)(uintptr_t)accum,        (uint64_t)pending | (uint64_t)defer << 1,
                                    (uint64_t)(uintptr_t)c->rs.ps.o_pdf, (uint64_t)(tp != nullptr),
                                    (uint64_t)(uintptr_t)c->rs.ps.lobes, (uint64_t)(uintptr_t)c->rs.ps.rec,
                                    (uint64_t)(uintptr_t)c->rs.ps.gmisc, (uint64_t)(uintptr_t)gt.params,
                                    (uint64_t)gt.train,                  (uint64_t)lr_bits};
        std::vector<unsigned char> key(sizeof(FrameParams) + sizeof(DevScene) + sizeof(extra));
        std::memcpy(key.data(), &fp, sizeof(FrameParams));
        std::memcpy(key.data() + sizeof(FrameParams), &sc, sizeof(DevScene));
        std::memcpy(key.data() + sizeof(FrameParams) + sizeof(DevScene), extra, sizeof(extra));
        FrameGraph& g = c->graph;
        if (g.exec == nullptr || g.key != key) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
            g.timer.release();
            cudaGraph_t graph = nullptr;
            uint64_t before = c->rs.launches;
            // Unprofiled frames run each CONNECT on the side stream, beside
            // the next EXTEND (stage timers need the stages in sequence).
            const bool overlap = tp == nullptr;
            if (pending || overlap)
                if (int32_t rc2 = ensure_side_stream(c)) return rc2;
            const ConnectOverlap ov{c->side_stream, c->ev_ready, c->ev_done};
            LUC_CUDA(c, cudaStreamBeginCapture(c->own_stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            GuideTrain gcap = gt;
            if (pending) {
                // Fork: the previous frame's step on the side stream.
                cudaEventRecord(c->ev_fork, c->own_stream);
                cudaStreamWaitEvent(c->side_stream, c->ev_fork, 0);
                launch_guide_step(c->rs, c->guide_pending_cap, luc_guide_dev(c), gt, c->side_stream);
                cudaEventRecord(c->ev_join, c->side_stream);
                gcap.join = c->ev_join;
                c->rs.launches += 3;
            }
            record_batch(c->rs, sc, fp, accum, c->own_stream, tp ? &g.timer : nullptr, &gcap, overlap ? &ov : nullptr);
            LUC_CUDA(c, cudaStreamEndCapture(c->own_stream, &graph), "end capture");
            cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ie != cudaSuccess) {
                g.exec = nullptr;
                return luc_cuda_fail(c, ie, "instantiate frame graph");
            }
            g.launches = c->rs.launches - before;
            c->rs.launches = before;
            g.key = key;
            g.profiled = tp != nullptr;
        }
        LUC_CUDA(c, cudaGraphLaunch(g.exec, s), "launch frame graph");
        c->rs.launches += g.launches;
        c->stats.paths += fp.num_paths;
        if (defer) {
            c->guide_pending = true;
            c->guide_pending_cap = fp.rec_cap;
        }
    } else {
        for (uint32_t done = 0; done < spp;) {
            uint32_t n = (uint32_t)std::min<uint64_t>(per_batch, spp - done);
            fp.sample_base = u->sample_offset + done;
            LUC_CUDA(c, cudaMemcpyAsync(c->frame_word.p, &fp.sample_base, 4, cudaMemcpyHostToDevice, s),
                     "upload sample base");
            fp.batch_samples = n;
            fp.num_paths = (uint64_t)n * pixels;
            record_batch(c->rs, sc, fp, accum, s, tp, &gt);
            done += n;
            c->stats.paths += fp.num_paths;
        }
    }
    cudaEventRecord(e1, s);
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return luc_cuda_fail(c, le, "render launch");
    float conv = -1.0f;
    const bool measure = (flags & LUC_FLAG_MEASURE) != 0;
    if (measure) {
        rc = luc_record_convergence(c, accum, (uint32_t)pixels, s);
        if (rc) return rc;
        LUC_CUDA(c, cudaMemcpyAsync(&conv, c->conv_scratch.as<float2>() + 64, 4, cudaMemcpyDeviceToHost, s),
                 "read convergence");
    }
    if (out_host) {
        LUC_CUDA(c, cudaMemcpyAsync(out_host, accum, pixels * sizeof(GpuAccum), cudaMemcpyDeviceToHost, s),
                 "read back accumulator");
    }
    unsigned long long counts[8] = {0};
    LUC_CUDA(c, cudaMemcpyAsync(counts, c->rs.ps.stat, sizeof(counts), cudaMemcpyDeviceToHost, s), "read counters");
    cudaError_t se = cudaStreamSynchronize(s);
    if (se != cudaSuccess) {
        int32_t code = out_host ? LUC_ERR_READBACK : LUC_ERR_LAUNCH;
        return luc_fail(c, code, std::string("render: ") + cudaGetErrorString(se));
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->stats.ms_total = ms;
    c->stats.convergence = measure ? conv : -1.0;
    c->stats.launches = c->rs.launches;
    c->stats.rays_extend = counts[0];
    c->stats.nodes_extend = counts[1];
    c->stats.tris_extend = counts[2];
    c->stats.rays_shadow = counts[3];
    c->stats.nodes_shadow = counts[4];
    c->stats.tris_shadow = counts[5];
    c->stats.blas_extend = counts[6];
    c->stats.blas_shadow = counts[7];
    if (tp) {
        double st[StageTimer::kCount] = {0};
        if (one_batch && c->use_graphs) c->graph.timer.accumulate(st);
        else tp->collect(st);
        c->stats.ms_generate = st[StageTimer::kGenerate];
        c->stats.ms_extend = st[StageTimer::kExtend];
        c->stats.ms_shade = st[StageTimer::kShade];
        c->stats.ms_connect = st[StageTimer::kConnect];
        c->stats.ms_resolve = st[StageTimer::kResolve];
        c->stats.ms_guide = st[StageTimer::kGuide];
        c->stats.ms_train = st[StageTimer::kTrain];
    }
    return LUC_OK;
}

int32_t luc_get_stats(const luc_ctx* c, luc_render_stats* out) {
    if (!c || !out) return LUC_ERR_VALIDATION;
    *out = c->stats;
    return LUC_OK;
}

}  // extern "C"

// Camera::write_uniforms + integrator::build_uniforms (crates/core/src/
// camera.rs:344-365, integrator.rs:153-178) for callers that hold a camera
// rather than baked uniforms. f32 throughout, glibc tanf, no contraction.
extern "C" int32_t luc_camera_uniforms(const float* eye, const float* look_at, const float* up, float vfov_deg,
                                       float aperture, float focus_distance, uint32_t width, uint32_t height,
                                       GpuUniforms* out) {
    if (!eye || !look_at || !up || !out || width == 0 || height == 0) return LUC_ERR_VALIDATION;
    auto sub = [](const float* a, const float* b, float* o) { o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2]; };
    auto dotf = [](const float* a, const float* b) { return ((a[0] * b[0]) + (a[1] * b[1])) + (a[2] * b[2]); };
    auto crossf = [](const float* a, const float* b, float* o) {
        o[0] = a[1] * b[2] - b[1] * a[2];
        o[1] = a[2] * b[0] - b[2] * a[0];
        o[2] = a[0] * b[1] - b[0] * a[1];
    };
    auto norm = [&](float* a) {
        float r = 1.0f / std::sqrt(dotf(a, a));
        a[0] = a[0] * r; a[1] = a[1] * r; a[2] = a[2] * r;
    };
    float fwd[3], right[3], upv[3], down[3];
    sub(look_at, eye, fwd);
    norm(fwd);
    crossf(fwd, up, right);
    norm(right);
    crossf(right, fwd, upv);
    down[0] = -upv[0]; down[1] = -upv[1]; down[2] = -upv[2];
    const float PI = 3.14159265358979323846f;
    float aspect = (float)width / (float)height;
    float half_h = std::tan(vfov_deg * (PI / 180.0f) * 0.5f) * focus_distance;
    float half_w = half_h * aspect;
    std::memset(out, 0, sizeof(GpuUniforms));
    for (int k = 0; k < 3; ++k) {
        out->cam_origin[k] = eye[k];
        out->cam_horizontal[k] = right[k] * (2.0f * half_w);
        out->cam_vertical[k] = down[k] * (2.0f * half_h);
        out->cam_upper_left[k] = ((eye[k] + fwd[k] * focus_distance) - right[k] * half_w) - down[k] * half_h;
    }
    out->lens_radius = aperture * 0.5f;
    out->focus_distance = focus_distance;
    out->width = width;
    out->height = height;
    return LUC_OK;
}
