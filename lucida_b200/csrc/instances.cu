// Device-built instancing for animated two-level scenes: one LBVH per mesh
// (the BLASes, built once by luc_upload_meshes) and a TLAS rebuilt by LBVH
// over the instances' world bounds every time the placements change
// (luc_set_instances), with no host-side tree work. The reference builds
// both levels once on the CPU with binned SAH (crates/core/src/scene.rs:
// 252-345); the node layout produced here is the same flattened form
// (every BLAS, then the TLAS; instance rows appended to the primitives in
// TLAS-leaf order), so the traversal and shading code serve both.
//
// Per instance the device inverts the caller's object-to-world transform by
// the adjugate (each entry its cofactor / det, IEEE division, no FMA) and
// takes the world bounds as the eight corners of the BLAS box through the
// inverse of that inverse, padded as Aabb::pad does (instance.rs:98-113), so
// the oracle reproduces every bit.
#include <algorithm>
#include <cmath>
#include <string>
#include "ctx.cuh"

namespace luc {

struct Aff {
    float m[3][4];
};

__device__ __forceinline__ Aff aff_inverse(const Aff& a) {
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
    const float c[3][3] = {{c00, c01, c02}, {c10, c11, c12}, {c20, c21, c22}};
    Aff r;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) r.m[i][j] = c[i][j] / det;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        r.m[i][3] = -((r.m[i][0] * m[0][3] + r.m[i][1] * m[1][3]) + r.m[i][2] * m[2][3]);
    return r;
}

__device__ __forceinline__ void aff_point(const Aff& a, float x, float y, float z, float (&o)[3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i) o[i] = ((a.m[i][0] * x + a.m[i][1] * y) + a.m[i][2] * z) + a.m[i][3];
}

// Per instance: the packed world-to-object row set and the padded world box
// (6 floats) for the TLAS build. Meshes and materials were validated on the
// host.
__global__ void k_instances_prepare(const float* __restrict__ o2w, const uint32_t* __restrict__ mesh,
                                    const uint32_t* __restrict__ material, uint32_t n,
                                    const uint32_t* __restrict__ mesh_root, const float* __restrict__ mesh_bounds,
                                    GpuInstance* __restrict__ rows, float* __restrict__ boxes) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Aff f;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int k = 0; k < 4; ++k) f.m[r][k] = o2w[12 * (size_t)i + 4 * r + k];
        const Aff w = aff_inverse(f);
        const uint32_t me = mesh[i];
        GpuInstance g;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            g.inv_row0[j] = w.m[0][j];
            g.inv_row1[j] = w.m[1][j];
            g.inv_row2[j] = w.m[2][j];
            g.inv_translation[j] = w.m[j][3];
        }
        g.blas_root = mesh_root[me];
        g.kind = PRIM_KIND_INSTANCE;
        g.material = material[i];
        g._pad0 = 0.0f;
        rows[i] = g;
        // Instance::world_bounds: the forward transform recovered from the
        // stored inverse, all eight corners, then Aabb::pad.
        const Aff tw = aff_inverse(w);
        const float* b = mesh_bounds + 6 * (size_t)me;
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int c = 0; c < 8; ++c) {
            float p[3];
            aff_point(tw, (c & 1) ? b[3] : b[0], (c & 2) ? b[4] : b[1], (c & 4) ? b[5] : b[2], p);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                lo[k] = fminf(lo[k], p[k]);
                hi[k] = fmaxf(hi[k], p[k]);
            }
        }
        float* o = boxes + 6 * (size_t)i;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float pad = 1.0e-6f * (1.0f + fmaxf(fabsf(lo[k]), fabsf(hi[k])));
            o[k] = lo[k] - pad;
            o[3 + k] = hi[k] + pad;
        }
    }
}

// Copy LBVH nodes into the shared array: internal children += node_offset,
// leaves += leaf_offset (a triangle range for a BLAS, the first instance row
// for the TLAS).
__global__ void k_rebase_nodes(const float4* __restrict__ src, uint32_t n, uint32_t node_offset, uint32_t leaf_offset,
                               float4* __restrict__ dst) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 a = src[2 * i], b = src[2 * i + 1];
        uint32_t lf = __float_as_uint(a.w), count = __float_as_uint(b.w);
        a.w = __uint_as_float(lf + (count ? leaf_offset : node_offset));
        dst[2 * i] = a;
        dst[2 * i + 1] = b;
    }
}

__global__ void k_gather_instances(const GpuInstance* __restrict__ src, const uint32_t* __restrict__ order, uint32_t n,
                                   GpuInstance* __restrict__ dst) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[order[i]];
}
// The instances' padded world boxes (the TLAS build's inputs) in TLAS-leaf
// order, lo and hi as two float4 per instance.
__global__ void k_gather_boxes(const float* __restrict__ boxes6, const uint32_t* __restrict__ order, uint32_t n,
                               float4* __restrict__ dst) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* b = boxes6 + 6 * (size_t)order[i];
        dst[2 * (size_t)i] = make_float4(b[0], b[1], b[2], 0.0f);
        dst[2 * (size_t)i + 1] = make_float4(b[3], b[4], b[5], 0.0f);
    }
}

// Object-space bounds of one mesh: the root of its freshly built LBVH.
__global__ void k_mesh_bounds(const float4* __restrict__ root, float* __restrict__ out6) {
    float4 a = root[0], b = root[1];
    out6[0] = a.x;
    out6[1] = a.y;
    out6[2] = a.z;
    out6[3] = b.x;
    out6[4] = b.y;
    out6[5] = b.z;
}

static int grid_n(uint64_t n, int sms) { return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 8)); }

}  // namespace luc

using namespace luc;

// Reallocate `b` to at least `bytes`, keeping its first `keep` bytes.
static cudaError_t grow_keep(luc_ctx* c, DevBuf& b, size_t bytes, size_t keep) {
    if (b.p && b.bytes >= bytes) return cudaSuccess;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) return e;
    if (b.p && keep) e = cudaMemcpyAsync(p, b.p, std::min(keep, b.bytes), cudaMemcpyDeviceToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (b.p) cudaFree(b.p);
    b.p = p;
    b.bytes = bytes;
    return e;
}

// One LBVH per mesh range over the uploaded object-space triangles (in
// lb_tris): nodes rebased into c->nodes (children absolute, leaves absolute
// triangle indices), each range's triangles gathered into leaf order in
// c->tris, per-mesh root and bounds recorded. Returns the BLAS node total.
int32_t luc_build_blases(luc_ctx* c, const uint32_t* first, const uint32_t* count, uint32_t nm, uint32_t ntris,
                         uint32_t* blas_nodes) {
    cudaStream_t s = c->stream;
    uint64_t cap = 0;
    for (uint32_t m = 0; m < nm; ++m) cap += 2ull * count[m];
    LUC_CUDA(c, c->nodes.ensure(cap * sizeof(GpuBvhNode)), "alloc blas nodes");
    LUC_CUDA(c, c->tris.ensure((size_t)ntris * sizeof(GpuTriangle)), "alloc triangles");
    LUC_CUDA(c, c->mesh_bounds.ensure((size_t)nm * 24), "alloc mesh bounds");
    c->host_mesh_root.assign(nm, 0u);
    uint32_t off = 0;
    for (uint32_t m = 0; m < nm; ++m) {
        const GpuTriangle* src = c->lb_tris.as<GpuTriangle>() + first[m];
        int32_t rc = luc_triangle_boxes_device(c, src, c->positions.as<float4>(), count[m]);
        if (rc) return rc;
        uint32_t nn = 0;
        rc = luc_lbvh_device(c, count[m], &nn);
        if (rc) return rc;
        k_rebase_nodes<<<grid_n(nn, c->num_sms), 256, 0, s>>>(c->lb_nodes.as<float4>(), nn, off, first[m],
                                                             c->nodes.as<float4>() + 2 * (size_t)off);
        rc = luc_gather_triangles(c, src, c->tris.as<GpuTriangle>() + first[m], c->lb_vals.as<uint32_t>(), count[m]);
        if (rc) return rc;
        k_mesh_bounds<<<1, 1, 0, s>>>(c->lb_nodes.as<float4>(), c->mesh_bounds.as<float>() + 6 * (size_t)m);
        c->host_mesh_root[m] = off;
        off += nn;
        // lb_nodes / lb_vals are reused by the next mesh's build.
        LUC_CUDA(c, cudaStreamSynchronize(s), "blas build");
    }
    LUC_CUDA(c, upload(c->mesh_root, c->host_mesh_root.data(), nm, s), "upload mesh roots");
    LUC_CUDA(c, cudaGetLastError(), "blas build");
    *blas_nodes = off;
    return LUC_OK;
}

extern "C" {

int32_t luc_set_instances(luc_ctx* c, const float* object_to_world, const uint32_t* mesh, const uint32_t* material,
                          uint32_t n) {
    if (!c || (n && (!object_to_world || !mesh || !material))) return LUC_ERR_VALIDATION;
    if (c->num_meshes == 0) return luc_fail(c, LUC_ERR_VALIDATION, "no meshes uploaded (luc_upload_meshes)");
    if (n == 0) return luc_fail(c, LUC_ERR_VALIDATION, "at least one instance is needed");
    if (n > (1u << 24)) return luc_fail(c, LUC_ERR_VALIDATION, "at most 2^24 instances");
    for (uint32_t i = 0; i < n; ++i) {
        if (mesh[i] >= c->num_meshes) return luc_fail(c, LUC_ERR_VALIDATION, "instance " + std::to_string(i) + ": bad mesh");
        if (material[i] != 0xFFFFFFFFu && material[i] >= c->num_materials)
            return luc_fail(c, LUC_ERR_VALIDATION, "instance " + std::to_string(i) + ": bad material");
        const float* m = object_to_world + 12 * (size_t)i;
        for (int k = 0; k < 12; ++k)
            if (!std::isfinite(m[k])) return luc_fail(c, LUC_ERR_VALIDATION, "instance " + std::to_string(i) + ": non-finite transform");
        double det = (double)m[0] * ((double)m[5] * m[10] - (double)m[6] * m[9]) -
                     (double)m[1] * ((double)m[4] * m[10] - (double)m[6] * m[8]) +
                     (double)m[2] * ((double)m[4] * m[9] - (double)m[5] * m[8]);
        if (!(std::fabs(det) > 1e-20)) return luc_fail(c, LUC_ERR_VALIDATION, "instance " + std::to_string(i) + ": singular transform");
    }
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    const uint32_t np_ = (uint32_t)c->host_prims.size();
    const uint32_t bn = c->blas_nodes;
    if (n > c->inst_capacity) {
        // Room for the instance rows after the analytic primitives and for the
        // largest TLAS (2n - 1 nodes) after the BLASes; BLAS contents kept.
        LUC_CUDA(c, grow_keep(c, c->nodes, ((size_t)bn + 2 * n) * sizeof(GpuBvhNode), (size_t)bn * sizeof(GpuBvhNode)),
                 "grow nodes");
        LUC_CUDA(c, grow_keep(c, c->tnodes, ((size_t)bn + 2 * n) * 64, (size_t)bn * 64), "grow traversal nodes");
        LUC_CUDA(c, c->prims.ensure(((size_t)np_ + n) * sizeof(GpuPrimitive)), "grow primitives");
        LUC_CUDA(c, cudaMemcpyAsync(c->prims.p, c->host_prims.data(), (size_t)np_ * sizeof(GpuPrimitive),
                                    cudaMemcpyHostToDevice, s), "upload primitives");
        LUC_CUDA(c, c->inst_box.ensure((size_t)n * 2 * sizeof(float4)), "grow instance boxes");
        c->inst_capacity = n;  // moved arrays change the DevScene bytes, which key the frame graph
    }
    LUC_CUDA(c, c->inst_in.ensure((size_t)n * 56), "alloc instance input");
    float* d_o2w = c->inst_in.as<float>();
    uint32_t* d_mesh = reinterpret_cast<uint32_t*>(d_o2w + 12 * (size_t)n);
    uint32_t* d_mat = d_mesh + n;
    LUC_CUDA(c, cudaMemcpyAsync(d_o2w, object_to_world, (size_t)n * 48, cudaMemcpyHostToDevice, s), "upload transforms");
    LUC_CUDA(c, cudaMemcpyAsync(d_mesh, mesh, (size_t)n * 4, cudaMemcpyHostToDevice, s), "upload meshes");
    LUC_CUDA(c, cudaMemcpyAsync(d_mat, material, (size_t)n * 4, cudaMemcpyHostToDevice, s), "upload materials");
    LUC_CUDA(c, c->inst_tmp.ensure((size_t)n * sizeof(GpuInstance)), "alloc instance rows");
    LUC_CUDA(c, c->lb_boxes.ensure((size_t)n * 24), "alloc instance boxes");
    k_instances_prepare<<<grid_n(n, c->num_sms), 256, 0, s>>>(d_o2w, d_mesh, d_mat, n, c->mesh_root.as<uint32_t>(),
                                                             c->mesh_bounds.as<float>(), c->inst_tmp.as<GpuInstance>(),
                                                             c->lb_boxes.as<float>());
    LUC_CUDA(c, cudaGetLastError(), "prepare instances");
    uint32_t tn = 0;
    int32_t rc = luc_lbvh_device(c, n, &tn, c->tlas_leaf);
    if (rc) return rc;
    k_rebase_nodes<<<grid_n(tn, c->num_sms), 256, 0, s>>>(c->lb_nodes.as<float4>(), tn, bn, np_,
                                                         c->nodes.as<float4>() + 2 * (size_t)bn);
    k_gather_instances<<<grid_n(n, c->num_sms), 256, 0, s>>>(c->inst_tmp.as<GpuInstance>(), c->lb_vals.as<uint32_t>(), n,
                                                            reinterpret_cast<GpuInstance*>(c->prims.as<GpuPrimitive>() + np_));
    k_gather_boxes<<<grid_n(n, c->num_sms), 256, 0, s>>>(c->lb_boxes.as<float>(), c->lb_vals.as<uint32_t>(), n,
                                                        c->inst_box.as<float4>());
    LUC_CUDA(c, cudaGetLastError(), "tlas");
    rc = luc_build_tnodes_range(c, bn, bn + tn);
    if (rc) return rc;
    bool wide_tlas = false;
    if (c->wide_nodes) {
        rc = luc_build_wide_tlas(c, bn, bn + tn, np_ + n, n, &wide_tlas);
        if (rc) return rc;
    }
    GpuBvhNode root;
    LUC_CUDA(c, cudaMemcpyAsync(&root, c->nodes.as<GpuBvhNode>() + bn, sizeof(root), cudaMemcpyDeviceToHost, s), "read tlas root");
    LUC_CUDA(c, cudaStreamSynchronize(s), "set instances");
    // Scene bounds (the guide's default box): the TLAS root's world box and
    // the analytic primitives.
    for (int a = 0; a < 3; ++a) {
        c->scene_lo[a] = root.bounds_min[a];
        c->scene_hi[a] = root.bounds_max[a];
    }
    for (const GpuPrimitive& p : c->host_prims) {
        for (int a = 0; a < 3; ++a) {
            float lo = p.position[a], hi = p.position[a];
            if (p.kind == PRIM_KIND_QUAD) {
                lo = std::min({lo, lo + p.edge_u[a], lo + p.edge_v[a], lo + p.edge_u[a] + p.edge_v[a]});
                hi = std::max({hi, hi + p.edge_u[a], hi + p.edge_v[a], hi + p.edge_u[a] + p.edge_v[a]});
            } else {
                lo -= p.radius;
                hi += p.radius;
            }
            c->scene_lo[a] = std::min(c->scene_lo[a], lo);
            c->scene_hi[a] = std::max(c->scene_hi[a], hi);
        }
    }
    DevScene& d = c->scene;
    d.prims = c->prims.as<GpuPrimitive>();
    d.num_prims = np_;
    d.nodes = c->nodes.as<float4>();
    d.tnodes = c->tnodes.as<float4>();
    // The BLASes' wide trees (built at upload) stay; the TLAS's wide tree is
    // this frame's (null: the binary child pairs are walked).
    d.wnodes = c->wide_nodes ? c->wnodes.as<float4>() : nullptr;
    d.wsoup = c->wide_nodes ? c->wsoup.as<float4>() : nullptr;
    d.blas_wide = c->wide_nodes ? c->blas_wide.as<uint32_t>() : nullptr;
    d.twnodes = wide_tlas ? c->twnodes.as<float4>() : nullptr;
    d.twsoup = wide_tlas ? c->twsoup.as<uint32_t>() : nullptr;
    d.num_nodes = bn + 2 * c->inst_capacity;  // fixed while the capacity holds, so frame graphs keep replaying
    d.inst = reinterpret_cast<const GpuInstance*>(d.prims + np_);
    d.inst_box = c->inst_cull ? c->inst_box.as<float4>() : nullptr;
    d.num_instances = n;
    d.tlas_root = bn;
    d.blas_roots = c->mesh_root.as<uint32_t>();
    d.num_blas = c->num_meshes;
    c->tlas_nodes = tn;
    c->total_nodes = bn + tn;
    c->needs_instances = false;
    return LUC_OK;
}

int32_t luc_read_scene(luc_ctx* c, uint32_t which, void* out, uint64_t capacity, uint64_t* bytes) {
    if (!c || !bytes) return LUC_ERR_VALIDATION;
    if (!c->has_scene) return luc_fail(c, LUC_ERR_VALIDATION, "no scene uploaded");
    const DevScene& d = c->scene;
    const void* src = nullptr;
    uint64_t n = 0;
    switch (which) {
        case 0: src = c->nodes.p; n = (uint64_t)c->total_nodes * sizeof(GpuBvhNode); break;
        case 1: src = c->tris.p; n = (uint64_t)d.num_tris * sizeof(GpuTriangle); break;
        case 2: src = c->prims.p; n = ((uint64_t)d.num_prims + d.num_instances) * sizeof(GpuPrimitive); break;
        case 3: src = c->wnodes.p; n = d.wnodes ? (uint64_t)c->wide_nodes * 80 : 0; break;
        case 4: src = c->wsoup.p; n = d.wnodes ? (uint64_t)d.num_tris * 48 : 0; break;
        default:
            return luc_fail(c, LUC_ERR_VALIDATION,
                            "which: 0 nodes, 1 triangles, 2 primitives, 3 wide nodes, 4 wide triangle soup");
    }
    *bytes = n;
    if (!out || n == 0) return LUC_OK;
    if (capacity < n) return luc_fail(c, LUC_ERR_VALIDATION, "output buffer too small");
    cudaSetDevice(c->device);
    LUC_CUDA(c, cudaMemcpyAsync(out, src, n, cudaMemcpyDeviceToHost, c->stream), "read scene");
    LUC_CUDA(c, cudaStreamSynchronize(c->stream), "read scene");
    return LUC_OK;
}

}  // extern "C"
