// The context behind the C ABI: device, stream, resident scene, path pool.
#pragma once
#include <string>
#include "render.cuh"
#include "../../include/luc_cuda.h"

// A growable device allocation owned by the context.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, n ? n : 16);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const { return (T*)p; }
};

// One captured frame: the whole GENERATE..RESOLVE sequence of a single-batch
// render as a CUDA graph, replayed while the frame's parameters repeat.
struct FrameGraph {
    std::vector<unsigned char> key;
    cudaGraphExec_t exec = nullptr;
    luc::StageTimer timer;  // event nodes inside the graph (profiled frames)
    uint64_t launches = 0;
    bool profiled = false;
};

constexpr uint32_t kLbvhMaxLeaf = 4;  // LBVH_MAX_LEAF (lbvh.rs:185)

struct luc_ctx {
    int device = 0;
    // Test hook (luc_debug_waits): the next radix sort's or tensor-core
    // forward's bounded wait is made to run out after dbg_limit polls of a
    // flag nothing sets. One-shot: the call that uses it clears dbg_mode.
    uint32_t dbg_mode = 0, dbg_limit = 0;
    FrameGraph graph;
    bool use_graphs = true;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    int num_sms = 148;
    // Resident scene.
    DevBuf materials, prims, lights, positions, attrs, tris, nodes, env_px, env_cond, env_marg, env_row_sin, energy;
    DevBuf tnodes, soup;  // traversal layout derived from nodes / tris
    DevBuf wnodes, wsoup, wtasks, wctr;  // compressed 8-wide tree (wide.cu)
    DevBuf twnodes, twsoup;              // the TLAS's 8-wide tree, rebuilt with it
    DevBuf wroots, blas_wide;            // its roots; BLAS binary root -> wide root (two-level scenes)
    DevBuf conv_scratch;                 // convergence meter partials + result (stats.cu)
    DevBuf upload_scratch;               // upload: validation word, vertex-bound keys
    uint32_t wide_nodes = 0;             // 0: the scene traverses the binary tree
    bool use_wide = true;                // LUC_BINARY_BVH=1 turns the wide tree off
    DevBuf blas_roots;    // distinct BLAS roots of an instanced scene
    // Meshes uploaded for device-built instancing (luc_upload_meshes): per
    // mesh its BLAS root node and object-space bounds (6 floats), the BLAS
    // node total (= the TLAS's first node), the analytic primitives, and the
    // instance capacity the buffers are sized for.
    DevBuf mesh_root, mesh_bounds, inst_in, inst_tmp;
    // Device-built instancing: each instance's padded world box in TLAS-leaf
    // order (two float4), tested before its BLAS is entered.
    DevBuf inst_box;
    bool inst_cull = true;  // LUC_INST_CULL=0 enters every BLAS of a TLAS leaf
    uint32_t tlas_leaf = 1;  // instances per TLAS leaf at most (luc_set_tlas_leaf)
    std::vector<uint32_t> host_mesh_root;
    std::vector<GpuPrimitive> host_prims;
    uint32_t blas_nodes = 0, inst_capacity = 0, num_meshes = 0;
    bool needs_instances = false;
    uint32_t total_nodes = 0, tlas_nodes = 0;
    // Batched renders: launch shape, and the device tables of the last batch.
    uint32_t batch_block = 128, batch_chunk = 32;
    DevBuf b_scenes, b_jobs, b_segs, b_pixoff, b_scratch;  // nodes as uploaded or built; TLAS nodes of the last luc_set_instances
    luc::DevScene scene{};
    bool has_scene = false;
    uint32_t num_materials = 0;
    // Path pool and frame.
    luc::RenderState rs;
    DevBuf pool, accum_tmp, frame_word;  // frame_word: the batch's first sample index (FrameParams::sbase)
    luc_render_stats stats{};
    uint64_t path_budget = 1ull << 25;
    // LBVH / sort scratch.
    DevBuf lb_tris, lb_pos, lb_boxes, lb_keys, lb_vals, lb_keys2, lb_vals2, lb_hist, lb_karras, lb_parent,
        lb_nbounds, lb_subtree, lb_flags, lb_nodes, lb_rank, lb_misc, lb_icount, lb_look, lb_codes;
    // Denoiser scratch.
    DevBuf dn_in, dn_out, dn_a, dn_b, dn_dev;
    // Learned guide: FP32 master, Adam moments, gradient, packed weights,
    // bookkeeping words, per-path mixtures, training records, host-call io.
    DevBuf g_params, g_m, g_v, g_grad, g_wbf, g_bias, g_misc, g_lobes, g_rec, g_io, g_part;
    bool guide_ready = false, guide_train = true;
    uint32_t guide_rec_cap = 1u << 18;
    // The last guided frame's gradient step, not yet run (its records' cap),
    // and the stream and events that run it beside the next frame's start.
    bool guide_pending = false;
    uint32_t guide_pending_cap = 0;
    cudaStream_t side_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_ready = nullptr, ev_done = nullptr;  // CONNECT beside the next EXTEND
    cudaEvent_t ev_up0 = nullptr, ev_up1 = nullptr;     // uploads beside the BVH build
    float guide_lr = 1.0e-2f;
    float guide_lo[3] = {0, 0, 0}, guide_hi[3] = {1, 1, 1};
    // Bounds of the uploaded scene (vertices and analytic primitives).
    float scene_lo[3] = {0, 0, 0}, scene_hi[3] = {0, 0, 0};
};

// Host array -> DevBuf (grown to n elements), asynchronously on stream s.
template <class T>
cudaError_t upload(DevBuf& b, const T* src, size_t n, cudaStream_t s) {
    cudaError_t e = b.ensure(n * sizeof(T));
    if (e != cudaSuccess || n == 0 || !src) return e;
    return cudaMemcpyAsync(b.p, src, n * sizeof(T), cudaMemcpyHostToDevice, s);
}

// Error helpers: record a message and return a LUC_ERR_* code.
int32_t luc_fail(luc_ctx* c, int32_t code, const std::string& msg);
int32_t luc_cuda_fail(luc_ctx* c, cudaError_t e, const char* what);
#define LUC_CUDA(ctx, call, what)                                   \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return luc_cuda_fail((ctx), _e, (what)); \
    } while (0)

// Implemented in lbvh.cu: build an LBVH on the device over `n` boxes already
// resident at lb_boxes (min xyz, max xyz as 6 floats each), leaving the
// relaid-out tree in lb_nodes (count in *num_nodes) and the sorted order
// (leaf primitive order) in lb_vals.
// max_leaf: the collapse keeps subtrees of at most this many primitives as
// one leaf (kLbvhMaxLeaf for the reference's builds).
int32_t luc_lbvh_device(luc_ctx* c, uint32_t n, uint32_t* num_nodes, uint32_t max_leaf = kLbvhMaxLeaf);
// Triangle boxes (padded as bvh.rs:100-111) from resident triangles/positions
// into lb_boxes.
int32_t luc_triangle_boxes_device(luc_ctx* c, const GpuTriangle* tris_dev, const float4* pos_dev, uint32_t n);
// Stable LSD radix sort of n (key, value) pairs resident in lb_keys/lb_vals;
// result in lb_keys/lb_vals.
int32_t luc_radix_sort_device(luc_ctx* c, uint32_t n);
// Gather triangles into leaf order on the device: dst[i] = src[order[i]].
int32_t luc_gather_triangles(luc_ctx* c, const GpuTriangle* src, GpuTriangle* dst, const uint32_t* order, uint32_t n);
// Implemented in wavefront.cu: derive the traversal layout (child-pair
// records, triangle soup) from the resident nodes and triangles.
int32_t luc_build_traversal(luc_ctx* c, uint32_t num_nodes, uint32_t num_tris);
// guide_tc.cu: the guide MLP forward on tcgen05 (n rows of 9 inputs -> 40
// raw outputs); *err becomes nonzero if a bounded wait ran out.
cudaError_t launch_guide_forward_tc(const float* in9, uint32_t n, const luc::GuideDev& g, float* out40, uint32_t* err,
                                    int num_sms, cudaStream_t s);
// guide_tc.cu: per-bounce guide inference on tcgen05 (the render's path);
// guide_tc_setup opts its kernels into their shared memory (before capture).
void launch_guide_infer_tc(const luc::RenderState& rs, const luc::DevScene& sc, const luc::FrameParams& fp,
                           uint32_t depth, cudaStream_t s);
cudaError_t guide_tc_setup();
// guide_tc.cu: one gradient evaluation over `cap` records on tcgen05 (the
// per-CTA slices go to `part`, the biases and loss to grad / gmisc); returns
// the number of slices.
uint32_t launch_guide_gradient_tc(const float4* rec, uint32_t cap, uint32_t* gmisc, const luc::GuideDev& g,
                                  float* grad, float* part, int num_sms, cudaStream_t s);
// stats.cu: record the convergence meter over a device accumulator on `s`;
// the figure lands in c->conv_scratch after 64 float2 partials.
int32_t luc_record_convergence(luc_ctx* c, const GpuAccum* accum, uint32_t pixels, cudaStream_t s);
// wide.cu: collapse the binary tree into c->wnodes / c->wsoup (sets
// c->wide_nodes; 0 when the tree is too deep for the level budget).
int32_t luc_build_wide(luc_ctx* c, uint32_t num_nodes, uint32_t num_tris);
// The same over several roots (one wide tree each, wide node k = roots[k]'s
// tree); with `map`, fills c->blas_wide (binary root -> wide root).
int32_t luc_build_wide_roots(luc_ctx* c, const uint32_t* roots, uint32_t nroots, bool map, uint32_t num_nodes,
                             uint32_t num_tris);
// The TLAS (binary nodes [root, num_nodes), leaves of <= 4 instances) into
// c->twnodes / c->twsoup; *ok false when it keeps the binary walk.
int32_t luc_build_wide_tlas(luc_ctx* c, uint32_t root, uint32_t num_nodes, uint32_t prim_bound, uint32_t ninst,
                            bool* ok);
int32_t luc_build_tnodes_range(luc_ctx* c, uint32_t begin, uint32_t end);
// Implemented in instances.cu: one LBVH per mesh range of the triangles in
// lb_tris into c->nodes / c->tris (see luc_upload_meshes).
int32_t luc_build_blases(luc_ctx* c, const uint32_t* first, const uint32_t* count, uint32_t nm, uint32_t ntris,
                         uint32_t* blas_nodes);
// Implemented in guide.cu: the guide's device view and training buffers,
// and per-frame allocations (mixtures for `paths` paths, records).
luc::GuideDev luc_guide_dev(const luc_ctx* c);
luc::GuideTrain luc_guide_train_state(luc_ctx* c);
int32_t luc_guide_prepare_frame(luc_ctx* c, uint64_t paths);
int32_t luc_guide_flush(luc_ctx* c);
// wavefront.cu: fill the Sobol byte tables on the current device.
cudaError_t luc_init_sobol_tables(cudaStream_t s);
// capi.cu: grow the path pool to `paths` paths and `max_depth` bounces.
int32_t ensure_pool(luc_ctx* c, uint64_t paths, uint32_t max_depth);
// Implemented in denoise.cu.
int32_t luc_denoise_device(luc_ctx* c, const GpuAccum* accum_dev, uint32_t w, uint32_t h,
                           const luc_denoise_params* p, GpuAccum* out_dev, bool half_guides);
