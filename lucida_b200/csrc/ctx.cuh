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

struct luc_ctx {
    int device = 0;
    uint64_t scene_version = 0;
    FrameGraph graph;
    bool use_graphs = true;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    int num_sms = 148;
    // Resident scene.
    DevBuf materials, prims, lights, positions, attrs, tris, nodes, env_px, env_cond, env_marg, env_row_sin, energy;
    DevBuf tnodes, soup;  // traversal layout derived from nodes / tris
    DevBuf blas_roots;    // distinct BLAS roots of an instanced scene
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
    DevBuf g_params, g_m, g_v, g_grad, g_wbf, g_bias, g_misc, g_lobes, g_rec, g_io;
    bool guide_ready = false, guide_train = true;
    uint32_t guide_rec_cap = 1u << 18;
    float guide_lr = 1.0e-2f;
    float guide_lo[3] = {0, 0, 0}, guide_hi[3] = {1, 1, 1};
    // Bounds of the uploaded scene (vertices and analytic primitives).
    float scene_lo[3] = {0, 0, 0}, scene_hi[3] = {0, 0, 0};
};

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
int32_t luc_lbvh_device(luc_ctx* c, uint32_t n, uint32_t* num_nodes);
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
// Implemented in guide.cu: the guide's device view and training buffers,
// and per-frame allocations (mixtures for `paths` paths, records).
luc::GuideDev luc_guide_dev(const luc_ctx* c);
luc::GuideTrain luc_guide_train_state(luc_ctx* c);
int32_t luc_guide_prepare_frame(luc_ctx* c, uint64_t paths);
// Implemented in denoise.cu.
int32_t luc_denoise_device(luc_ctx* c, const GpuAccum* accum_dev, uint32_t w, uint32_t h,
                           const luc_denoise_params* p, GpuAccum* out_dev);
