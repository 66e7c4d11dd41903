/*
 * luc_cuda.h — the C ABI of liblucida_cuda.so, the B200 (sm_100a) drop-in for
 * Lucida's wgpu harness (crate `pt-gpu`, crates/gpu/src).
 *
 * Plain pointers and sizes only; every struct crossing the boundary is one of
 * the `#[repr(C)]` layouts from crates/core/src/gpu_layout.rs restated in
 * lucida_layout.h, so a Rust `crates/cuda` shim passes `bytemuck` slices of
 * its `SceneBlob` straight through.
 *
 * Conventions
 *   - Ownership: the caller owns every host array and only lends it for the
 *     duration of the call. The context owns all device memory it allocates.
 *     A `*_dev` pointer argument is caller-owned device memory on the
 *     context's device.
 *   - Errors: every entry point returns 0 on success or a negative LUC_ERR_*
 *     code, which map one-to-one onto pt_gpu::GpuError (crates/gpu/src/
 *     lib.rs:100-112); luc_last_error() has the message. Nothing aborts.
 *   - Threading: one context per host thread; a context is not re-entrant.
 *     All work is queued on the context's stream (its own, or the one given
 *     to luc_set_stream) and every entry point that returns host data
 *     synchronises that stream before returning.
 */
#ifndef LUC_CUDA_H
#define LUC_CUDA_H

#include <stdint.h>
#include "lucida_layout.h"

#ifdef __cplusplus
extern "C" {
#endif

/* GpuError (crates/gpu/src/lib.rs:100-112) */
#define LUC_OK 0
#define LUC_ERR_NO_DEVICE (-1)  /* GpuError::NoAdapter / NoDevice */
#define LUC_ERR_LAUNCH (-2)     /* GpuError::Shader: module load or kernel launch failed */
#define LUC_ERR_READBACK (-3)   /* GpuError::Readback: device->host copy failed */
#define LUC_ERR_VALIDATION (-4) /* GpuError::Validation: bad argument, layout, size, or device status word */
#define LUC_ERR_OUT_OF_MEMORY (-5)

/* luc_render arch_flags (Architecture, crates/gpu/src/lib.rs:38-66). */
#define LUC_ARCH_WAVEFRONT 0x0u
/* One thread per pixel walks its samples and paths to the end in registers
 * (Architecture::Megakernel): same accumulator as the wavefront. Not with
 * LUC_FLAG_GUIDED. */
#define LUC_ARCH_MEGAKERNEL 0x1u
/* Skip the first-hit guide channels (albedo/normal/depth) of the
 * accumulator: they are needed only by the denoiser. */
#define LUC_FLAG_NO_GUIDES 0x100u
/* Record per-stage CUDA events during the render (luc_get_stats). */
#define LUC_FLAG_PROFILE 0x200u
/* Learned path guiding (no reference counterpart): one-sample MIS between
 * the BSDF and the guide's vMF mixture (fraction 0.5 each) at opaque,
 * non-specular vertices, with the mixture pdf in both MIS sites; after each
 * batch of samples the guide takes one Adam step on the batch's records
 * (luc_guide_configure). Requires luc_guide_init. */
#define LUC_FLAG_GUIDED 0x400u
/* Instanced scenes: cast shadow rays the way the reference does
 * (crates/core/src/scene.rs:577-606, shaders/wavefront/connect.wgsl:36-55),
 * testing the analytic primitives and then every mesh's triangles
 * untransformed, in object space, instead of through the two-level
 * hierarchy. For parity with the reference; the default is the two-level
 * any-hit. No effect on scenes without instances. */
#define LUC_FLAG_REFERENCE_SHADOWS 0x800u
/* After the render, run the convergence meter (luc_convergence) over the
 * accumulator; luc_get_stats reports it (render_with_measured,
 * crates/gpu/src/lib.rs:86-97). */
#define LUC_FLAG_MEASURE 0x1000u

/* Test hooks for the bounded device waits (luc_debug_waits). */
#define LUC_DEBUG_NONE 0u
#define LUC_DEBUG_SORT_ORPHAN_TILE 1u /* next radix sort: tile 0 never runs, tile 1's look-back waits on it */
#define LUC_DEBUG_TC_NO_COMMIT 2u     /* next tensor-core guide forward: no MMA issued, no commit to the mbarrier */

typedef struct luc_ctx luc_ctx;

/* The SceneBlob upload (crates/core/src/gpu_layout.rs:706-770 plus the
 * environment textures of crates/gpu/src/lib.rs:263-359). */
typedef struct luc_scene_view {
    const GpuMaterial* materials;
    uint32_t num_materials;
    /* Analytic primitives (spheres, quads) followed by `num_instances`
     * GpuInstance rows, as SceneBlob::primitives_upload lays them out. */
    const GpuPrimitive* primitives;
    uint32_t num_primitives; /* analytic only */
    uint32_t num_instances;
    const GpuLight* lights;
    uint32_t num_lights;
    const float* positions; /* [x, y, z, w] per vertex */
    const GpuVertexAttr* vertex_attrs;
    uint32_t num_vertices;
    const GpuTriangle* triangles;
    uint32_t num_triangles;
    /* The caller's BVH over `triangles` (leaves index triangles directly,
     * i.e. compacted as Bvh::compact_primitives leaves them). When
     * num_bvh_nodes == 0 and there are triangles, the context builds an LBVH
     * on the device (30-bit Morton, radix sort, Karras, fit, relayout) and
     * reorders its own copy of the triangles into leaf order. */
    const GpuBvhNode* bvh_nodes;
    uint32_t num_bvh_nodes;
    uint32_t tlas_root;
    /* Equirectangular environment: RGBA32F texels, row 0 = zenith, and the
     * packed CDF rectangle (cdf_width x (env_height + 1)): rows 0..h-1 hold
     * the per-row conditionals (env_width + 1 entries), row h the marginal
     * (env_height + 1 entries). env_width == 0 means no map. */
    const float* env_pixels;
    uint32_t env_width, env_height;
    const float* env_cdf;
    uint32_t env_cdf_width;
    float env_total_weight;
} luc_scene_view;

/* LbvhBuilder output (crates/gpu/src/lbvh.rs:724-733 GpuBuildOutput, plus
 * the relaid-out tree Lbvh::from_parts produces). Every pointer is a
 * caller-allocated host array or null (skipped). Sizes for n primitives:
 * codes/order: n; karras: 2(n-1); parent: 2n-1; node_bounds: 6(2n-1) floats;
 * subtree_size: n-1; scene_bounds: 6 floats (centroid box);
 * nodes: up to 2n-1 GpuBvhNode (count returned in *num_nodes);
 * prim_indices: n. */
typedef struct luc_lbvh_out {
    uint32_t* codes;        /* Morton code per primitive, input order */
    uint32_t* order;        /* sorted permutation */
    uint32_t* karras;       /* (left, right) per internal node */
    uint32_t* parent;       /* per node id, 0xFFFFFFFF for the root */
    float* node_bounds;     /* (min xyz, max xyz) per node id */
    uint32_t* subtree_size; /* per internal node */
    float* scene_bounds;    /* centroid bounds */
    GpuBvhNode* nodes;      /* relaid-out tree */
    uint32_t* prim_indices;
    uint32_t num_nodes;     /* out */
} luc_lbvh_out;

/* DenoiseParams (crates/core/src/denoise.rs:62-94). */
typedef struct luc_denoise_params {
    uint32_t iterations;
    float sigma_normal, sigma_depth, sigma_luminance, sigma_albedo;
} luc_denoise_params;

/* Per-render statistics (filled by luc_render; stage times only under
 * LUC_FLAG_PROFILE). */
typedef struct luc_render_stats {
    double ms_total;       /* device time of the whole render, CUDA events */
    double ms_generate, ms_extend, ms_shade, ms_connect, ms_resolve;
    uint64_t launches;     /* kernels this library launched */
    uint64_t rays_extend;  /* closest-hit rays traced */
    uint64_t rays_shadow;  /* shadow rays traced */
    uint64_t paths;        /* camera paths started */
    uint64_t nodes_extend, tris_extend; /* BVH node visits / triangle tests, closest hit */
    uint64_t nodes_shadow, tris_shadow; /* the same for shadow rays */
    double ms_guide, ms_train; /* guide inference and training (LUC_FLAG_GUIDED) */
    double convergence;    /* LUC_FLAG_MEASURE: the convergence meter's figure; -1 otherwise or when no
                              pixel is measurable */
    uint64_t blas_extend, blas_shadow; /* two-level scenes: instance BLASes entered, closest hit / shadow */
} luc_render_stats;

/* Layout contract: returns LUC_LAYOUT_VERSION. */
uint32_t luc_layout_version(void);
/* Byte size of each boundary struct, for a caller's own layout assertion
 * (gpu_layout.rs:993-1166): which = 0 material, 1 primitive, 2 light,
 * 3 vertex attr, 4 triangle, 5 bvh node, 6 accum, 7 uniforms, 8 instance. */
uint32_t luc_sizeof(uint32_t which);

/* Gpu::new (crates/gpu/src/lib.rs:133-242). */
int32_t luc_create(int32_t device, luc_ctx** out);
void luc_destroy(luc_ctx* ctx);
const char* luc_last_error(const luc_ctx* ctx);
/* Queue this context's work on a caller stream (a cudaStream_t); null
 * restores the context's own stream. */
int32_t luc_set_stream(luc_ctx* ctx, void* cuda_stream);

/* Upload a scene (replaces the previous one). */
int32_t luc_upload_scene(luc_ctx* ctx, const luc_scene_view* scene);

/* render(scene, camera, spp, bounces) -> HDR accumulator:
 * pt_gpu::render_with(.., Architecture::Wavefront) / wavefront::
 * render_native_on (crates/gpu/src/lib.rs:69-79, wavefront.rs:134-140).
 * `u` carries camera, resolution, frame_seed, sample_offset, sampling_mode,
 * sampler_kind and background, exactly as integrator::build_uniforms writes
 * them; its samples_per_launch and max_depth fields are ignored in favour of
 * `spp` and `max_depth`. Samples sample_offset .. sample_offset+spp-1 of
 * every pixel are traced and summed into the accumulator with the
 * semantics of RESOLVE (shaders/wavefront/resolve.wgsl:36-47).
 * Exactly one of out_host / out_dev is non-null:
 *   out_host — width*height GpuAccum, overwritten with this render alone;
 *   out_dev  — caller device array of width*height GpuAccum, accumulated
 *              into (progressive rendering). */
int32_t luc_render(luc_ctx* ctx, const GpuUniforms* u, uint32_t spp, uint32_t max_depth, uint32_t arch_flags,
                   GpuAccum* out_host, void* out_dev);
int32_t luc_get_stats(const luc_ctx* ctx, luc_render_stats* out);

/* Camera::write_uniforms (crates/core/src/camera.rs:344-365): fills the
 * camera block plus width/height of `out` (all other fields zeroed) from a
 * look-at camera with vertical field of view in degrees; aspect = w/h. */
int32_t luc_camera_uniforms(const float* eye, const float* look_at, const float* up, float vfov_deg,
                            float aperture, float focus_distance, uint32_t width, uint32_t height,
                            GpuUniforms* out);

/* LbvhBuilder::build / build_parts (crates/gpu/src/lbvh.rs:369-665). */
int32_t luc_lbvh_build(luc_ctx* ctx, const GpuTriangle* triangles, uint32_t n, const float* positions,
                       uint32_t num_vertices, luc_lbvh_out* out);
/* LBVH over arbitrary boxes (min xyz, max xyz per box): the per-frame TLAS
 * over instance world bounds. Outputs as luc_lbvh_build. */
int32_t luc_lbvh_build_boxes(luc_ctx* ctx, const float* boxes, uint32_t n, luc_lbvh_out* out);
/* LbvhBuilder::sort (crates/gpu/src/lbvh.rs:669-714): stable ascending sort
 * of (key, value) pairs by key. Host arrays. */
int32_t luc_sort_u32(luc_ctx* ctx, const uint32_t* keys, const uint32_t* vals, uint32_t n, uint32_t* keys_out,
                     uint32_t* vals_out);
/* Device-resident variant: sorts keys_dev/vals_dev in place (n pairs). */
int32_t luc_sort_u32_dev(luc_ctx* ctx, void* keys_dev, void* vals_dev, uint32_t n);

/* Per-function device evaluation, as Lucida's shader eval harness
 * (crates/gpu/src/eval.rs, shaders/test/eval_bsdf.wgsl) does for WGSL.
 * luc_eval_bsdf: material `m` seen from the front (front != 0) or back.
 *   mode 0 = surface::sample (bsdf.rs:1571-1661): in3 = (u_lobe, u.x, u.y),
 *            outputs wi, weight (f|cos|/pdf) and pdf;
 *   mode 1 = surface::eval + surface::pdf at (wo, wi = in3): outputs f, pdf.
 * luc_eval_env: the resident scene's environment map.
 *   mode 0 = EnvMap::sample (envmap.rs:235-275): in = u (2 floats), outputs
 *            direction, radiance, pdf;
 *   mode 1 = EnvMap::radiance + pdf at direction in (3 floats).
 * n entries, host arrays, 3 floats per vector. */
int32_t luc_eval_bsdf(luc_ctx* ctx, const GpuMaterial* m, int32_t front, const float* wo3, const float* in3,
                      uint32_t n, int32_t mode, float* out_wi3, float* out_f3, float* out_pdf);
int32_t luc_eval_env(luc_ctx* ctx, const float* in, uint32_t n, int32_t mode, float* dir3, float* rad3, float* pdf);
/* Ray queries against the resident scene, n rays of 8 floats (origin xyz,
 * t_max, direction xyz, unused), host arrays.
 *   mode 0 = Scene::intersect (crates/core/src/scene.rs:452-527): out holds
 *            n x (t, u, v, id as u32 bits), id = triangle (leaf order) or
 *            analytic primitive | 0x80000000, 0xFFFFFFFF on a miss (t_max
 *            is not used);
 *   mode 1 = Scene::occluded (scene.rs:577-606) within (1e-4, t_max): out
 *            holds n u32, 1 = occluded. */
int32_t luc_intersect(luc_ctx* ctx, const float* rays8, uint32_t n, int32_t mode, void* out);
/* Convergence meter (ConvergenceMeter, crates/gpu/src/stats.rs;
 * shaders/stats/convergence.wgsl): over a device accumulator of `pixels`
 * GpuAccum, the mean relative standard error of the pixel means, taken over
 * pixels with >= 2 samples and mean luminance > 1e-3 (-1 if none). Assumes
 * independent samples: with Sobol it over-reports. */
int32_t luc_convergence(luc_ctx* ctx, const void* accum_dev, uint32_t pixels, float* out);
/* Bandwidth reference (no reference counterpart; the benchmark's roofline
 * denominator for L2-resident traffic): `passes` streaming reads of `bytes`
 * (a multiple of 16, 16-byte aligned) of caller device memory on the ctx's
 * stream, asynchronous. sink_dev: 148 * 8 u32 the kernel XORs into. Over a
 * buffer that fits and stays in L2 it measures L2 read bandwidth. */
int32_t luc_read_sweep(luc_ctx* ctx, const void* buf_dev, uint64_t bytes, uint32_t passes, void* sink_dev);
/* Test hook (no reference counterpart): make the next call of one kind wait
 * on a flag nothing sets, so its bounded wait runs out after `limit` polls
 * and the call returns its error status (a radix sort: LUC_ERR_VALIDATION,
 * "look-back wait gave up"; luc_guide_forward: LUC_ERR_LAUNCH, "a
 * tensor-core wait ran out"), with the context usable afterwards. Nothing
 * faults or hangs: the waits are the kernels' own bounded loops, and no
 * tensor-core work is left in flight. One-shot; LUC_DEBUG_NONE cancels. */
int32_t luc_debug_waits(luc_ctx* ctx, uint32_t mode, uint32_t limit);
/* Sample-range shards (crates/gpu/tests/cpu_gpu_agreement.rs:119-168: a
 * progressive render equals a one-shot one, so per-rank accumulators over
 * disjoint sample ranges sum to the frame's): out[px] = parts[0][px] +
 * parts[1][px] + ... field by field, in rank order, on the ctx's stream
 * (asynchronous). parts_dev: nparts consecutive arrays of `pixels` GpuAccum
 * (device, 16-byte aligned), e.g. the output of an all-gather; out_dev may
 * alias parts_dev's first array. */
int32_t luc_accum_merge(luc_ctx* ctx, const void* parts_dev, uint32_t nparts, uint32_t pixels, void* out_dev);

/* Sort without allocating: the variant of luc_sort_u32_dev for callers that
 * cannot call cudaMalloc (a host that reserves all device memory up front, or
 * a frame loop where an allocation would synchronise the device). It has no
 * counterpart in the reference. Sorts n <= luc_sort_u32_static_max() = 2^20
 * (key, value) pairs of caller device memory in place on `stream` (a
 * cudaStream_t of the current device; null = the legacy default stream) and
 * returns when the sort is done. Scratch is a file-scope device array (about
 * 8.3 MiB, held on every GPU that loads the library until exit), shared by
 * every call: calls that overlap on the GPU race. Each call looks up the
 * array's device address in the current context, and it is synchronous: it
 * waits on `stream` for the sort and reads back its status before returning.
 * Larger n returns LUC_ERR_VALIDATION; messages go to err_msg (may be null). */
int32_t luc_sort_u32_static(void* keys_dev, void* vals_dev, uint32_t n, void* stream, char* err_msg,
                            uint32_t err_len);
uint32_t luc_sort_u32_static_max(void);

/* ---- Device-built instancing (no reference counterpart: the reference
 * builds its BLASes and TLAS once, on the CPU, with binned SAH in
 * Scene::build_instances, crates/core/src/scene.rs:252-345) ----
 * luc_upload_meshes uploads a scene like luc_upload_scene (no instances, no
 * tree) whose triangles are grouped into meshes (ascending, disjoint ranges
 * [first, first + count)) in object space, and builds one LBVH per mesh on the
 * device. luc_set_instances then places the meshes: per instance a row-major
 * 3x4 object-to-world transform (12 floats), a mesh index and a material
 * override (UINT32_MAX keeps the triangles' own); the device inverts each
 * transform, bounds each instance in world space and rebuilds the TLAS by
 * LBVH over those boxes. Call it again whenever the placements change (per
 * frame); rendering needs at least one call after the upload. */
int32_t luc_upload_meshes(luc_ctx* ctx, const luc_scene_view* view, const uint32_t* mesh_first,
                          const uint32_t* mesh_count, uint32_t num_meshes);
int32_t luc_set_instances(luc_ctx* ctx, const float* object_to_world, const uint32_t* mesh, const uint32_t* material,
                          uint32_t num_instances);
/* Leaf size of the TLAS that luc_set_instances (and an instanced upload)
 * builds: subtrees of at most max_leaf instances (1..64) collapse into one
 * leaf. The reference builds its TLAS with LBVH_MAX_LEAF = 4 (lbvh.rs:185);
 * pass 4 for its node layout bit for bit. The default, 1, tests every
 * instance's box in the tree walk's near-first order instead of looping over
 * a leaf's instances (the instanced frame of 4096 instances renders 16%
 * faster). Renders are the same either way: every walk keeps the nearest hit
 * (only which of two exactly tied hits wins can differ). Takes effect at the
 * next TLAS build. */
int32_t luc_set_tlas_leaf(luc_ctx* ctx, uint32_t max_leaf);
/* Copy the resident scene's arrays to the host: which = 0 BVH nodes (every
 * BLAS then the TLAS), 1 triangles (leaf order), 2 primitives (analytic, then
 * instance rows in TLAS-leaf order), 3 compressed 8-wide nodes (80 B each;
 * 0 bytes when the scene traverses the binary tree), 4 the wide tree's
 * triangle soup (48 B per triangle: p0 with the leaf-order index in p0.w as
 * u32 bits, p1 - p0, p2 - p0). *bytes receives the size; out may be null to
 * query it. */
int32_t luc_read_scene(luc_ctx* ctx, uint32_t which, void* out, uint64_t capacity, uint64_t* bytes);

/* ---- Batched multi-scene rendering (no reference counterpart) ----
 * Renders many jobs (a resident scene, its uniforms, spp, bounces and a
 * device accumulator each) through one shared path pool: the pool is filled
 * in waves of whole samples taken from the jobs in order, paths of different
 * scenes share the ray and hit queues and find their scene through their
 * wave segment, and the whole batch is recorded as one CUDA graph. Each
 * job's scene is the resident scene of its own context (luc_upload_scene on
 * the same device; single-level scenes); the batch runs on `ctx`'s stream
 * and pool. Accumulators are accumulated into, as luc_render does. */
typedef struct luc_batch_job {
    luc_ctx* scene;       /* context holding the scene */
    GpuUniforms uniforms; /* camera, size, seed, sampler, sampling */
    uint32_t spp, max_depth;
    void* accum_dev;      /* width * height GpuAccum on the device */
} luc_batch_job;
/* Launch shape of the traversal stages: threads per block (64, 128, 256)
 * and the queue entries a block claims per pull (32 = one warp at a time,
 * else 1024, 4096 or 16384 per block). */
typedef struct luc_batch_config {
    uint32_t block, chunk;
} luc_batch_config;
int32_t luc_batch_configure(luc_ctx* ctx, const luc_batch_config* cfg);
/* job_done_ms (num_jobs entries, may be null): device time from the batch's
 * start until the wave that finished the job; stats may be null. */
int32_t luc_render_batch(luc_ctx* ctx, const luc_batch_job* jobs, uint32_t num_jobs, double* job_done_ms,
                         luc_render_stats* stats);
/* Time every launch shape on the batch's first `waves` waves (rendering into
 * scratch accumulators, the jobs' own are untouched), keep the fastest as
 * the context's configuration and return it. tried (may be null) receives,
 * per tried shape, {block, chunk, ms} as 3 doubles, in the order block in
 * {64, 128, 256} x chunk in {32, 1024, 4096, 16384}. */
int32_t luc_batch_autotune(luc_ctx* ctx, const luc_batch_job* jobs, uint32_t num_jobs, uint32_t waves,
                           luc_batch_config* best, double* tried);

/* ---- Learned path-guiding proposal (no reference counterpart) ----
 * Model: frequency-encoded position (12 frequencies per axis over the guide's
 * box), shading normal and outgoing direction (4 each), 120 features padded to
 * 128 -> 64 -> 64 -> 64 -> 40 ReLU MLP, BF16 weights and FP32 accumulation on
 * the tensor cores; outputs 8 vMF lobes (direction, kappa = min(1 +
 * softplus, 1e4), softmax weight). Parameters: kGParams = 19176 floats in the
 * order W1[64][128], b1[64], W2[64][64], b2, W3[64][64], b3, W4[40][64], b4[40].
 * Training: loss -sum F log q(wi) / sum F over path-vertex records, Adam
 * (0.9, 0.999, 1e-8). */
typedef struct luc_guide_info {
    uint32_t steps;        /* Adam steps taken */
    uint32_t last_records; /* records in the last step */
    float last_loss;       /* loss of the last step */
    uint32_t threshold;    /* current recording fraction, out of 65536 */
    uint32_t num_params;   /* 19176 */
    uint32_t tc_error;     /* nonzero: a tensor-core kernel's bounded wait ran out (inference results invalid) */
} luc_guide_info;

/* Initialise the guide: params (num_params floats) or, when null, a seeded
 * uniform +-sqrt(6 / (fan_in + fan_out)) initialisation; the position box
 * lo/hi (3 floats each) or, when both are null, the uploaded scene's bounds.
 * Resets the Adam state. */
int32_t luc_guide_init(luc_ctx* ctx, const float* params, uint64_t seed, const float* lo, const float* hi);
/* train != 0: one Adam step after every batch of a LUC_FLAG_GUIDED render on
 * up to records_per_step path vertices (default 2^18), learning rate lr
 * (default 1e-2). train == 0 renders with the guide frozen. */
int32_t luc_guide_configure(luc_ctx* ctx, uint32_t train, uint32_t records_per_step, float lr);
int32_t luc_guide_get_params(luc_ctx* ctx, float* out);
int32_t luc_guide_stats(luc_ctx* ctx, luc_guide_info* out);
/* Raw network outputs (40 floats per row) for rows of 9 floats: position,
 * shading normal, outgoing direction. Host arrays. */
/* luc_guide_forward through a chosen implementation: path 0 the tcgen05
 * tensor-core kernel (what luc_guide_forward runs), 1 the mma.sync kernel. */
int32_t luc_guide_forward_ex(luc_ctx* ctx, const float* in9, uint32_t n, int32_t path, float* out40);
int32_t luc_guide_forward(luc_ctx* ctx, const float* in9, uint32_t n, float* out40);
/* Host training records, 20 floats each: position, F, normal, -, outgoing
 * direction, -, sampled direction, -, 4 unused. steps == 0: the gradient of
 * the loss (num_params floats into grad_out) at the current parameters, which
 * stay unchanged; steps > 0: that many Adam steps on these records. loss_out
 * (may be null) receives the loss of the last evaluation. */
int32_t luc_guide_train_records(luc_ctx* ctx, const float* records, uint32_t n, uint32_t steps, float* grad_out,
                                float* loss_out);
/* vMF mixture of given raw outputs (40 floats per row): mode 0 samples it
 * with in3 = 3 uniforms per row (lobe choice, then the lobe) into dir3 and
 * its pdf; mode 1 evaluates the pdf at the unit directions in3. */
int32_t luc_guide_mixture(luc_ctx* ctx, const float* raw40, const float* in3, uint32_t n, int32_t mode, float* dir3,
                          float* pdf);

/* Denoiser::run (crates/gpu/src/denoise.rs:103-210): edge-avoiding à-trous
 * over an accumulator (radiance/albedo/normal/depth sums and samples);
 * writes an Accum-shaped image with samples = 1. Host arrays. */
int32_t luc_denoise(luc_ctx* ctx, const GpuAccum* accum, uint32_t width, uint32_t height,
                    const luc_denoise_params* params, GpuAccum* out);
/* The same on device buffers (GpuAccum arrays; out must not alias accum),
 * queued on the context's stream without synchronising. With
 * LUC_DENOISE_HALF_GUIDES the edge-stopping guides (normal, depth, albedo)
 * are kept in FP16 (no reference counterpart): 10 bytes of guide per tap
 * instead of 20, the colour stays FP32. */
#define LUC_DENOISE_HALF_GUIDES 0x1u
int32_t luc_denoise_dev(luc_ctx* ctx, const void* accum_dev, uint32_t width, uint32_t height,
                        const luc_denoise_params* params, uint32_t flags, void* out_dev);

#ifdef __cplusplus
} /* extern "C" */
#endif
#endif /* LUC_CUDA_H */
