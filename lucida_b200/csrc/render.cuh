// Shared host/device declarations for the wavefront integrator.
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>
#include "guide.cuh"
#include "scene_dev.cuh"

namespace luc {

// Per-depth device counters: queue length entering the depth, shadow rays
// appended at the depth.
constexpr uint32_t kCtrStride = 8;
constexpr uint32_t kCtrQueue = 0;
constexpr uint32_t kCtrShadow = 1;
constexpr uint32_t kCtrPullExtend = 2;  // ray-pull cursor of EXTEND at this depth
constexpr uint32_t kCtrPullConnect = 3;  // ray-pull cursor of CONNECT at this depth
// Split frames: extended paths whose ray hit a surface, by material class
// (kCtrHit + class slot: 4 = reflective non-metal, 6 = metal, 7 =
// transmissive), and those whose ray escaped (5).
constexpr uint32_t kCtrHit = 4;
constexpr uint32_t kCtrMiss = 5;
constexpr uint32_t kCtrHit1 = 6;
constexpr uint32_t kCtrHit2 = 7;
__host__ __device__ constexpr uint32_t hit_slot(uint32_t cls) { return cls == 0 ? kCtrHit : (cls == 1 ? kCtrHit1 : kCtrHit2); }

// SoA path pool, one float4 per field per path (128-bit accesses).
struct PathState {
    float4* o_pdf;  // ray origin, prev_bsdf_pdf
    float4* dir;    // ray direction, -
    float4* thr;    // throughput, sampler state (u32 bits)
    float4* rad;    // radiance accumulated along the path
    float4* prev;   // previous vertex (for the MIS light pdf)
    float4* hit;    // t, u, v, id (u32 bits)
    uint32_t* hinst;  // instance of the hit (instanced scenes)
    float4* galb;   // first-hit albedo, depth
    float4* gnrm;   // first-hit shading normal
    float4* sh_o;   // shadow ray origin, t_max
    float4* sh_d;   // shadow ray direction, path id (u32 bits)
    float4* sh_c;   // shadow ray contribution
    uint32_t* queue[2];
    // Split frames: this depth's extended paths by outcome (k_classify):
    // hits by material class, escaped rays.
    uint32_t *hitq[3], *missq;
    uint32_t* ctr;
    // [0] extend rays, [1] extend node visits, [2] extend triangle tests,
    // [3] shadow rays, [4] shadow node visits, [5] shadow triangle tests.
    unsigned long long* stat;
    // Guided frames: the decoded mixture per queue position (kGLobeF4 float4
    // planes of lobe_stride entries), the training records and the guide's
    // bookkeeping words.
    float4* lobes;
    uint64_t lobe_stride;
    uint32_t* seg;  // batched renders: the wave segment each path belongs to
    float4* rec;
    uint32_t* gmisc;
};

struct FrameParams {
    uint64_t num_paths;  // pixels * batch_samples
    uint32_t pixels, width, height;
    uint32_t sample_base;  // host copy only: kernels read *sbase, so one captured graph serves every offset
    const uint32_t* sbase;  // device word: the batch's first sample index
    uint32_t batch_samples;
    uint32_t frame_seed, sampler_kind, sampling, max_depth;
    uint32_t guides;
    uint32_t guided;   // one-sample MIS with the learned proposal
    uint32_t rec_cap;  // training records per batch (0: no recording)
    // Hits and escaped rays shaded apart (hit queue for SHADE and the guide,
    // k_escape for the rest); single-scene frames.
    uint32_t split;
    GuideDev guide;
    float lens_radius;
    V3 cam_origin, cam_upper_left, cam_horizontal, cam_vertical;
};

// The paths SHADE and the guide's inference visit at `depth`, and the i-th
// of them: the hit queue in split frames, else every extended path (all
// paths at depth 0, the survivor queue after).
LUC_D uint32_t shaded_count(const PathState& ps, const FrameParams& fp, uint32_t depth) {
    const uint32_t* c = ps.ctr + depth * kCtrStride;
    if (fp.split) return c[kCtrHit] + c[kCtrHit1] + c[kCtrHit2];
    return depth == 0 ? (uint32_t)fp.num_paths : c[kCtrQueue];
}
// In split frames the three class queues one after the other, so a warp's
// 32 consecutive paths share a material class except at two boundaries.
LUC_D uint32_t shaded_path(const PathState& ps, const FrameParams& fp, uint32_t depth, uint32_t i) {
    if (fp.split) {
        const uint32_t* c = ps.ctr + depth * kCtrStride;
        const uint32_t n0 = c[kCtrHit], n1 = c[kCtrHit1];
        if (i < n0) return ps.hitq[0][i];
        i -= n0;
        return i < n1 ? ps.hitq[1][i] : ps.hitq[2][i - n1];
    }
    return depth == 0 ? i : ps.queue[depth & 1][i];
}

// CUDA-event marks between stages, accumulated per stage.
struct StageTimer {
    enum Stage { kGenerate = 0, kExtend, kShade, kConnect, kResolve, kGuide, kTrain, kEnd, kCount };
    std::vector<cudaEvent_t> events;
    std::vector<int> stages;
    void mark(cudaStream_t s, int stage) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        // Inside a stream capture a plain record only orders the capture; the
        // external flag makes it an event-record node that fires on replay.
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(s, &cs);
        if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
        else cudaEventRecord(e, s);
        events.push_back(e);
        stages.push_back(stage);
    }
    // Adds the elapsed time of each interval to ms[stage of its start].
    void accumulate(double* ms) const {
        for (size_t i = 0; i + 1 < events.size(); ++i) {
            float t = 0.0f;
            cudaEventElapsedTime(&t, events[i], events[i + 1]);
            if (stages[i] < kEnd) ms[stages[i]] += t;
        }
    }
    void release() {
        for (auto e : events) cudaEventDestroy(e);
        events.clear();
        stages.clear();
    }
    void collect(double* ms) {
        accumulate(ms);
        release();
    }
};

struct RenderState {
    PathState ps{};
    uint64_t capacity = 0;  // paths
    uint32_t ctr_capacity = 0;
    int num_sms = 148;
    // Resident blocks per SM of each stage kernel (single-level / instanced).
    int extend_blocks = 0, connect_blocks = 0, shade_blocks = 0, shade_blocks_guided = 0;
    int extend_blocks_inst = 0, connect_blocks_inst = 0, shade_blocks_inst = 0, shade_blocks_guided_inst = 0;
    int extend_blocks_bin = 0, connect_blocks_bin = 0;  // single-level scenes on the binary tree
    int extend_blocks_inst_bin = 0, connect_blocks_inst_bin = 0;  // two-level scenes on binary BLASes
    bool guide_tc = true;  // guide inference on tcgen05 (LUC_GUIDE_TC=0: the mma.sync kernel)
    // Closest-hit traversal of single-level wide trees with the top 73
    // nodes (root and two levels) staged in shared memory (LUC_WIDE_STAGE=73).
    int wide_stage = 0;
    // Hits and escaped rays shaded apart (k_classify, k_escape, SHADE over
    // the hit queue); LUC_SPLIT_ESCAPES=0 shades every extended path in SHADE.
    bool split = true;
    int extend_blocks_stage = 8;
    uint64_t launches = 0;
};

void query_occupancy(RenderState& rs);
// Batched multi-scene renders (luc_render_batch). A job is one render of
// one resident scene; the pool is filled in waves, each a list of segments:
// `nsamples` whole samples (every pixel) of one job, `count` = nsamples *
// pixels paths starting at `first` in the wave. Stage kernels find a path's
// scene and frame parameters through its segment.
struct BatchJobDev {
    FrameParams fp;  // per job: size, camera, sampler, sampling, max_depth, seed
    uint32_t scene;
    GpuAccum* accum;
};
struct BatchSegDev {
    uint32_t first, count, job, sample_base, nsamples, scene;
};
struct BatchDev {
    const DevScene* scenes;
    const BatchJobDev* jobs;
    const BatchSegDev* segs;  // this wave's segments
    uint32_t num_segs;
    uint32_t chunk;           // queue entries a CTA claims per pull (EXTEND / CONNECT)
};

// Guide training buffers (FP32 master weights, Adam moments, gradient) and
// the packed copies the kernels read.
struct GuideTrain {
    float *params, *m, *v, *grad;
    uint16_t* wbf;
    float* bias;
    float* part;  // per-CTA weight-gradient slices of the training kernel
    float lr;
    bool train;
    // defer: the batch ends after k_guide_finalize; its gradient step runs
    // at the start of the next guided frame, beside GENERATE and the first
    // EXTEND. join: the event such a step records; the frame waits for it
    // after its first EXTEND (before any guide inference or SHADE).
    bool defer = false;
    cudaEvent_t join = nullptr;
};

// CONNECT on a second stream: CONNECT(d) runs beside EXTEND(d+1) and its
// guide inference; the frame waits for it before SHADE(d+1), which rewrites
// the shadow-ray buffers and the path radiance CONNECT adds to, and before
// RESOLVE.
struct ConnectOverlap {
    cudaStream_t side;
    cudaEvent_t ready, done;
};
void record_batch(RenderState& rs, const DevScene& sc, const FrameParams& fp, GpuAccum* accum, cudaStream_t stream,
                  StageTimer* timer, const GuideTrain* gt, const ConnectOverlap* ov = nullptr);
// megakernel.cu: one batch of the megakernel architecture (every path of
// fp.num_paths from start to end in one launch, then RESOLVE).
void record_megakernel(const RenderState& rs, const DevScene& sc, const FrameParams& fp, GpuAccum* accum,
                       cudaStream_t s);
// wavefront.cu: RESOLVE of one batch from the pool's radiance and guides.
void launch_resolve(const RenderState& rs, const FrameParams& fp, GpuAccum* accum, cudaStream_t stream);
// One wave of a batched render (wavefront.cu); `block` is the EXTEND /
// CONNECT block size (64, 128 or 256).
// `wide`: every scene of the batch traverses a wide tree (or has no
// triangles), so the wide-only traversal kernels serve them all.
void record_wave(RenderState& rs, const BatchDev& bd, const uint32_t* pix_off, uint32_t num_paths,
                 uint32_t total_pixels, uint32_t max_depth, int block, bool wide, cudaStream_t s);
int batch_blocks_per_sm(int block, bool connect, bool wide);
// guide.cu: per-depth inference and the post-batch training step.
void launch_guide_infer(const RenderState& rs, const DevScene& sc, const FrameParams& fp, uint32_t depth,
                        cudaStream_t s);
void launch_guide_train(const RenderState& rs, const FrameParams& fp, const GuideTrain& gt, cudaStream_t s);
// The two halves of launch_guide_train: record weights (needs the batch's
// path pool) and the gradient step on them (records and guide state only).
void launch_guide_finalize(const RenderState& rs, const FrameParams& fp, cudaStream_t s);
void launch_guide_step(const RenderState& rs, uint32_t cap, const GuideDev& g, const GuideTrain& gt, cudaStream_t s);

}  // namespace luc
