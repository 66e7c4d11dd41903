// Batched multi-scene rendering (luc_render_batch) and its autotuner.
//
// The shared path pool is filled in waves: the host walks the jobs in order
// and cuts each into segments of whole samples (every pixel of `nsamples`
// samples) until the pool is full, then opens the next wave. A wave runs the
// ordinary stage sequence over paths of mixed scenes — GENERATE finds each
// path's segment by binary search, EXTEND / SHADE / CONNECT reach the scene
// and frame parameters through it, RESOLVE adds each segment's samples in
// sample order onto its job's accumulator — so a batch of uneven jobs keeps
// the pool full instead of draining it per scene. The whole batch is one
// CUDA graph, with an event node after every wave for per-job completion
// times. No reference counterpart: the reference renders one scene per call.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>
#include "ctx.cuh"

using namespace luc;

namespace {

struct Wave {
    uint32_t seg_begin, seg_count, num_paths, total_pixels, max_depth;
};
struct Plan {
    std::vector<BatchSegDev> segs;
    std::vector<uint32_t> pixoff;  // per segment, relative to its wave
    std::vector<Wave> waves;
    std::vector<uint32_t> job_wave;  // wave holding each job's last segment
    uint32_t max_depth = 1;
    uint64_t capacity = 0;
};

FrameParams job_params(const luc_batch_job& j) {
    const GpuUniforms* u = &j.uniforms;
    FrameParams fp{};
    fp.pixels = u->width * u->height;
    fp.width = u->width;
    fp.height = u->height;
    fp.frame_seed = u->frame_seed;
    fp.sampler_kind = u->sampler_kind;
    fp.sampling = u->sampling_mode;
    fp.max_depth = j.max_depth;
    fp.guides = 1u;
    fp.lens_radius = u->lens_radius;
    fp.cam_origin = ld3(u->cam_origin);
    fp.cam_upper_left = ld3(u->cam_upper_left);
    fp.cam_horizontal = ld3(u->cam_horizontal);
    fp.cam_vertical = ld3(u->cam_vertical);
    return fp;
}

int32_t validate(luc_ctx* c, const luc_batch_job* jobs, uint32_t n) {
    if (!jobs || n == 0) return luc_fail(c, LUC_ERR_VALIDATION, "no jobs");
    for (uint32_t i = 0; i < n; ++i) {
        const luc_batch_job& j = jobs[i];
        const std::string at = "job " + std::to_string(i) + ": ";
        if (!j.scene || !j.scene->has_scene || j.scene->needs_instances)
            return luc_fail(c, LUC_ERR_VALIDATION, at + "no resident scene");
        if (j.scene->device != c->device) return luc_fail(c, LUC_ERR_VALIDATION, at + "scene on another device");
        if (j.scene->scene.num_instances) return luc_fail(c, LUC_ERR_VALIDATION, at + "instanced scenes are not batched");
        const GpuUniforms& u = j.uniforms;
        if (u.width == 0 || u.height == 0 || (uint64_t)u.width * u.height > c->path_budget)
            return luc_fail(c, LUC_ERR_VALIDATION, at + "image empty or larger than the path pool");
        if (j.spp == 0 || j.max_depth == 0 || j.max_depth > 256)
            return luc_fail(c, LUC_ERR_VALIDATION, at + "spp must be positive and max_depth in 1..=256");
        if (u.sampling_mode > 2 || u.sampler_kind > 1) return luc_fail(c, LUC_ERR_VALIDATION, at + "bad sampling mode");
        if (!j.accum_dev) return luc_fail(c, LUC_ERR_VALIDATION, at + "no accumulator");
    }
    return LUC_OK;
}

Plan make_plan(const luc_batch_job* jobs, uint32_t n, uint64_t capacity, uint32_t max_waves) {
    Plan pl;
    pl.capacity = capacity;
    pl.job_wave.assign(n, 0);
    Wave w{0, 0, 0, 0, 1};
    auto close = [&]() {
        if (w.seg_count) pl.waves.push_back(w);
        w = Wave{(uint32_t)pl.segs.size(), 0, 0, 0, 1};
    };
    for (uint32_t j = 0; j < n && pl.waves.size() < max_waves; ++j) {
        const uint32_t pixels = jobs[j].uniforms.width * jobs[j].uniforms.height;
        uint32_t left = jobs[j].spp, sample = jobs[j].uniforms.sample_offset;
        while (left && pl.waves.size() < max_waves) {
            uint64_t fit = (capacity - w.num_paths) / pixels;
            if (fit == 0) {
                close();
                continue;
            }
            uint32_t k = (uint32_t)std::min<uint64_t>(left, fit);
            pl.segs.push_back(BatchSegDev{w.num_paths, k * pixels, j, sample, k, j});
            pl.pixoff.push_back(w.total_pixels);
            w.seg_count++;
            w.num_paths += k * pixels;
            w.total_pixels += pixels;
            w.max_depth = std::max(w.max_depth, jobs[j].max_depth);
            left -= k;
            sample += k;
            pl.job_wave[j] = (uint32_t)pl.waves.size();
        }
    }
    if (pl.waves.size() < max_waves) close();
    for (const Wave& x : pl.waves) pl.max_depth = std::max(pl.max_depth, x.max_depth);
    return pl;
}

// Upload the tables, capture every wave into one graph, run it; wave_ms (one
// per wave) receives each wave's completion time from the start.
int32_t run_plan(luc_ctx* c, const luc_batch_job* jobs, uint32_t n, const Plan& pl, uint32_t block, uint32_t chunk,
                 std::vector<double>& wave_ms, double* total_ms) {
    cudaStream_t s = c->stream;
    uint64_t most = 1;
    for (const Wave& x : pl.waves) most = std::max<uint64_t>(most, x.num_paths);
    int32_t rc = ensure_pool(c, most, pl.max_depth);
    if (rc) return rc;
    if (c->rs.shade_blocks == 0) query_occupancy(c->rs);
    std::vector<DevScene> scenes(n);
    std::vector<BatchJobDev> jd(n);
    bool wide = true;
    for (uint32_t j = 0; j < n; ++j) {
        scenes[j] = jobs[j].scene->scene;
        wide = wide && (scenes[j].wnodes || scenes[j].num_tris == 0);
        scenes[j].background = ld3(jobs[j].uniforms.background);
        scenes[j].reference_shadows = false;
        jd[j] = BatchJobDev{job_params(jobs[j]), j, (GpuAccum*)jobs[j].accum_dev};
    }
    LUC_CUDA(c, upload(c->b_scenes, scenes.data(), scenes.size(), s), "upload batch scenes");
    LUC_CUDA(c, upload(c->b_jobs, jd.data(), jd.size(), s), "upload batch jobs");
    LUC_CUDA(c, upload(c->b_segs, pl.segs.data(), pl.segs.size(), s), "upload batch segments");
    LUC_CUDA(c, upload(c->b_pixoff, pl.pixoff.data(), pl.pixoff.size(), s), "upload batch offsets");
    LUC_CUDA(c, cudaMemsetAsync(c->rs.ps.stat, 0, 8 * sizeof(unsigned long long), s), "clear counters");
    LUC_CUDA(c, cudaStreamSynchronize(s), "batch tables");
    std::vector<cudaEvent_t> ev(pl.waves.size() + 1);
    for (auto& e : ev) cudaEventCreate(&e);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    LUC_CUDA(c, cudaStreamBeginCapture(c->own_stream, cudaStreamCaptureModeThreadLocal), "begin batch capture");
    for (size_t w = 0; w < pl.waves.size(); ++w) {
        const Wave& x = pl.waves[w];
        BatchDev bd{c->b_scenes.as<DevScene>(), c->b_jobs.as<BatchJobDev>(), c->b_segs.as<BatchSegDev>() + x.seg_begin,
                    x.seg_count, chunk};
        record_wave(c->rs, bd, c->b_pixoff.as<uint32_t>() + x.seg_begin, x.num_paths, x.total_pixels, x.max_depth,
                    (int)block, wide, c->own_stream);
        cudaEventRecordWithFlags(ev[w + 1], c->own_stream, cudaEventRecordExternal);
    }
    cudaError_t ce = cudaStreamEndCapture(c->own_stream, &graph);
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
        for (auto& e : ev) cudaEventDestroy(e);
        return luc_cuda_fail(c, ce, "batch graph");
    }
    cudaEventRecord(ev[0], s);
    ce = cudaGraphLaunch(exec, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    cudaGraphExecDestroy(exec);
    if (ce != cudaSuccess) {
        for (auto& e : ev) cudaEventDestroy(e);
        return luc_fail(c, LUC_ERR_LAUNCH, std::string("batch: ") + cudaGetErrorString(ce));
    }
    wave_ms.assign(pl.waves.size(), 0.0);
    for (size_t w = 0; w < pl.waves.size(); ++w) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev[0], ev[w + 1]);
        wave_ms[w] = ms;
    }
    *total_ms = wave_ms.empty() ? 0.0 : wave_ms.back();
    for (auto& e : ev) cudaEventDestroy(e);
    return LUC_OK;
}

bool valid_shape(uint32_t block, uint32_t chunk) {
    return (block == 64 || block == 128 || block == 256) &&
           (chunk == 32 || chunk == 1024 || chunk == 4096 || chunk == 16384);
}

}  // namespace

extern "C" {

int32_t luc_batch_configure(luc_ctx* c, const luc_batch_config* cfg) {
    if (!c || !cfg) return LUC_ERR_VALIDATION;
    if (!valid_shape(cfg->block, cfg->chunk))
        return luc_fail(c, LUC_ERR_VALIDATION, "block must be 64, 128 or 256 and chunk 32, 1024, 4096 or 16384");
    c->batch_block = cfg->block;
    c->batch_chunk = cfg->chunk;
    return LUC_OK;
}

int32_t luc_render_batch(luc_ctx* c, const luc_batch_job* jobs, uint32_t n, double* job_done_ms,
                         luc_render_stats* stats) {
    if (!c) return LUC_ERR_VALIDATION;
    cudaSetDevice(c->device);
    if (int32_t rc = validate(c, jobs, n)) return rc;
    Plan pl = make_plan(jobs, n, c->path_budget, 0xFFFFFFFFu);
    std::vector<double> wave_ms;
    double total = 0.0;
    if (int32_t rc = run_plan(c, jobs, n, pl, c->batch_block, c->batch_chunk, wave_ms, &total)) return rc;
    if (job_done_ms)
        for (uint32_t j = 0; j < n; ++j) job_done_ms[j] = wave_ms[pl.job_wave[j]];
    if (stats) {
        unsigned long long counts[8] = {0};
        LUC_CUDA(c, cudaMemcpy(counts, c->rs.ps.stat, sizeof(counts), cudaMemcpyDeviceToHost), "read counters");
        luc_render_stats st{};
        st.ms_total = total;
        for (const BatchSegDev& sg : pl.segs) st.paths += sg.count;
        st.rays_extend = counts[0];
        st.nodes_extend = counts[1];
        st.tris_extend = counts[2];
        st.rays_shadow = counts[3];
        st.nodes_shadow = counts[4];
        st.tris_shadow = counts[5];
        st.launches = c->rs.launches;
        *stats = st;
    }
    return LUC_OK;
}

int32_t luc_batch_autotune(luc_ctx* c, const luc_batch_job* jobs, uint32_t n, uint32_t waves, luc_batch_config* best,
                           double* tried) {
    if (!c || !best) return LUC_ERR_VALIDATION;
    cudaSetDevice(c->device);
    if (int32_t rc = validate(c, jobs, n)) return rc;
    if (waves == 0) return luc_fail(c, LUC_ERR_VALIDATION, "waves must be positive");
    Plan pl = make_plan(jobs, n, c->path_budget, waves);
    // Scratch accumulators for the jobs the calibration touches.
    std::vector<luc_batch_job> scratch(jobs, jobs + n);
    std::vector<uint64_t> off(n, 0);
    uint64_t bytes = 0;
    for (uint32_t j = 0; j < n; ++j) {
        off[j] = bytes;
        bytes += (uint64_t)jobs[j].uniforms.width * jobs[j].uniforms.height * sizeof(GpuAccum);
        uint64_t last = 0;
        for (const BatchSegDev& sg : pl.segs)
            if (sg.job == j) last = 1;
        if (!last) bytes = off[j];  // untouched by the calibration waves
    }
    LUC_CUDA(c, c->b_scratch.ensure(std::max<uint64_t>(bytes, 256)), "alloc autotune scratch");
    for (uint32_t j = 0; j < n; ++j) scratch[j].accum_dev = (char*)c->b_scratch.p + off[j];
    const uint32_t blocks[3] = {64, 128, 256}, chunks[4] = {32, 1024, 4096, 16384};
    double best_ms = 1e300;
    std::vector<double> wave_ms;
    int k = 0;
    for (uint32_t b : blocks) {
        for (uint32_t ch : chunks) {
            double ms = 0.0;
            if (int32_t rc = run_plan(c, scratch.data(), n, pl, b, ch, wave_ms, &ms)) return rc;
            if (tried) {
                tried[3 * k] = b;
                tried[3 * k + 1] = ch;
                tried[3 * k + 2] = ms;
            }
            ++k;
            if (ms < best_ms) {
                best_ms = ms;
                *best = luc_batch_config{b, ch};
            }
        }
    }
    c->batch_block = best->block;
    c->batch_chunk = best->chunk;
    return LUC_OK;
}

}  // extern "C"
