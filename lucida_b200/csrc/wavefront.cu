// Wavefront path integrator on sm_100a: GENERATE -> (EXTEND -> SHADE ->
// CONNECT) x max_depth -> RESOLVE, the stage split of Lucida's
// crates/gpu/src/wavefront.rs:152-676 with the per-path semantics of the CPU
// reference integrator (crates/core/src/integrator.rs:209-589).
//
// Design (B200-first, not a translation of the WGSL):
//   * path state is SoA in HBM, one 16-byte float4 per field, so every stage
//     does 128-bit coalesced loads/stores; the whole spp x pixel pool is in
//     flight at once when it fits (a 1024^2 x 16 spp frame is 3.4 GB);
//   * stages are persistent grid-stride kernels sized to the SM count; queue
//     lengths live on the device and are read by the next stage, so the host
//     never synchronises inside a frame and the whole frame is captured into
//     one CUDA graph;
//   * SHADE compacts survivors and shadow rays with warp-aggregated atomics
//     (one atomicAdd per warp, ballot + popc for the slot);
//   * CONNECT adds each shadow ray's contribution into its own path (one
//     shadow ray per path per bounce), so no atomics and the radiance sum keeps
//     the CPU's accumulation order: emission(d), NEE(d), emission(d+1), ...;
//   * RESOLVE sums a pixel's samples in sample order onto the accumulator,
//     which makes batched and progressive renders bit-identical to one shot.
#include <type_traits>

#include "ctx.cuh"
#include "shade.cuh"

namespace luc {

// Path-state records are touched once per stage and the pool is far larger
// than L2: load and store them evict-first (ld/st.global.cs) so the BVH nodes
// and the triangle soup the traversal re-reads stay L2-resident.
__device__ __forceinline__ void store4(float4* p, V3 v, float w) { __stcs(p, make_float4(v.x, v.y, v.z, w)); }
__device__ __forceinline__ float4 ld4(const float4* p) { return __ldcs(p); }

// One atomic per warp: fold this thread's traversal counters into stat[k..k+2].
// stat: rays, node visits, triangle tests; blas_slot: BLAS entries.
__device__ __forceinline__ void flush_counts(unsigned long long* stat, unsigned long long* blas_slot, uint32_t rays,
                                             const TravCount& tc) {
    unsigned long long r = rays, nv = tc.nodes, tt = tc.tris, nb = tc.blas;
    for (int off = 16; off > 0; off >>= 1) {
        r += __shfl_down_sync(0xFFFFFFFFu, r, off);
        nv += __shfl_down_sync(0xFFFFFFFFu, nv, off);
        tt += __shfl_down_sync(0xFFFFFFFFu, tt, off);
        nb += __shfl_down_sync(0xFFFFFFFFu, nb, off);
    }
    if ((threadIdx.x & 31u) == 0 && r) {
        atomicAdd(stat + 0, r);
        atomicAdd(stat + 1, nv);
        atomicAdd(stat + 2, tt);
        if (nb) atomicAdd(blas_slot, nb);
    }
}
__device__ __forceinline__ V3 xyz(float4 a) { return V3{a.x, a.y, a.z}; }

// GENERATE (shaders/wavefront/generate.wgsl:35-88; camera.rs:373-405).
// Camera ray and sampler state of path p: pixel `pixel`, sample `sample`.
__device__ __forceinline__ void generate_one(PathState& ps, const FrameParams& fp, uint64_t p, uint32_t pixel,
                                             uint32_t sample) {
    Sampler smp = make_sampler(fp.sampler_kind, fp.frame_seed, pixel, sample);
    V3 origin, dir;
    camera_ray(fp, pixel, smp, origin, dir);
    store4(ps.o_pdf + p, origin, 0.0f);
    store4(ps.dir + p, dir, 0.0f);
    __stcs(ps.thr + p, make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(smp.state)));
    __stcs(ps.rad + p, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    store4(ps.prev + p, origin, 0.0f);
    if (fp.guides) {
        ps.galb[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        ps.gnrm[p] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

__global__ void __launch_bounds__(256) k_generate(PathState ps, FrameParams fp) {
    const uint64_t n = fp.num_paths;
    const uint32_t sbase = *fp.sbase;
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x)
        generate_one(ps, fp, p, (uint32_t)(p % fp.pixels), sbase + (uint32_t)(p / fp.pixels));
}

// The last segment whose first path is <= p (segments sorted by `first`).
__device__ __forceinline__ uint32_t find_segment(const BatchDev& bd, uint32_t p) {
    uint32_t lo = 0, hi = bd.num_segs;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (bd.segs[mid].first <= p) lo = mid;
        else hi = mid;
    }
    return lo;
}

// GENERATE of a batched wave: every path learns its segment (job, sample).
__global__ void __launch_bounds__(256) k_generate_batch(PathState ps, BatchDev bd, uint32_t num_paths) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < num_paths; p += gridDim.x * blockDim.x) {
        const uint32_t s = find_segment(bd, p);
        const BatchSegDev sg = bd.segs[s];
        const FrameParams& fp = bd.jobs[sg.job].fp;
        const uint32_t q = p - sg.first;
        ps.seg[p] = s;
        generate_one(ps, fp, p, q % fp.pixels, sg.sample_base + q / fp.pixels);
    }
}

// EXTEND (shaders/wavefront/extend.wgsl:35-68): closest hit per queued path.
// Persistent ray pull: each warp claims 32 queue entries at a time from the
// depth's cursor until the queue is drained, so fast warps keep taking work
// instead of idling behind slow ones; with bd.chunk > 32 (batched renders,
// chosen by the autotuner) a whole CTA claims `chunk` entries per pull.
// kBatch: each ray's scene comes from its path's wave segment.
// Wide-tree traversal runs at 32 warps per SM (64 registers): the loop is
// latency-bound, and occupancy beat the registers the compiler would take.
constexpr int wide_min_blocks(int threads) { return 1024 / threads; }
// k_extend_dyn refills a warp's finished lanes once this many are idle
// (measured best against 1, 16 and 32).
constexpr int kExtendRefill = 8;
// Blocks of 128 threads per SM for the two-level dynamic-fetch walks (64
// registers) and their refill threshold: the instanced frame (4096
// instances, 8 frames) ran 64.4 / 64.6 / 70.2 / 73.0 / 68.0 Mpaths/s at 6 / 5
// / 7 / 8 / 10 blocks, and at 8 blocks 73.5 refilling at 4 idle lanes (8:
// 73.0; 16 at 6 blocks: 61.6).
constexpr int kInstDynBlocks = 8;
constexpr int kInstRefill = 4;
// Entries of the walks' node-group stacks kept in shared memory (the rest in
// local memory, which competes with the tree for L1). Single-level walks: the
// displaced-sphere frame ran 394.0 / 428.6 / 430.9 / 428.8 Mpaths/s with 0 /
// 4 / 8 / 16 entries. Two-level walks keep theirs in local memory: with 4 /
// 8 / 16 BLAS entries in shared memory the instanced frame ran 69.4 / 68.3 /
// 67.2 Mpaths/s against 72.3 (its three-million-triangle BLASes need the L1),
// and a TLAS stack in shared memory spilled registers.
constexpr int kWalkSharedStack = 8;
constexpr int kBlasSharedStack = 0;
constexpr int kTlasSharedStack = 0;
template <int kThreads, bool kAny, int kInst>
using DynWalk = std::conditional_t<
    kInst == 2,
    InstWalkW<kAny, GroupStack<kTlasSharedStack, kThreads, kTlasStack>, GroupStack<kBlasSharedStack, kThreads, kWideStack>>,
    std::conditional_t<kInst == 1, InstWalk<kAny>, WideWalkT<GroupStack<kWalkSharedStack, kThreads, kWideStack>>>>;


// Two-level closest-hit walks (kInst) at 28 warps per SM (72 registers): the
// instanced frame's EXTEND took 602 ms at 32 warps (spilling) and 574 at 28.
template <bool kInst, bool kBatch, int kThreads, int kWide>
__global__ void __launch_bounds__(kThreads, kWide == 1 ? (kInst ? 7 * 128 / kThreads : wide_min_blocks(kThreads)) : 1) k_extend(PathState ps, const __grid_constant__ DevScene sc_arg, FrameParams fp,
                                                     BatchDev bd, uint32_t depth) {
    const uint32_t len = depth == 0 ? (uint32_t)fp.num_paths : ps.ctr[depth * kCtrStride + kCtrQueue];
    const uint32_t* queue = ps.queue[depth & 1];
    uint32_t* pull = ps.ctr + depth * kCtrStride + kCtrPullExtend;
    const uint32_t lane = threadIdx.x & 31u;
    TravCount tc;
    uint32_t rays = 0;
    auto trace = [&](uint32_t i) {
        uint32_t p = depth == 0 ? i : queue[i];
        float4 o4 = ld4(ps.o_pdf + p), d4 = ld4(ps.dir + p);
        const DevScene& sc = kBatch ? bd.scenes[bd.segs[ps.seg[p]].scene] : sc_arg;
        float t, u, v;
        uint32_t inst;
        uint32_t id = closest_hit<kInst, kWide>(sc, xyz(o4), xyz(d4), t, u, v, inst, tc);
        __stcs(ps.hit + p, make_float4(t, u, v, __uint_as_float(id)));
        if (kInst) ps.hinst[p] = inst;
        ++rays;
    };
    if (kBatch && bd.chunk > 32u) {
        __shared__ uint32_t cta_base;
        for (;;) {
            if (threadIdx.x == 0) cta_base = atomicAdd(pull, bd.chunk);
            __syncthreads();
            const uint32_t cb = cta_base;
            __syncthreads();
            if (cb >= len) break;
            const uint32_t end = min(cb + bd.chunk, len);
            for (uint32_t i = cb + threadIdx.x; i < end; i += kThreads) trace(i);
        }
    } else {
        for (;;) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(pull, 32u);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base >= len) break;
            if (base + lane < len) trace(base + lane);
            __syncwarp();
        }
    }
    flush_counts(ps.stat, ps.stat + 6, rays, tc);
}

// EXTEND on the wide tree of a single-level scene, with dynamic ray fetch
// (Aila and Laine 2009; Aila, Laine and Karras 2012): each warp walks 32
// rays one node at a time and, whenever at least kRefill lanes have finished,
// refills them with the next rays of the queue (one atomic per refill), so
// lanes do not idle until the warp's longest ray ends. Each ray's walk is
// wide_trace's (WideWalk), so the hits are the same.
// kStage > 0: the first kStage wide nodes (the top levels) are copied into
// shared memory when the block starts and read from there.
// kInst: a two-level scene whose BLASes have wide trees, walked a step at a
// time: 1 by InstWalk (binary TLAS), 2 by InstWalkW (8-wide TLAS).
template <int kThreads, int kRefill, int kStage = 0, int kInst = 0>
__global__ void __launch_bounds__(kThreads, kInst ? kInstDynBlocks * 128 / kThreads : wide_min_blocks(kThreads))
    k_extend_dyn(PathState ps, const __grid_constant__ DevScene sc, FrameParams fp, uint32_t depth) {
    __shared__ float4 stage[kStage > 0 ? 5 * kStage : 1];
    if (kStage > 0) {
        const uint32_t nf4 = 5 * min((uint32_t)kStage, sc.num_wnodes);
        for (uint32_t i = threadIdx.x; i < nf4; i += kThreads) stage[i] = __ldg(sc.wnodes + i);
        __syncthreads();
    }
    const uint32_t len = depth == 0 ? (uint32_t)fp.num_paths : ps.ctr[depth * kCtrStride + kCtrQueue];
    const uint32_t* queue = ps.queue[depth & 1];
    uint32_t* pull = ps.ctr + depth * kCtrStride + kCtrPullExtend;
    const uint32_t lane = threadIdx.x & 31u, below = (1u << lane) - 1u;
    TravCount tc;
    uint32_t rays = 0, p = 0, pid = kMiss;
    bool live = false, exhausted = false;
    constexpr int kShared = kInst == 0 ? kWalkSharedStack : kInst == 2 ? kBlasSharedStack : 0;
    __shared__ uint2 s_stack[kShared > 0 ? kShared : 1][kThreads];
    __shared__ uint2 s_tstack[kInst == 2 && kTlasSharedStack > 0 ? kTlasSharedStack : 1][kThreads];
    DynWalk<kThreads, false, kInst> w;
    w.bind(&s_stack[0][threadIdx.x], &s_tstack[0][threadIdx.x]);
    for (;;) {
        const uint32_t need = __ballot_sync(0xFFFFFFFFu, !live);
        if (!exhausted && __popc(need) >= kRefill) {
            const uint32_t leader = __ffs(need) - 1u, n = __popc(need);
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(pull, n);
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            exhausted = base + n >= len;
            if (!live) {
                const uint32_t i = base + __popc(need & below);
                if (i < len) {
                    p = depth == 0 ? i : queue[i];
                    const V3 o = xyz(ld4(ps.o_pdf + p)), d = xyz(ld4(ps.dir + p));
                    float best_t = kTMax;
                    pid = kMiss;
                    analytic_closest(sc, o, d, best_t, pid);  // Scene::intersect: primitives first
                    if constexpr (kInst != 0) w.begin(sc, o, d, best_t);
                    else w.begin(0u, o, d, best_t);
                    live = true;
                }
            }
        }
        if (__ballot_sync(0xFFFFFFFFu, live) == 0) {
            if (exhausted) break;
            continue;
        }
        // One node per refill check (measured best against 4, 8 and 16).
        bool over = false;
        if constexpr (kInst != 0) over = live && w.step(sc, kTMin, tc);
        else over = live && w.template step<false, kStage>(sc, kTMin, tc, stage);
        if (over) {
            __stcs(ps.hit + p, make_float4(w.tmax, w.found ? w.bu : 0.0f, w.found ? w.bv : 0.0f,
                                           __uint_as_float(w.found ? w.btri : pid)));
            if constexpr (kInst != 0) ps.hinst[p] = w.found ? w.binst : 0u;
            ++rays;
            live = false;
        }
    }
    flush_counts(ps.stat, ps.stat + 6, rays, tc);
}

// CONNECT on the wide tree of a single-level scene with the same dynamic
// ray fetch as k_extend_dyn: any-hit walks end at their first hit, so their
// lengths vary even more than closest-hit walks, and a warp that waited for
// its longest shadow ray idled most of its lanes. Each ray's walk is
// wide_trace<true>'s (WideWalk), after the analytic primitives (occluded()'s
// order), so the visibility and the counters are the same.
template <int kThreads, int kRefill, int kInst = 0>
__global__ void __launch_bounds__(kThreads, kInst ? kInstDynBlocks * 128 / kThreads : wide_min_blocks(kThreads))
    k_connect_dyn(PathState ps, const __grid_constant__ DevScene sc, uint32_t depth) {
    const uint32_t len = ps.ctr[depth * kCtrStride + kCtrShadow];
    uint32_t* pull = ps.ctr + depth * kCtrStride + kCtrPullConnect;
    const uint32_t lane = threadIdx.x & 31u, below = (1u << lane) - 1u;
    TravCount tc;
    uint32_t rays = 0, slot = 0;
    bool live = false, exhausted = false;
    constexpr int kShared = kInst == 0 ? kWalkSharedStack : kInst == 2 ? kBlasSharedStack : 0;
    __shared__ uint2 s_stack[kShared > 0 ? kShared : 1][kThreads];
    __shared__ uint2 s_tstack[kInst == 2 && kTlasSharedStack > 0 ? kTlasSharedStack : 1][kThreads];
    DynWalk<kThreads, true, kInst> w;
    w.bind(&s_stack[0][threadIdx.x], &s_tstack[0][threadIdx.x]);
    auto finish = [&](bool occluded) {
        if (!occluded) {
            const uint32_t p = __float_as_uint(ld4(ps.sh_d + slot).w);
            const float4 c4 = ld4(ps.sh_c + slot), r4 = ld4(ps.rad + p);
            __stcs(ps.rad + p, make_float4(r4.x + c4.x, r4.y + c4.y, r4.z + c4.z, 0.0f));
        }
        ++rays;
        live = false;
    };
    for (;;) {
        const uint32_t need = __ballot_sync(0xFFFFFFFFu, !live);
        if (!exhausted && __popc(need) >= kRefill) {
            const uint32_t leader = __ffs(need) - 1u, n = __popc(need);
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(pull, n);
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            exhausted = base + n >= len;
            if (!live) {
                const uint32_t i = base + __popc(need & below);
                if (i < len) {
                    slot = i;
                    const float4 o4 = ld4(ps.sh_o + i), d4 = ld4(ps.sh_d + i);
                    const V3 o = xyz(o4), d = xyz(d4);
                    live = true;
                    if (analytic_any(sc, o, d, o4.w)) finish(true);
                    else if constexpr (kInst != 0) w.begin(sc, o, d, o4.w);
                    else w.begin(0u, o, d, o4.w);
                }
            }
        }
        if (__ballot_sync(0xFFFFFFFFu, live) == 0) {
            if (exhausted) break;
            continue;
        }
        bool over = false;
        if constexpr (kInst != 0) over = live && w.step(sc, kTMin, tc);
        else over = live && w.template step<true>(sc, kTMin, tc);
        if (over) finish(w.found);
    }
    flush_counts(ps.stat + 3, ps.stat + 7, rays, tc);
}

// Warp-aggregated append: one atomicAdd per warp. Every lane of the warp must
// call this (it uses full-warp ballots).
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool pred) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t mask = __ballot_sync(0xFFFFFFFFu, pred);
    if (mask == 0) return 0xFFFFFFFFu;
    uint32_t leader = __ffs(mask) - 1u;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    return pred ? base + (uint32_t)__popc(mask & ((1u << lane) - 1u)) : 0xFFFFFFFFu;
}

// SHADE's sink for shade_vertex: the path pool. The path's next ray and the
// first-hit guides are stored where they are computed; the shadow ray waits
// in registers for the warp-aggregated append at the end of the step.
// Guided frames also write the vertex's training record (a threshold-
// selected subset of the candidates, warp-aggregated counters).
template <bool kGuided>
struct PoolSink {
    const PathState& ps;
    const Sampler& smp;
    uint32_t p, depth, sbase, rec_threshold, rec_cap;
    V3 dir_in;
    bool survive = false, cast = false;
    V3 sh_o{0, 0, 0}, sh_d{0, 0, 0}, sh_c{0, 0, 0};
    float sh_t = 0.0f;
    __device__ PoolSink(const PathState& ps_, uint32_t p_, uint32_t depth_, uint32_t sbase_, uint32_t thr_,
                        uint32_t cap_, V3 dir_, const Sampler& smp_)
        : ps(ps_), smp(smp_), p(p_), depth(depth_), sbase(sbase_), rec_threshold(thr_), rec_cap(cap_), dir_in(dir_) {}
    __device__ __forceinline__ V3 prev() const { return xyz(ps.prev[p]); }
    __device__ __forceinline__ void guides(V3 albedo, float t, V3 normal) {
        store4(ps.galb + p, albedo, t);
        store4(ps.gnrm + p, normal, 0.0f);
    }
    __device__ __forceinline__ void shadow(V3 o, V3 d, float t_max, V3 c) {
        cast = true;
        sh_o = o;
        sh_d = d;
        sh_t = t_max;
        sh_c = c;
    }
    __device__ __forceinline__ void next(V3 norg, V3 ndir, float npdf, V3 thr, V3 hit_pos, V3 hit_nrm, bool record,
                                         V3 rad) {
        store4(ps.o_pdf + p, norg, npdf);
        store4(ps.dir + p, ndir, 0.0f);
        __stcs(ps.thr + p, make_float4(thr.x, thr.y, thr.z, __uint_as_float(smp.state)));
        uint32_t slot1 = 0u;
        if (kGuided && record) {
            // Opportunistic warp aggregation of the two counters.
            const uint32_t lane = threadIdx.x & 31u;
            uint32_t am = __activemask();
            uint32_t leader = __ffs(am) - 1u;
            if (lane == leader) atomicAdd(ps.gmisc + kGmCandidates, (uint32_t)__popc(am));
            uint32_t h = mix32(p * 0x9E3779B9u ^ (depth << 27) ^ (sbase * 0x85EBCA6Bu));
            const bool want = (h & 0xFFFFu) < rec_threshold;
            uint32_t wm = __ballot_sync(am, want);
            if (want) {
                uint32_t wl0 = __ffs(wm) - 1u, base = 0;
                if (lane == wl0) base = atomicAdd(ps.gmisc + kGmRecords, (uint32_t)__popc(wm));
                base = __shfl_sync(wm, base, wl0);
                const uint32_t slot = base + (uint32_t)__popc(wm & ((1u << lane) - 1u));
                if (slot < rec_cap) {
                    float4* r = ps.rec + kGRecF4 * (size_t)slot;
                    r[0] = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, __uint_as_float(p));
                    r[1] = make_float4(hit_nrm.x, hit_nrm.y, hit_nrm.z, thr.x);
                    r[2] = make_float4(-dir_in.x, -dir_in.y, -dir_in.z, thr.y);
                    r[3] = make_float4(ndir.x, ndir.y, ndir.z, thr.z);
                    r[4] = make_float4(rad.x, rad.y, rad.z, npdf);
                    slot1 = slot + 1u;
                }
            }
        }
        store4(ps.prev + p, hit_pos, __uint_as_float(slot1));
        survive = true;
    }
};

// SHADE (shaders/wavefront/shade.wgsl:119-348), one bounce of
// integrator.rs:227-400 per queued path.
//
// kGuided: one-sample MIS between the BSDF and the learned mixture at opaque,
// non-specular vertices (selection fraction 0.5 each, one extra dimension for
// the choice), with p = 0.5 p_bsdf + 0.5 p_guide as the path's sampling pdf in
// both MIS sites (emission hit and NEE); plus training records for a
// threshold-selected subset of those vertices.
//
// kBatch: the path's scene and frame parameters come from its wave segment
// (luc_render_batch) instead of the kernel arguments.
//
// 6 blocks of 128 per SM (80 registers, about 450 bytes spilled). SHADE is bound by the latency of its
// path-state, triangle and material loads. When it shaded escaped rays too,
// 8 blocks (64 registers, about 700 bytes spilled to L1) ran best (7 -> 8:
// 16.0 -> 15.5 ms per displaced-sphere frame); with the hits alone, split by
// material class, and the traversal stacks partly in shared memory, 6 blocks
// run 9.42 ms against 9.78 at 8 and 9.58 at 7.
// kSobol (launched only for Sobol frames) and kSkyMis (MIS frames of scenes
// lit only by an environment map): the code of the other cases is compiled
// out of the kernel whose top stall is instruction fetch (displaced-sphere
// frame: SHADE 15.6 ms generic, 14.7 with kSobol and no light sampling,
// 14.4 with MIS and the environment fixed too).
template <bool kGuided, bool kInst, bool kBatch = false, bool kSobol = false, bool kSkyMis = false>
__global__ void __launch_bounds__(128, 6) k_shade(PathState ps, const __grid_constant__ DevScene sc_arg,
                                                  const __grid_constant__ FrameParams fp_arg, BatchDev bd,
                                                  uint32_t depth) {
    const uint32_t len = shaded_count(ps, fp_arg, depth);
    const uint32_t rec_threshold = kGuided ? ps.gmisc[kGmThreshold] : 65536u;
    const uint32_t sbase_arg = kBatch ? 0u : *fp_arg.sbase;
    uint32_t* next_queue = ps.queue[(depth + 1) & 1];
    uint32_t* next_len = ps.ctr + (depth + 1) * kCtrStride + kCtrQueue;
    uint32_t* shadow_len = ps.ctr + depth * kCtrStride + kCtrShadow;
    const uint32_t stride = gridDim.x * blockDim.x;
    // Warp-uniform trip count so the ballots below see every lane.
    const uint32_t warp0 = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u;
    for (uint32_t base = warp0; base < len; base += stride) {
        const uint32_t i = base + (threadIdx.x & 31u);
        bool active = i < len;
        bool survive = false, cast = false;
        uint32_t p = 0;
        V3 sh_o{0, 0, 0}, sh_d{0, 0, 0}, sh_c{0, 0, 0};
        float sh_t = 0.0f;
        if (active) {
            p = shaded_path(ps, fp_arg, depth, i);
            const BatchSegDev* seg = kBatch ? bd.segs + ps.seg[p] : nullptr;
            const BatchJobDev* job = kBatch ? bd.jobs + seg->job : nullptr;
            const DevScene& sc = kBatch ? bd.scenes[job->scene] : sc_arg;
            const FrameParams& fp = kBatch ? job->fp : fp_arg;
            const uint32_t sbase = kBatch ? seg->sample_base : sbase_arg;
            const uint32_t q = kBatch ? p - seg->first : p;  // path index within its own frame
            float4 o4 = ld4(ps.o_pdf + p), d4 = ld4(ps.dir + p), h4 = ld4(ps.hit + p), t4 = ld4(ps.thr + p),
                   r4 = ld4(ps.rad + p);
            const V3 dir = xyz(d4);
            V3 rad = xyz(r4);
            uint32_t pixel = (uint32_t)(q % fp.pixels);
            Sampler smp;
            smp.kind = kSobol ? LUC_SAMPLER_SOBOL : fp.sampler_kind;
            smp.state = __float_as_uint(t4.w);
            smp.index = sbase + (uint32_t)(q / fp.pixels);
            smp.seed = sobol_pixel_seed(pixel, fp.frame_seed);
            if (kGuided) {
                // The record made at the previous vertex (slot + 1 in prev.w)
                // starts its incident-radiance estimate here.
                const uint32_t slot1 = __float_as_uint(ps.prev[p].w);
                if (slot1 != 0u) {
                    float* rs = reinterpret_cast<float*>(ps.rec + kGRecF4 * (size_t)(slot1 - 1u) + 4);
                    rs[0] = rad.x;
                    rs[1] = rad.y;
                    rs[2] = rad.z;
                }
            }
            PoolSink<kGuided> sink(ps, p, depth, sbase, rec_threshold, fp.rec_cap, dir, smp);
            if (shade_vertex<kGuided, kInst, kSkyMis>(sc, fp, depth, smp, xyz(o4), dir, xyz(t4), rad, o4.w, h4,
                                             kInst ? ps.hinst[p] : 0u, ps.lobes + i, ps.lobe_stride, sink))
                store4(ps.rad + p, rad, 0.0f);
            survive = sink.survive;
            if (sink.cast) {
                cast = true;
                sh_o = sink.sh_o;
                sh_d = sink.sh_d;
                sh_t = sink.sh_t;
                sh_c = sink.sh_c;
            }
        }
        uint32_t slot = warp_append(next_len, survive);
        if (survive) next_queue[slot] = p;
        uint32_t sslot = warp_append(shadow_len, cast);
        if (cast) {
            store4(ps.sh_o + sslot, sh_o, sh_t);
            store4(ps.sh_d + sslot, sh_d, __uint_as_float(p));
            store4(ps.sh_c + sslot, sh_c, 0.0f);
        }
    }
}

// Split frames: this depth's extended paths into hit queues by material
// class and the escaped queue, so that SHADE's warps run hits only, mostly
// of one class (the BSDF's lobe choice and sampling code follow the class),
// and escaped rays are shaded apart (k_escape): a warp mixing the two ran
// the short escape code and the long surface code one after the other.
// Appends are aggregated per block of kClassifyItems x 256 paths (one atomic
// per queue per block): with one per warp the counters' atomics bounded the
// kernel.
constexpr int kClassifyItems = 8;
// Material class of a hit: 0 reflective non-metal, 1 metal, 2 transmissive
// (the lobes make_surface enables).
LUC_D uint32_t hit_class(const DevScene& sc, const PathState& ps, uint32_t p, uint32_t id) {
    uint32_t m;
    if (id & kAnalytic) {
        m = __ldg(&sc.prims[id & ~kAnalytic].material);
    } else {
        m = __ldg(&sc.tris[id].material);
        if (sc.num_instances) {
            const uint32_t o = __ldg(&sc.inst[ps.hinst[p]].material);
            if (o != 0xFFFFFFFFu) m = o;
        }
    }
    const float metallic = clampf(__ldg(&sc.materials[m].metallic), 0.0f, 1.0f);
    const float transmission = clampf(__ldg(&sc.materials[m].transmission), 0.0f, 1.0f) * (1.0f - metallic);
    return transmission > 0.0f ? 2u : (metallic >= 0.5f ? 1u : 0u);
}
__global__ void __launch_bounds__(256) k_classify(PathState ps, const __grid_constant__ DevScene sc, FrameParams fp,
                                                  uint32_t depth) {
    constexpr uint32_t kPerBlock = 256u * kClassifyItems;
    __shared__ uint32_t s_cnt[4][8];  // per warp: hits of class 0, 1, 2, escapes
    __shared__ uint32_t s_base[4];
    const uint32_t len = depth == 0 ? (uint32_t)fp.num_paths : ps.ctr[depth * kCtrStride + kCtrQueue];
    const uint32_t* queue = ps.queue[depth & 1];
    uint32_t* ctr = ps.ctr + depth * kCtrStride;
    uint32_t* out[4] = {ps.hitq[0], ps.hitq[1], ps.hitq[2], ps.missq};
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, lt = (1u << lane) - 1u;
    for (uint32_t base = blockIdx.x * kPerBlock; base < len; base += gridDim.x * kPerBlock) {
        uint32_t p[kClassifyItems], cls[kClassifyItems];
        uint32_t n[4] = {0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < kClassifyItems; ++k) {
            const uint32_t i = base + (uint32_t)k * 256u + tid;
            const bool active = i < len;
            p[k] = active ? (depth == 0 ? i : queue[i]) : 0u;
            cls[k] = 4u;  // inactive
            if (active) {
                const uint32_t id = __float_as_uint(__ldcs(&ps.hit[p[k]].w));
                cls[k] = id == kMiss ? 3u : hit_class(sc, ps, p[k], id);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) n[q] += __popc(__ballot_sync(0xFFFFFFFFu, cls[k] == (uint32_t)q));
        }
        if (lane < 4) s_cnt[lane][warp] = n[lane];
        __syncthreads();
        if (tid < 4) {
            uint32_t t = 0;
            for (int w = 0; w < 8; ++w) {
                const uint32_t c = s_cnt[tid][w];
                s_cnt[tid][w] = t;
                t += c;
            }
            s_base[tid] = t ? atomicAdd(ctr + (tid < 3 ? hit_slot(tid) : kCtrMiss), t) : 0u;
        }
        __syncthreads();
        uint32_t off[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) off[q] = s_base[q] + s_cnt[q][warp];
#pragma unroll
        for (int k = 0; k < kClassifyItems; ++k) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t b = __ballot_sync(0xFFFFFFFFu, cls[k] == (uint32_t)q);
                if (cls[k] == (uint32_t)q) out[q][off[q] + __popc(b & lt)] = p[k];
                off[q] += __popc(b);
            }
        }
        __syncthreads();  // s_cnt / s_base are rewritten by the next round
    }
}

// Split frames: the escaped paths of this depth, shaded as SHADE shades a
// miss (escape_vertex), and in guided frames the training record of the
// previous vertex opened as SHADE opens it.
template <bool kGuided, bool kSkyMis>
__global__ void __launch_bounds__(256) k_escape(PathState ps, const __grid_constant__ DevScene sc,
                                                const __grid_constant__ FrameParams fp, uint32_t depth) {
    const uint32_t n = ps.ctr[depth * kCtrStride + kCtrMiss];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t p = ps.missq[i];
        const float4 o4 = ld4(ps.o_pdf + p), d4 = ld4(ps.dir + p), t4 = ld4(ps.thr + p), r4 = ld4(ps.rad + p);
        V3 rad = xyz(r4);
        if (kGuided) {
            const uint32_t slot1 = __float_as_uint(ps.prev[p].w);
            if (slot1 != 0u) {
                float* rs = reinterpret_cast<float*>(ps.rec + kGRecF4 * (size_t)(slot1 - 1u) + 4);
                rs[0] = rad.x;
                rs[1] = rad.y;
                rs[2] = rad.z;
            }
        }
        if (escape_vertex<kSkyMis>(sc, fp, depth, xyz(d4), xyz(t4), rad, o4.w)) store4(ps.rad + p, rad, 0.0f);
    }
}

// CONNECT (shaders/wavefront/connect.wgsl:58-84): any-hit shadow rays, with
// the same persistent ray pull as EXTEND. Two-level scenes use it when their
// walk cannot be stepped (binary BLASes, or the reference's object-space
// shadow rays); it runs at 32 warps per SM there too (the instanced frame's
// CONNECT took 133 ms unbounded with 82 registers at 24 warps, 110 at 28
// warps, 103 at 32, when it walked every instanced shadow ray).
template <bool kInst, bool kBatch, int kThreads, int kWide>
__global__ void __launch_bounds__(kThreads, kWide == 1 || kInst ? wide_min_blocks(kThreads) : 1) k_connect(PathState ps, const __grid_constant__ DevScene sc_arg, BatchDev bd,
                                                      uint32_t depth) {
    const uint32_t len = ps.ctr[depth * kCtrStride + kCtrShadow];
    uint32_t* pull = ps.ctr + depth * kCtrStride + kCtrPullConnect;
    const uint32_t lane = threadIdx.x & 31u;
    TravCount tc;
    uint32_t rays = 0;
    auto trace = [&](uint32_t i) {
        float4 o4 = ld4(ps.sh_o + i), d4 = ld4(ps.sh_d + i);
        uint32_t p = __float_as_uint(d4.w);
        const DevScene& sc = kBatch ? bd.scenes[bd.segs[ps.seg[p]].scene] : sc_arg;
        if (!occluded<kInst, kWide>(sc, xyz(o4), xyz(d4), o4.w, tc)) {
            float4 c4 = ld4(ps.sh_c + i), r4 = ld4(ps.rad + p);
            __stcs(ps.rad + p, make_float4(r4.x + c4.x, r4.y + c4.y, r4.z + c4.z, 0.0f));
        }
        ++rays;
    };
    if (kBatch && bd.chunk > 32u) {
        __shared__ uint32_t cta_base;
        for (;;) {
            if (threadIdx.x == 0) cta_base = atomicAdd(pull, bd.chunk);
            __syncthreads();
            const uint32_t cb = cta_base;
            __syncthreads();
            if (cb >= len) break;
            const uint32_t end = min(cb + bd.chunk, len);
            for (uint32_t i = cb + threadIdx.x; i < end; i += kThreads) trace(i);
        }
    } else {
        for (;;) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(pull, 32u);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base >= len) break;
            if (base + lane < len) trace(base + lane);
            __syncwarp();
        }
    }
    flush_counts(ps.stat + 3, ps.stat + 7, rays, tc);
}

// RESOLVE (shaders/wavefront/resolve.wgsl:14-48): per pixel, this batch's
// samples in sample order, added one at a time onto the accumulator.
__global__ void __launch_bounds__(256) k_resolve(PathState ps, FrameParams fp, GpuAccum* accum) {
    for (uint32_t px = blockIdx.x * blockDim.x + threadIdx.x; px < fp.pixels; px += gridDim.x * blockDim.x) {
        GpuAccum a = accum[px];
        V3 r = ld3(a.radiance), r2 = ld3(a.radiance_sq), al = ld3(a.albedo), nn = ld3(a.normal);
        float dep = a.depth;
        for (uint32_t j = 0; j < fp.batch_samples; ++j) {
            uint64_t p = (uint64_t)px + (uint64_t)j * fp.pixels;
            V3 q = xyz(ps.rad[p]);
            r = r + q;
            r2 = r2 + q * q;
            if (fp.guides) {
                float4 g = ps.galb[p];
                al = al + xyz(g);
                dep = dep + g.w;
                nn = nn + xyz(ps.gnrm[p]);
            }
        }
        a.radiance[0] = r.x; a.radiance[1] = r.y; a.radiance[2] = r.z;
        a.radiance_sq[0] = r2.x; a.radiance_sq[1] = r2.y; a.radiance_sq[2] = r2.z;
        a.albedo[0] = al.x; a.albedo[1] = al.y; a.albedo[2] = al.z;
        a.normal[0] = nn.x; a.normal[1] = nn.y; a.normal[2] = nn.z;
        a.depth = dep;
        a.samples = a.samples + (float)fp.batch_samples;
        accum[px] = a;
    }
}

// RESOLVE of a batched wave: per (segment, pixel), the segment's samples in
// sample order onto its job's accumulator. Threads walk the wave's pixels
// segment after segment (pixel offsets are prefix sums over segments).
__global__ void __launch_bounds__(256) k_resolve_batch(PathState ps, BatchDev bd, const uint32_t* __restrict__ pix_off,
                                                       uint32_t total_pixels) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total_pixels; t += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = bd.num_segs;
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (pix_off[mid] <= t) lo = mid;
            else hi = mid;
        }
        const BatchSegDev sg = bd.segs[lo];
        const BatchJobDev& job = bd.jobs[sg.job];
        const uint32_t px = t - pix_off[lo], pixels = job.fp.pixels;
        GpuAccum a = job.accum[px];
        V3 r = ld3(a.radiance), r2 = ld3(a.radiance_sq), al = ld3(a.albedo), nn = ld3(a.normal);
        float dep = a.depth;
        for (uint32_t j = 0; j < sg.nsamples; ++j) {
            uint64_t p = (uint64_t)sg.first + px + (uint64_t)j * pixels;
            V3 q = xyz(ps.rad[p]);
            r = r + q;
            r2 = r2 + q * q;
            if (job.fp.guides) {
                float4 g = ps.galb[p];
                al = al + xyz(g);
                dep = dep + g.w;
                nn = nn + xyz(ps.gnrm[p]);
            }
        }
        a.radiance[0] = r.x; a.radiance[1] = r.y; a.radiance[2] = r.z;
        a.radiance_sq[0] = r2.x; a.radiance_sq[1] = r2.y; a.radiance_sq[2] = r2.z;
        a.albedo[0] = al.x; a.albedo[1] = al.y; a.albedo[2] = al.z;
        a.normal[0] = nn.x; a.normal[1] = nn.y; a.normal[2] = nn.z;
        a.depth = dep;
        a.samples = a.samples + (float)sg.nsamples;
        job.accum[px] = a;
    }
}

// Traversal layout (see scene_dev.cuh): child-pair records per internal
// node and the (p0, e1, e2) triangle soup.
__global__ void k_make_tnodes(const float4* __restrict__ nodes, uint32_t begin, uint32_t end, float4* __restrict__ tn) {
    for (uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
        float4 b = nodes[2 * i + 1];
        if (__float_as_uint(b.w) != 0u) continue;  // leaves have no record
        uint32_t c0 = __float_as_uint(nodes[2 * i].w);
        float4 a0 = nodes[2 * c0], b0 = nodes[2 * c0 + 1], a1 = nodes[2 * c0 + 2], b1 = nodes[2 * c0 + 3];
        uint32_t n0 = __float_as_uint(b0.w), n1 = __float_as_uint(b1.w);
        float4* o = tn + 4 * (size_t)i;
        o[0] = make_float4(a0.x, a0.y, a0.z, b0.x);
        o[1] = make_float4(b0.y, b0.z, a1.x, a1.y);
        o[2] = make_float4(a1.z, b1.x, b1.y, b1.z);
        uint4 r = make_uint4(n0 ? __float_as_uint(a0.w) : c0, n0, n1 ? __float_as_uint(a1.w) : c0 + 1, n1);
        reinterpret_cast<uint4*>(o)[3] = r;
    }
}
__global__ void k_make_soup(const GpuTriangle* __restrict__ tris, const float4* __restrict__ pos, uint32_t n,
                            float4* __restrict__ soup) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        GpuTriangle t = tris[k];
        float4 p0 = pos[t.i0], p1 = pos[t.i1], p2 = pos[t.i2];
        soup[3 * (size_t)k] = make_float4(p0.x, p0.y, p0.z, 0.0f);
        soup[3 * (size_t)k + 1] = make_float4(p1.x - p0.x, p1.y - p0.y, p1.z - p0.z, 0.0f);
        soup[3 * (size_t)k + 2] = make_float4(p2.x - p0.x, p2.y - p0.y, p2.z - p0.z, 0.0f);
    }
}

void query_occupancy(RenderState& rs) {
    auto occ = [](const void* k) {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, 128, 0);
        return b > 0 ? b : 8;
    };
    rs.extend_blocks = occ((const void*)k_extend_dyn<128, kExtendRefill>);
    rs.extend_blocks_stage = occ((const void*)k_extend_dyn<128, kExtendRefill, 73>);
    rs.connect_blocks = occ((const void*)k_connect_dyn<128, kExtendRefill>);
    rs.extend_blocks_bin = occ((const void*)k_extend<false, false, 128, 0>);
    rs.connect_blocks_bin = occ((const void*)k_connect<false, false, 128, 0>);
    rs.shade_blocks = occ((const void*)k_shade<false, false>);
    rs.shade_blocks_guided = occ((const void*)k_shade<true, false>);
    rs.extend_blocks_inst = occ((const void*)k_extend_dyn<128, kInstRefill, 0, 2>);
    rs.connect_blocks_inst = occ((const void*)k_connect_dyn<128, kInstRefill, 2>);
    rs.extend_blocks_inst_bin = occ((const void*)k_extend<true, false, 128, 0>);
    rs.connect_blocks_inst_bin = occ((const void*)k_connect<true, false, 128, 0>);
    rs.shade_blocks_inst = occ((const void*)k_shade<false, true>);
    rs.shade_blocks_guided_inst = occ((const void*)k_shade<true, true>);
}

// SHADE of one bounce, specialised on the frame's sampler and on MIS frames
// of scenes lit only by their environment map.
template <bool kGuided, bool kInst>
void launch_shade(const RenderState& rs, int grid, const DevScene& sc, const FrameParams& fp, uint32_t d,
                  cudaStream_t s) {
    const bool sobol = fp.sampler_kind == LUC_SAMPLER_SOBOL;
    const bool sky_mis = fp.sampling == LUC_SAMPLING_MIS && sc.num_lights == 0 && sc.has_env;
    if (sobol && sky_mis)
        k_shade<kGuided, kInst, false, true, true><<<grid, 128, 0, s>>>(rs.ps, sc, fp, BatchDev{}, d);
    else if (sobol)
        k_shade<kGuided, kInst, false, true, false><<<grid, 128, 0, s>>>(rs.ps, sc, fp, BatchDev{}, d);
    else
        k_shade<kGuided, kInst><<<grid, 128, 0, s>>>(rs.ps, sc, fp, BatchDev{}, d);
}

// Host side: record one batch of the frame on `stream` (graph-capturable:
// fixed launch shapes, device-resident lengths).
void record_batch(RenderState& rs, const DevScene& sc, const FrameParams& fp, GpuAccum* accum, cudaStream_t stream,
                  StageTimer* timer, const GuideTrain* gt, const ConnectOverlap* ov) {
    const int sms = rs.num_sms;
    const uint32_t stride_ctr = kCtrStride * (fp.max_depth + 2);
    bool connect_out = false;  // a CONNECT on ov->side not yet waited for
    auto join_connect = [&]() {
        if (connect_out) cudaStreamWaitEvent(stream, ov->done, 0);
        connect_out = false;
    };
    cudaMemsetAsync(rs.ps.ctr, 0, stride_ctr * sizeof(uint32_t), stream);
    if (timer) timer->mark(stream, StageTimer::kGenerate);
    {
        uint64_t blocks = (fp.num_paths + 255) / 256;
        int grid = (int)std::min<uint64_t>(blocks, (uint64_t)sms * 16);
        k_generate<<<grid, 256, 0, stream>>>(rs.ps, fp);
        rs.launches++;
    }
    for (uint32_t d = 0; d < fp.max_depth; ++d) {
        if (timer) timer->mark(stream, StageTimer::kExtend);
        const bool inst = sc.num_instances > 0, wide = inst ? sc.blas_wide != nullptr : sc.wnodes != nullptr;
        if (inst && wide && sc.twnodes)
            k_extend_dyn<128, kInstRefill, 0, 2><<<sms * rs.extend_blocks_inst, 128, 0, stream>>>(rs.ps, sc, fp, d);
        else if (inst && wide)
            k_extend_dyn<128, kInstRefill, 0, 1><<<sms * rs.extend_blocks_inst, 128, 0, stream>>>(rs.ps, sc, fp, d);
        else if (inst)
            k_extend<true, false, 128, 0><<<sms * rs.extend_blocks_inst_bin, 128, 0, stream>>>(rs.ps, sc, fp,
                                                                                               BatchDev{}, d);
        else if (wide && rs.wide_stage == 73)
            k_extend_dyn<128, kExtendRefill, 73><<<sms * rs.extend_blocks_stage, 128, 0, stream>>>(rs.ps, sc, fp, d);
        else if (wide)
            k_extend_dyn<128, kExtendRefill><<<sms * rs.extend_blocks, 128, 0, stream>>>(rs.ps, sc, fp, d);
        else
            k_extend<false, false, 128, 0><<<sms * rs.extend_blocks_bin, 128, 0, stream>>>(rs.ps, sc, fp, BatchDev{}, d);
        if (fp.split) {
            k_classify<<<sms * 4, 256, 0, stream>>>(rs.ps, sc, fp, d);
            rs.launches++;
        }
        if (d == 0 && gt && gt->join) cudaStreamWaitEvent(stream, gt->join, 0);  // the previous frame's step
        if (fp.guided && d + 1 < fp.max_depth) {
            if (timer) timer->mark(stream, StageTimer::kGuide);
            launch_guide_infer(rs, sc, fp, d, stream);
            rs.launches++;
        }
        join_connect();
        if (timer) timer->mark(stream, StageTimer::kShade);
        if (fp.split) {
            const bool sky_mis = fp.sampling == LUC_SAMPLING_MIS && sc.num_lights == 0 && sc.has_env;
            if (fp.guided && sky_mis) k_escape<true, true><<<sms * 8, 256, 0, stream>>>(rs.ps, sc, fp, d);
            else if (fp.guided) k_escape<true, false><<<sms * 8, 256, 0, stream>>>(rs.ps, sc, fp, d);
            else if (sky_mis) k_escape<false, true><<<sms * 8, 256, 0, stream>>>(rs.ps, sc, fp, d);
            else k_escape<false, false><<<sms * 8, 256, 0, stream>>>(rs.ps, sc, fp, d);
            rs.launches++;
        }
        if (fp.guided && inst)
            launch_shade<true, true>(rs, sms * rs.shade_blocks_guided_inst, sc, fp, d, stream);
        else if (fp.guided)
            launch_shade<true, false>(rs, sms * rs.shade_blocks_guided, sc, fp, d, stream);
        else if (inst)
            launch_shade<false, true>(rs, sms * rs.shade_blocks_inst, sc, fp, d, stream);
        else
            launch_shade<false, false>(rs, sms * rs.shade_blocks, sc, fp, d, stream);
        rs.launches += 2;
        if (d + 1 < fp.max_depth && (fp.sampling == LUC_SAMPLING_NEE || fp.sampling == LUC_SAMPLING_MIS) &&
            sc.light_strategies > 0) {
            if (timer) timer->mark(stream, StageTimer::kConnect);
            cudaStream_t cs = stream;
            if (ov) {
                cudaEventRecord(ov->ready, stream);
                cudaStreamWaitEvent(ov->side, ov->ready, 0);
                cs = ov->side;
            }
            // Two-level shadow rays walk the wide BLASes in lock step
            // (InstWalk); the reference's object-space shadow rays and
            // binary-only scenes keep the nested any-hit walk.
            if (inst && wide && sc.twnodes && !sc.reference_shadows)
                k_connect_dyn<128, kInstRefill, 2><<<sms * rs.connect_blocks_inst, 128, 0, cs>>>(rs.ps, sc, d);
            else if (inst && wide && !sc.reference_shadows)
                k_connect_dyn<128, kInstRefill, 1><<<sms * rs.connect_blocks_inst, 128, 0, cs>>>(rs.ps, sc, d);
            else if (inst)
                k_connect<true, false, 128, 0><<<sms * rs.connect_blocks_inst_bin, 128, 0, cs>>>(rs.ps, sc,
                                                                                                 BatchDev{}, d);
            else if (wide)
                k_connect_dyn<128, kExtendRefill><<<sms * rs.connect_blocks, 128, 0, cs>>>(rs.ps, sc, d);
            else
                k_connect<false, false, 128, 0><<<sms * rs.connect_blocks_bin, 128, 0, cs>>>(rs.ps, sc, BatchDev{}, d);
            rs.launches++;
            if (ov) {
                cudaEventRecord(ov->done, ov->side);
                connect_out = true;
            }
        }
    }
    if (fp.max_depth == 0 && gt && gt->join) cudaStreamWaitEvent(stream, gt->join, 0);
    join_connect();
    if (timer) timer->mark(stream, StageTimer::kResolve);
    k_resolve<<<sms * 8, 256, 0, stream>>>(rs.ps, fp, accum);
    rs.launches++;
    if (fp.guided && fp.rec_cap && gt && gt->train) {
        if (timer) timer->mark(stream, StageTimer::kTrain);
        if (gt->defer) {
            launch_guide_finalize(rs, fp, stream);
            rs.launches += 1;
        } else {
            launch_guide_train(rs, fp, *gt, stream);
            rs.launches += 4;
        }
    }
    if (timer) timer->mark(stream, StageTimer::kEnd);
}

// RESOLVE of one batch (the megakernel's paths end in the same pool fields).
void launch_resolve(const RenderState& rs, const FrameParams& fp, GpuAccum* accum, cudaStream_t stream) {
    k_resolve<<<rs.num_sms * 8, 256, 0, stream>>>(rs.ps, fp, accum);
}

}  // namespace luc

int32_t luc_build_traversal(luc_ctx* c, uint32_t num_nodes, uint32_t num_tris) {
    using namespace luc;
    LUC_CUDA(c, c->tnodes.ensure((size_t)num_nodes * 64), "alloc traversal nodes");
    LUC_CUDA(c, c->soup.ensure((size_t)num_tris * 48), "alloc triangle soup");
    int g1 = (int)std::min<uint64_t>((num_nodes + 255) / 256, (uint64_t)c->num_sms * 32);
    int g2 = (int)std::min<uint64_t>((num_tris + 255) / 256, (uint64_t)c->num_sms * 32);
    k_make_tnodes<<<g1, 256, 0, c->stream>>>(c->nodes.as<float4>(), 0u, num_nodes, c->tnodes.as<float4>());
    k_make_soup<<<g2, 256, 0, c->stream>>>(c->tris.as<GpuTriangle>(), c->positions.as<float4>(), num_tris,
                                           c->soup.as<float4>());
    LUC_CUDA(c, cudaGetLastError(), "traversal layout");
    return LUC_OK;
}

// Child-pair records for nodes [begin, end) only (a TLAS rebuilt after the
// BLASes, whose records stay).
int32_t luc_build_tnodes_range(luc_ctx* c, uint32_t begin, uint32_t end) {
    using namespace luc;
    if (end <= begin) return LUC_OK;
    int g = (int)std::min<uint64_t>((end - begin + 255) / 256, (uint64_t)c->num_sms * 32);
    k_make_tnodes<<<g, 256, 0, c->stream>>>(c->nodes.as<float4>(), begin, end, c->tnodes.as<float4>());
    LUC_CUDA(c, cudaGetLastError(), "traversal layout");
    return LUC_OK;
}

namespace luc {

// One wave of a batched render (graph-capturable: fixed shapes, lengths on
// the device). `block` selects the EXTEND / CONNECT instantiation.
template <int B, int W>
static void wave_traverse(RenderState& rs, const BatchDev& bd, const FrameParams& fpw, uint32_t d, bool connect,
                          int ext_blocks, int con_blocks, cudaStream_t s) {
    const int sms = rs.num_sms;
    if (!connect) k_extend<false, true, B, W><<<sms * ext_blocks, B, 0, s>>>(rs.ps, DevScene{}, fpw, bd, d);
    else k_connect<false, true, B, W><<<sms * con_blocks, B, 0, s>>>(rs.ps, DevScene{}, bd, d);
}
template <int B>
static void wave_traverse(RenderState& rs, const BatchDev& bd, const FrameParams& fpw, uint32_t d, bool connect,
                          int ext_blocks, int con_blocks, bool wide, cudaStream_t s) {
    if (wide) wave_traverse<B, 1>(rs, bd, fpw, d, connect, ext_blocks, con_blocks, s);
    else wave_traverse<B, 0>(rs, bd, fpw, d, connect, ext_blocks, con_blocks, s);
}

template <int W>
static const void* batch_kernel(int block, bool connect) {
    if (block == 64) return connect ? (const void*)k_connect<false, true, 64, W> : (const void*)k_extend<false, true, 64, W>;
    if (block == 256)
        return connect ? (const void*)k_connect<false, true, 256, W> : (const void*)k_extend<false, true, 256, W>;
    return connect ? (const void*)k_connect<false, true, 128, W> : (const void*)k_extend<false, true, 128, W>;
}

int batch_blocks_per_sm(int block, bool connect, bool wide) {
    int b = 0;
    const void* k = wide ? batch_kernel<1>(block, connect) : batch_kernel<0>(block, connect);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, block, 0);
    return b > 0 ? b : 1;
}

void record_wave(RenderState& rs, const BatchDev& bd, const uint32_t* pix_off, uint32_t num_paths,
                 uint32_t total_pixels, uint32_t max_depth, int block, bool wide, cudaStream_t s) {
    const int sms = rs.num_sms;
    cudaMemsetAsync(rs.ps.ctr, 0, kCtrStride * (max_depth + 2) * sizeof(uint32_t), s);
    k_generate_batch<<<(int)std::min<uint64_t>((num_paths + 255) / 256, (uint64_t)sms * 16), 256, 0, s>>>(rs.ps, bd,
                                                                                                      num_paths);
    FrameParams fpw{};
    fpw.num_paths = num_paths;
    const int eb = batch_blocks_per_sm(block, false, wide), cb = batch_blocks_per_sm(block, true, wide);
    for (uint32_t d = 0; d < max_depth; ++d) {
        if (block == 64) wave_traverse<64>(rs, bd, fpw, d, false, eb, cb, wide, s);
        else if (block == 256) wave_traverse<256>(rs, bd, fpw, d, false, eb, cb, wide, s);
        else wave_traverse<128>(rs, bd, fpw, d, false, eb, cb, wide, s);
        k_shade<false, false, true><<<sms * rs.shade_blocks, 128, 0, s>>>(rs.ps, DevScene{}, fpw, bd, d);
        rs.launches += 2;
        if (d + 1 < max_depth) {
            if (block == 64) wave_traverse<64>(rs, bd, fpw, d, true, eb, cb, wide, s);
            else if (block == 256) wave_traverse<256>(rs, bd, fpw, d, true, eb, cb, wide, s);
            else wave_traverse<128>(rs, bd, fpw, d, true, eb, cb, wide, s);
            rs.launches++;
        }
    }
    k_resolve_batch<<<(int)std::min<uint64_t>((total_pixels + 255) / 256, (uint64_t)sms * 16), 256, 0, s>>>(
        rs.ps, bd, pix_off, total_pixels);
    rs.launches += 2;
}

}  // namespace luc

namespace luc {
// Sobol dimension-1 byte tables (see sobol_dim1 in device_math.cuh).
__device__ uint32_t g_sobol_dim1_bytes[1024];

__global__ void k_init_sobol_tables() {
    const uint32_t t = threadIdx.x;  // 1024 threads: byte j = t / 256, value b = t % 256
    const uint32_t j = t >> 8, b = t & 255u;
    g_sobol_dim1_bytes[t] = sobol_dim1_loop(b << (8 * j));
}
}  // namespace luc

cudaError_t luc_init_sobol_tables(cudaStream_t s) {
    luc::k_init_sobol_tables<<<1, 1024, 0, s>>>();
    return cudaGetLastError();
}
