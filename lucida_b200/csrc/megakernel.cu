// Megakernel architecture (Architecture::Megakernel, crates/gpu/src/lib.rs:
// 38-79; shaders/trace/megakernel.wgsl:61-266): one thread per path (pixel,
// sample) walks the path to its end with its state in registers: camera ray,
// then per bounce closest hit, shade_vertex (the function the wavefront's
// SHADE runs) and the shadow ray traced at once. The path's radiance is
// summed in the wavefront's order (emission at a vertex, then that vertex's
// light sample, then the next vertex) and lands in the pool's radiance and
// guide fields, which RESOLVE adds per pixel in sample order: both
// architectures produce the same accumulator, bit for bit.
//
// No queues and no per-bounce state traffic: what a megakernel buys. On B200
// the wavefront is faster on both benchmark scenes (divergent paths keep
// whole warps waiting on their longest lane); the architecture is kept for
// parity with the reference and as the convergence meter's renderer.
#include "ctx.cuh"
#include "shade.cuh"

namespace luc {
namespace {

// shade_vertex's sink for a path held in registers.
struct RegSink {
    V3 prev_v;
    bool survive = false, cast = false, guide_hit = false;
    V3 sh_o{0, 0, 0}, sh_d{0, 0, 0}, sh_c{0, 0, 0};
    float sh_t = 0.0f;
    V3 norg{0, 0, 0}, ndir{0, 0, 1}, nthr{0, 0, 0}, hit_pos{0, 0, 0};
    float npdf = 0.0f;
    V3 galb{0, 0, 0}, gnrm{0, 0, 0};
    float gdepth = 0.0f;
    __device__ __forceinline__ V3 prev() const { return prev_v; }
    __device__ __forceinline__ void guides(V3 albedo, float t, V3 normal) {
        guide_hit = true;
        galb = albedo;
        gdepth = t;
        gnrm = normal;
    }
    __device__ __forceinline__ void shadow(V3 o, V3 d, float t_max, V3 c) {
        cast = true;
        sh_o = o;
        sh_d = d;
        sh_t = t_max;
        sh_c = c;
    }
    __device__ __forceinline__ void next(V3 o, V3 d, float pdf, V3 thr, V3 hp, V3, bool, V3) {
        survive = true;
        norg = o;
        ndir = d;
        npdf = pdf;
        nthr = thr;
        hit_pos = hp;
    }
};

template <bool kInst, int kWide>
// 4 blocks of 128 per SM (128 registers): the analytic Cornell box ran 420
// Mpaths/s at the compiler's 148-159 registers (3 blocks), 487 at 4 blocks,
// 437 at 6, 421 at 8.
__global__ void __launch_bounds__(128, 4) k_megakernel(PathState ps, const __grid_constant__ DevScene sc,
                                                    const __grid_constant__ FrameParams fp) {
    const uint32_t sbase = *fp.sbase;
    TravCount tce, tcs;
    uint32_t rays_e = 0, rays_s = 0;
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < fp.num_paths;
         p += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t px = (uint32_t)(p % fp.pixels);
        Sampler smp = make_sampler(fp.sampler_kind, fp.frame_seed, px, sbase + (uint32_t)(p / fp.pixels));
        V3 org, dir;
        camera_ray(fp, px, smp, org, dir);
        V3 thr{1.0f, 1.0f, 1.0f}, rad{0.0f, 0.0f, 0.0f}, prev = org;
        float prev_pdf = 0.0f;
        RegSink first;  // first-hit guides
        for (uint32_t depth = 0; depth < fp.max_depth; ++depth) {
            float t, u, v;
            uint32_t inst;
            const uint32_t id = closest_hit<kInst, kWide>(sc, org, dir, t, u, v, inst, tce);
            ++rays_e;
            RegSink sk;
            sk.prev_v = prev;
            shade_vertex<false, kInst>(sc, fp, depth, smp, org, dir, thr, rad, prev_pdf,
                                       make_float4(t, u, v, __uint_as_float(id)), inst, nullptr, 0u, sk);
            if (sk.guide_hit) first = sk;
            if (sk.cast) {  // CONNECT (shaders/wavefront/connect.wgsl:58-84)
                ++rays_s;
                if (!occluded<kInst, kWide>(sc, sk.sh_o, sk.sh_d, sk.sh_t, tcs)) rad = rad + sk.sh_c;
            }
            if (!sk.survive) break;
            org = sk.norg;
            dir = sk.ndir;
            prev_pdf = sk.npdf;
            thr = sk.nthr;
            prev = sk.hit_pos;
        }
        __stcs(ps.rad + p, make_float4(rad.x, rad.y, rad.z, 0.0f));
        if (fp.guides) {
            ps.galb[p] = first.guide_hit ? make_float4(first.galb.x, first.galb.y, first.galb.z, first.gdepth)
                                         : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            ps.gnrm[p] = first.guide_hit ? make_float4(first.gnrm.x, first.gnrm.y, first.gnrm.z, 0.0f)
                                         : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
    // One atomic per warp per counter (every lane reaches here: the loop
    // above has no early exit).
    unsigned long long v[8] = {rays_e, tce.nodes, tce.tris, rays_s, tcs.nodes, tcs.tris, tce.blas, tcs.blas};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        unsigned long long x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xFFFFFFFFu, x, o);
        if ((threadIdx.x & 31u) == 0) atomicAdd(ps.stat + k, x);
    }
}

template <bool kInst, int kWide>
int blocks_per_sm() {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void*)k_megakernel<kInst, kWide>, 128, 0);
    return b > 0 ? b : 1;
}

}  // namespace

// One batch: every path in one launch, then RESOLVE.
void record_megakernel(const RenderState& rs, const DevScene& sc, const FrameParams& fp, GpuAccum* accum,
                       cudaStream_t s) {
    const uint64_t want = (fp.num_paths + 127) / 128;
    if (sc.num_instances && sc.blas_wide) {
        static const int b = blocks_per_sm<true, 1>();
        k_megakernel<true, 1><<<(int)std::min<uint64_t>(want, (uint64_t)rs.num_sms * b), 128, 0, s>>>(rs.ps, sc, fp);
    } else if (sc.num_instances) {
        static const int b = blocks_per_sm<true, 0>();
        k_megakernel<true, 0><<<(int)std::min<uint64_t>(want, (uint64_t)rs.num_sms * b), 128, 0, s>>>(rs.ps, sc, fp);
    } else if (sc.wnodes) {
        static const int b = blocks_per_sm<false, 1>();
        k_megakernel<false, 1><<<(int)std::min<uint64_t>(want, (uint64_t)rs.num_sms * b), 128, 0, s>>>(rs.ps, sc, fp);
    } else {
        static const int b = blocks_per_sm<false, 0>();
        k_megakernel<false, 0><<<(int)std::min<uint64_t>(want, (uint64_t)rs.num_sms * b), 128, 0, s>>>(rs.ps, sc, fp);
    }
    launch_resolve(rs, fp, accum, s);
}

}  // namespace luc
