// Megakernel architecture (Architecture::Megakernel, crates/gpu/src/lib.rs:
// 38-79; shaders/trace/megakernel.wgsl:61-266): one thread per pixel walks
// its samples in order and each sample's path to the end, with the path in
// registers: camera ray, then per bounce closest hit, shade_vertex (the same
// function the wavefront's SHADE runs) and the shadow ray traced at once.
// The radiance of a path is summed in the wavefront's order (emission at a
// vertex, then that vertex's light sample, then the next vertex) and the
// samples of a pixel are added onto the accumulator in sample order, as
// RESOLVE does, so both architectures produce the same accumulator.
//
// No queues and no path pool: the right choice when paths are short and the
// scene trivial (the reference's README measures it faster there); for
// divergent, traversal-heavy frames the wavefront wins.
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
__global__ void __launch_bounds__(128) k_megakernel(const __grid_constant__ DevScene sc,
                                                    const __grid_constant__ FrameParams fp,
                                                    GpuAccum* __restrict__ accum, unsigned long long* stat) {
    const uint32_t sbase = *fp.sbase;
    TravCount tce, tcs;
    uint32_t rays_e = 0, rays_s = 0;
    for (uint32_t px = blockIdx.x * blockDim.x + threadIdx.x; px < fp.pixels; px += gridDim.x * blockDim.x) {
        GpuAccum a = accum[px];
        V3 r = ld3(a.radiance), r2 = ld3(a.radiance_sq), al = ld3(a.albedo), nn = ld3(a.normal);
        float dep = a.depth;
        for (uint32_t j = 0; j < fp.batch_samples; ++j) {
            Sampler smp = make_sampler(fp.sampler_kind, fp.frame_seed, px, sbase + j);
            V3 org, dir;
            camera_ray(fp, px, smp, org, dir);
            V3 thr{1.0f, 1.0f, 1.0f}, rad{0.0f, 0.0f, 0.0f}, prev = org;
            float prev_pdf = 0.0f;
            V3 g_alb{0.0f, 0.0f, 0.0f}, g_nrm{0.0f, 0.0f, 0.0f};
            float g_dep = 0.0f;
            for (uint32_t depth = 0; depth < fp.max_depth; ++depth) {
                float t, u, v;
                uint32_t inst;
                const uint32_t id = closest_hit<kInst, kWide>(sc, org, dir, t, u, v, inst, tce);
                ++rays_e;
                RegSink sk;
                sk.prev_v = prev;
                shade_vertex<false, kInst>(sc, fp, depth, smp, org, dir, thr, rad, prev_pdf,
                                           make_float4(t, u, v, __uint_as_float(id)), inst, nullptr, 0u, sk);
                if (sk.guide_hit) {
                    g_alb = sk.galb;
                    g_dep = sk.gdepth;
                    g_nrm = sk.gnrm;
                }
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
            // RESOLVE (shaders/wavefront/resolve.wgsl:14-48), one sample.
            r = r + rad;
            r2 = r2 + rad * rad;
            if (fp.guides) {
                al = al + g_alb;
                dep = dep + g_dep;
                nn = nn + g_nrm;
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
    // One atomic per warp per counter.
    unsigned long long v[6] = {rays_e, tce.nodes, tce.tris, rays_s, tcs.nodes, tcs.tris};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        unsigned long long x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xFFFFFFFFu, x, o);
        if ((threadIdx.x & 31u) == 0) atomicAdd(stat + k, x);
    }
}

template <bool kInst, int kWide>
int blocks_per_sm() {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, (const void*)k_megakernel<kInst, kWide>, 128, 0);
    return b > 0 ? b : 1;
}

}  // namespace

// One launch: every pixel, fp.batch_samples samples from *fp.sbase on.
void record_megakernel(const RenderState& rs, const DevScene& sc, const FrameParams& fp, GpuAccum* accum,
                       cudaStream_t s) {
    const uint64_t want = (fp.pixels + 127) / 128;
    if (sc.num_instances) {
        static const int b = blocks_per_sm<true, 0>();
        k_megakernel<true, 0><<<(int)std::min<uint64_t>(want, (uint64_t)rs.num_sms * b), 128, 0, s>>>(sc, fp, accum,
                                                                                                      rs.ps.stat);
    } else if (sc.wnodes) {
        static const int b = blocks_per_sm<false, 1>();
        k_megakernel<false, 1><<<(int)std::min<uint64_t>(want, (uint64_t)rs.num_sms * b), 128, 0, s>>>(sc, fp, accum,
                                                                                                       rs.ps.stat);
    } else {
        static const int b = blocks_per_sm<false, 0>();
        k_megakernel<false, 0><<<(int)std::min<uint64_t>(want, (uint64_t)rs.num_sms * b), 128, 0, s>>>(sc, fp, accum,
                                                                                                       rs.ps.stat);
    }
}

}  // namespace luc
