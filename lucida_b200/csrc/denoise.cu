// Edge-avoiding à-trous denoiser on sm_100a (crates/gpu/src/denoise.rs:
// 103-210, shaders/denoise/atrous.wgsl; CPU semantics crates/core/src/
// denoise.rs:101-228).
//
//   k_dn_prepare  : per pixel, from the accumulator: demodulated radiance
//                   (radiance/n / max(albedo/n, 1e-3)) with its luminance in
//                   .w, the guide (normal/n, depth/n) and the guide albedo's
//                   luminance — everything a tap reads, packed once;
//   k_dn_measure  : 3x3 luminance deviation of the demodulated signal, once;
//   k_dn_atrous   : one 5x5 B3-spline pass at stride 2^level with the normal,
//                   depth, luminance and albedo edge-stopping weights
//                   (ping-pong, `iterations` launches);
//   k_dn_modulate : multiply the albedo back; Accum-shaped output, samples = 1.
//
// A tap reads a float4 of colour+luminance, a float4 of guide and one float,
// 36 bytes; a 1920x1080 frame's buffers (~72 MB) stay in the 126 MB L2, so a
// pass costs HBM roughly one read and one write of the colour buffer.
#include <cuda_fp16.h>
#include "ctx.cuh"

namespace luc {

// Guide storage: FP32 (float4 normal+depth, float albedo luminance, float4
// albedo) or, with kHalf, FP16 (8 + 2 + 8 bytes): a tap then reads 16 B of
// colour plus 10 B of guides instead of 36 B.
template <bool kHalf>
struct GuideT;
template <>
struct GuideT<false> {
    using G = float4;
    using A = float;
    using C = float4;
    static __device__ __forceinline__ G pack(float4 v) { return v; }
    static __device__ __forceinline__ float4 unpack(G v) { return v; }
    static __device__ __forceinline__ A pack1(float v) { return v; }
    static __device__ __forceinline__ float unpack1(A v) { return v; }
};
template <>
struct GuideT<true> {
    using G = uint2;  // four halves
    using A = __half;
    using C = uint2;
    static __device__ __forceinline__ G pack(float4 v) {
        __half2 a = __floats2half2_rn(v.x, v.y), b = __floats2half2_rn(v.z, v.w);
        return make_uint2(*reinterpret_cast<uint32_t*>(&a), *reinterpret_cast<uint32_t*>(&b));
    }
    static __device__ __forceinline__ float4 unpack(G v) {
        float2 a = __half22float2(*reinterpret_cast<__half2*>(&v.x)), b = __half22float2(*reinterpret_cast<__half2*>(&v.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
    static __device__ __forceinline__ A pack1(float v) { return __float2half_rn(v); }
    static __device__ __forceinline__ float unpack1(A v) { return __half2float(v); }
};

struct DnParams {
    uint32_t w, h, stride;
    float sigma_normal, sigma_depth, sigma_luminance, sigma_albedo;
};

template <bool kHalf>
__global__ void k_dn_prepare(const GpuAccum* __restrict__ acc, uint32_t n, float4* __restrict__ color,
                             typename GuideT<kHalf>::G* __restrict__ guide, typename GuideT<kHalf>::A* __restrict__ alum,
                             typename GuideT<kHalf>::C* __restrict__ albedo) {
    using T = GuideT<kHalf>;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const GpuAccum a = acc[i];
        float inv = 1.0f / fmaxf(a.samples, 1.0f);
        V3 alb = vmax(ld3(a.albedo) * inv, splat(1.0e-3f));
        V3 rad = ld3(a.radiance) * inv / alb;
        color[i] = make_float4(rad.x, rad.y, rad.z, luminance(rad));
        V3 nrm = ld3(a.normal) * inv;
        guide[i] = T::pack(make_float4(nrm.x, nrm.y, nrm.z, a.depth * inv));
        alum[i] = T::pack1(luminance(alb));
        albedo[i] = T::pack(make_float4(alb.x, alb.y, alb.z, 0.0f));
    }
}

// denoise.rs:111-128 / atrous.wgsl measure
__global__ void k_dn_measure(const float4* __restrict__ color, uint32_t w, uint32_t h, float* __restrict__ dev) {
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    float sum = 0.0f, sum_sq = 0.0f, n = 0.0f;
    for (int dy = -1; dy <= 1; ++dy) {
        for (int dx = -1; dx <= 1; ++dx) {
            int px = (int)x + dx, py = (int)y + dy;
            if (px < 0 || py < 0 || px >= (int)w || py >= (int)h) continue;
            float l = __ldg(&color[(size_t)py * w + px].w);
            sum = sum + l;
            sum_sq = sum_sq + l * l;
            n = n + 1.0f;
        }
    }
    float mean = sum / n;
    dev[(size_t)y * w + x] = sqrtf(fmaxf(sum_sq / n - mean * mean, 0.0f));
}

__constant__ float kB3[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};

// denoise.rs:171-217 / atrous.wgsl atrous_pass
template <bool kHalf>
__global__ void __launch_bounds__(256) k_dn_atrous(const float4* __restrict__ cin, float4* __restrict__ cout,
                                                   const typename GuideT<kHalf>::G* __restrict__ guide,
                                                   const typename GuideT<kHalf>::A* __restrict__ alum,
                                                   const float* __restrict__ dev, DnParams p) {
    using T = GuideT<kHalf>;
    uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.w || y >= p.h) return;
    const size_t ci = (size_t)y * p.w + x;
    const float4 cg = T::unpack(guide[ci]);
    const float4 cc = __ldg(cin + ci);
    const float cl = cc.w;
    const float ca = fmaxf(T::unpack1(alum[ci]), 1.0e-3f);
    const float lum_scale = p.sigma_luminance * fmaxf(__ldg(dev + ci), 1.0e-4f);
    const float dscale = p.sigma_depth * fmaxf(fabsf(cg.w), 1.0e-3f);
    const float ascale = p.sigma_albedo * ca;
    V3 sum = splat(0.0f);
    float wsum = 0.0f;
    const int s = (int)p.stride;
    for (int ky = 0; ky < 5; ++ky) {
        int py = (int)y + (ky - 2) * s;
        if (py < 0 || py >= (int)p.h) continue;
        for (int kx = 0; kx < 5; ++kx) {
            int px = (int)x + (kx - 2) * s;
            if (px < 0 || px >= (int)p.w) continue;
            const size_t qi = (size_t)py * p.w + px;
            const float4 qg = T::unpack(guide[qi]);
            const float4 qc = __ldg(cin + qi);
            float nd = fmaxf(dot(V3{cg.x, cg.y, cg.z}, V3{qg.x, qg.y, qg.z}), 0.0f);
            // Edge-stopping weights with CUDA's f32 powf / expf (within 2 ulp):
            // the double-rounded forms the integrator uses cost four
            // double-precision calls per tap here, and the filter's
            // agreement with the oracle stays far inside its bound.
            float w_n = powf(nd, p.sigma_normal);
            float w_d = expf(-fabsf(cg.w - qg.w) / dscale);
            float w_l = expf(-fabsf(cl - qc.w) / lum_scale);
            float w_a = expf(-fabsf(ca - T::unpack1(alum[qi])) / ascale);
            float wgt = kB3[kx] * kB3[ky] * w_n * w_d * w_l * w_a;
            sum = sum + V3{qc.x, qc.y, qc.z} * wgt;
            wsum = wsum + wgt;
        }
    }
    if (wsum > 0.0f) {
        V3 o = sum / wsum;
        cout[ci] = make_float4(o.x, o.y, o.z, luminance(o));
    } else {
        cout[ci] = cc;
    }
}

template <bool kHalf>
__global__ void k_dn_modulate(const float4* __restrict__ color, const typename GuideT<kHalf>::C* __restrict__ albedo,
                              const typename GuideT<kHalf>::G* __restrict__ guide, uint32_t n,
                              GpuAccum* __restrict__ out) {
    using T = GuideT<kHalf>;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 c = color[i], a = T::unpack(albedo[i]), g = T::unpack(guide[i]);
        GpuAccum o;
        o.radiance[0] = c.x * a.x; o.radiance[1] = c.y * a.y; o.radiance[2] = c.z * a.z;
        o.samples = 1.0f;
        o.albedo[0] = a.x; o.albedo[1] = a.y; o.albedo[2] = a.z;
        o.depth = g.w;
        o.normal[0] = g.x; o.normal[1] = g.y; o.normal[2] = g.z;
        o.traversal = 0.0f;
        o.radiance_sq[0] = 0.0f; o.radiance_sq[1] = 0.0f; o.radiance_sq[2] = 0.0f;
        o._pad0 = 0.0f;
        out[i] = o;
    }
}

}  // namespace luc

using namespace luc;

template <bool kHalf>
static int32_t denoise_run(luc_ctx* c, const GpuAccum* accum, uint32_t w, uint32_t h, const luc_denoise_params* p,
                           GpuAccum* out) {
    using T = GuideT<kHalf>;
    const size_t n = (size_t)w * h;
    cudaStream_t s = c->stream;
    LUC_CUDA(c, c->dn_a.ensure(n * 16 * 2), "alloc denoise");  // colour ping + pong (FP32)
    LUC_CUDA(c, c->dn_b.ensure(n * (sizeof(typename T::G) + sizeof(typename T::C))), "alloc denoise");  // guide, albedo
    LUC_CUDA(c, c->dn_dev.ensure(n * (4 + sizeof(typename T::A)) + 16), "alloc denoise");  // deviation, albedo lum
    float4* ca = c->dn_a.as<float4>();
    float4* cb = ca + n;
    typename T::G* guide = c->dn_b.as<typename T::G>();
    typename T::C* albedo = reinterpret_cast<typename T::C*>(guide + n);
    float* dev = c->dn_dev.as<float>();
    typename T::A* alum = reinterpret_cast<typename T::A*>(dev + n);
    int grid1 = (int)std::min<size_t>((n + 255) / 256, (size_t)c->num_sms * 16);
    dim3 blk(16, 16), grid2((w + 15) / 16, (h + 15) / 16);
    k_dn_prepare<kHalf><<<grid1, 256, 0, s>>>(accum, (uint32_t)n, ca, guide, alum, albedo);
    k_dn_measure<<<grid2, blk, 0, s>>>(ca, w, h, dev);
    DnParams dp{w, h, 1, p->sigma_normal, p->sigma_depth, p->sigma_luminance, p->sigma_albedo};
    float4 *cur = ca, *nxt = cb;
    for (uint32_t level = 0; level < p->iterations; ++level) {
        dp.stride = 1u << level;
        k_dn_atrous<kHalf><<<grid2, blk, 0, s>>>(cur, nxt, guide, alum, dev, dp);
        std::swap(cur, nxt);
    }
    k_dn_modulate<kHalf><<<grid1, 256, 0, s>>>(cur, albedo, guide, (uint32_t)n, out);
    LUC_CUDA(c, cudaGetLastError(), "denoise");
    return LUC_OK;
}

int32_t luc_denoise_device(luc_ctx* c, const GpuAccum* accum, uint32_t w, uint32_t h, const luc_denoise_params* p,
                           GpuAccum* out, bool half_guides) {
    return half_guides ? denoise_run<true>(c, accum, w, h, p, out) : denoise_run<false>(c, accum, w, h, p, out);
}

extern "C" int32_t luc_denoise(luc_ctx* c, const GpuAccum* accum, uint32_t w, uint32_t h,
                               const luc_denoise_params* p, GpuAccum* out) {
    if (!c || !accum || !out || !p) return LUC_ERR_VALIDATION;
    if (w == 0 || h == 0) return luc_fail(c, LUC_ERR_VALIDATION, "zero-sized image");
    if (p->iterations > 16) return luc_fail(c, LUC_ERR_VALIDATION, "at most 16 a-trous iterations");
    cudaSetDevice(c->device);
    const size_t n = (size_t)w * h;
    cudaStream_t s = c->stream;
    LUC_CUDA(c, c->dn_in.ensure(n * sizeof(GpuAccum)), "alloc denoise");
    LUC_CUDA(c, c->dn_out.ensure(n * sizeof(GpuAccum)), "alloc denoise");
    LUC_CUDA(c, cudaMemcpyAsync(c->dn_in.p, accum, n * sizeof(GpuAccum), cudaMemcpyHostToDevice, s), "upload");
    int32_t rc = luc_denoise_device(c, c->dn_in.as<GpuAccum>(), w, h, p, c->dn_out.as<GpuAccum>(), false);
    if (rc) return rc;
    LUC_CUDA(c, cudaMemcpyAsync(out, c->dn_out.p, n * sizeof(GpuAccum), cudaMemcpyDeviceToHost, s), "readback");
    LUC_CUDA(c, cudaStreamSynchronize(s), "denoise");
    return LUC_OK;
}

// Device buffers in and out, on the context's stream (not synchronised);
// flags bit 0 keeps the guides in FP16.
extern "C" int32_t luc_denoise_dev(luc_ctx* c, const void* accum_dev, uint32_t w, uint32_t h,
                                   const luc_denoise_params* p, uint32_t flags, void* out_dev) {
    if (!c || !accum_dev || !out_dev || !p) return LUC_ERR_VALIDATION;
    if (w == 0 || h == 0) return luc_fail(c, LUC_ERR_VALIDATION, "zero-sized image");
    if (p->iterations > 16) return luc_fail(c, LUC_ERR_VALIDATION, "at most 16 a-trous iterations");
    if (flags & ~LUC_DENOISE_HALF_GUIDES) return luc_fail(c, LUC_ERR_VALIDATION, "unknown denoise flag");
    if (accum_dev == out_dev) return luc_fail(c, LUC_ERR_VALIDATION, "the output must not alias the accumulator");
    cudaSetDevice(c->device);
    return luc_denoise_device(c, (const GpuAccum*)accum_dev, w, h, p, (GpuAccum*)out_dev,
                              (flags & LUC_DENOISE_HALF_GUIDES) != 0);
}
