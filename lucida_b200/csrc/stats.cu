// Convergence meter (ConvergenceMeter, crates/gpu/src/stats.rs:1-173;
// shaders/stats/convergence.wgsl:1-141): the mean over measurable pixels of
// the relative standard error of the pixel's mean,
//   se / mean_lum,  se = sqrt(lum(max(sum_sq / n - mean^2, 0)) / n),
// over pixels with n >= 2 samples and mean luminance above 1e-3; -1 when no
// pixel qualifies. It assumes independent samples, so with Sobol it is an
// upper bound (the reference's note).
//
// Same two-pass shape and summation order as the reference: 64 blocks of
// 256 threads read the accumulator strided (coalesced), fold their partial
// (error, count) pairs by halving, and one block folds the 64 partials.
#include "ctx.cuh"

namespace luc {
namespace {

constexpr int kGroups = 64, kWg = 256;
constexpr float kMinLuminance = 1.0e-3f;

__device__ __forceinline__ void fold(float* e, float* n) {
    const int lid = threadIdx.x;
#pragma unroll 1
    for (int s = kWg / 2; s > 0; s /= 2) {
        if (lid < s) {
            e[lid] = e[lid] + e[lid + s];
            n[lid] = n[lid] + n[lid + s];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kWg) k_conv_reduce(const GpuAccum* __restrict__ accum, uint32_t pixels,
                                                     float2* __restrict__ partials) {
    __shared__ float e[kWg], n[kWg];
    float err = 0.0f, cnt = 0.0f;
    for (uint32_t i = blockIdx.x * kWg + threadIdx.x; i < pixels; i += gridDim.x * kWg) {
        const GpuAccum a = accum[i];
        const float ns = a.samples;
        if (ns >= 2.0f) {
            const V3 mean = ld3(a.radiance) / ns;
            const float mean_l = luminance(mean);
            if (mean_l > kMinLuminance) {
                const V3 var = vmax(ld3(a.radiance_sq) / ns - mean * mean, splat(0.0f));
                const float se = sqrtf(luminance(var) / ns);
                err = err + se / mean_l;
                cnt = cnt + 1.0f;
            }
        }
    }
    e[threadIdx.x] = err;
    n[threadIdx.x] = cnt;
    __syncthreads();
    fold(e, n);
    if (threadIdx.x == 0) partials[blockIdx.x] = make_float2(e[0], n[0]);
}

__global__ void __launch_bounds__(kWg) k_conv_finish(const float2* __restrict__ partials, float* __restrict__ result) {
    __shared__ float e[kWg], n[kWg];
    float err = 0.0f, cnt = 0.0f;
    for (int i = threadIdx.x; i < kGroups; i += kWg) {
        err = err + partials[i].x;
        cnt = cnt + partials[i].y;
    }
    e[threadIdx.x] = err;
    n[threadIdx.x] = cnt;
    __syncthreads();
    fold(e, n);
    if (threadIdx.x == 0) result[0] = n[0] > 0.0f ? e[0] / n[0] : -1.0f;
}

}  // namespace
}  // namespace luc

// Records the meter on `s`; the figure lands after the 64 partials in
// c->conv_scratch (device).
int32_t luc_record_convergence(luc_ctx* c, const GpuAccum* accum, uint32_t pixels, cudaStream_t s) {
    using namespace luc;
    LUC_CUDA(c, c->conv_scratch.ensure(kGroups * sizeof(float2) + 16), "allocate convergence scratch");
    float2* partials = c->conv_scratch.as<float2>();
    float* result = reinterpret_cast<float*>(partials + kGroups);
    k_conv_reduce<<<kGroups, kWg, 0, s>>>(accum, pixels, partials);
    k_conv_finish<<<1, kWg, 0, s>>>(partials, result);
    LUC_CUDA(c, cudaGetLastError(), "convergence meter");
    return LUC_OK;
}

extern "C" int32_t luc_convergence(luc_ctx* c, const void* accum_dev, uint32_t pixels, float* out) {
    if (!c || !out || (pixels && !accum_dev)) return LUC_ERR_VALIDATION;
    cudaSetDevice(c->device);
    int32_t rc = luc_record_convergence(c, (const GpuAccum*)accum_dev, pixels, c->stream);
    if (rc) return rc;
    const float* result = reinterpret_cast<const float*>(c->conv_scratch.as<float2>() + 64);
    LUC_CUDA(c, cudaMemcpyAsync(out, result, 4, cudaMemcpyDeviceToHost, c->stream), "read convergence");
    LUC_CUDA(c, cudaStreamSynchronize(c->stream), "convergence meter");
    return LUC_OK;
}

// ---------------------------------------------------------------- read bandwidth
// Streaming reads of a caller device buffer, `passes` times in one launch
// (128-bit loads, four in flight per thread, grid-stride over 148 x 8
// blocks): the bandwidth reference the
// benchmark sets its traversal figures against. Over a buffer smaller than the
// L2 (126 MB) that stays resident between passes it measures L2 read
// bandwidth; over one larger than the L2, HBM read bandwidth. One word per
// block goes to `sink` so the loads cannot be elided.
namespace luc {
namespace {
__global__ void __launch_bounds__(256) k_read_sweep(const uint4* __restrict__ buf, uint64_t n16, uint32_t passes,
                                                    uint32_t* sink) {
    uint32_t acc = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint32_t p = 0; p < passes; ++p) {
        uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
        for (; i + 3 * stride < n16; i += 4 * stride) {
            const uint4 a = __ldcg(buf + i), b = __ldcg(buf + i + stride), c = __ldcg(buf + i + 2 * stride),
                        d = __ldcg(buf + i + 3 * stride);
            acc ^= a.x ^ a.y ^ a.z ^ a.w ^ b.x ^ b.y ^ b.z ^ b.w ^ c.x ^ c.y ^ c.z ^ c.w ^ d.x ^ d.y ^ d.z ^ d.w;
        }
        for (; i < n16; i += stride) {
            const uint4 a = __ldcg(buf + i);
            acc ^= a.x ^ a.y ^ a.z ^ a.w;
        }
        acc = acc * 0x9E3779B1u + p;  // keeps the passes' loads from being merged
    }
    acc = __reduce_xor_sync(0xFFFFFFFFu, acc);
    if ((threadIdx.x & 31u) == 0u) atomicXor(sink + blockIdx.x, acc);
}
}  // namespace
}  // namespace luc

extern "C" int32_t luc_read_sweep(luc_ctx* c, const void* buf_dev, uint64_t bytes, uint32_t passes, void* sink_dev) {
    using namespace luc;
    if (!c || !buf_dev || !sink_dev || (bytes & 15u) || ((uintptr_t)buf_dev & 15u)) return LUC_ERR_VALIDATION;
    cudaSetDevice(c->device);
    // All passes in one launch: at L2-resident sizes a launch per pass would
    // measure launch latency as much as bandwidth.
    k_read_sweep<<<148 * 8, 256, 0, c->stream>>>((const uint4*)buf_dev, bytes / 16, passes, (uint32_t*)sink_dev);
    LUC_CUDA(c, cudaGetLastError(), "read sweep");
    return LUC_OK;
}
