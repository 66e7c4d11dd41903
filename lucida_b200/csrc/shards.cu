// Merging sample-range shards. A frame split across GPUs by sample range
// (rank r renders samples [r*spp, (r+1)*spp) of every pixel; the RNG is a pure
// function of frame, pixel and sample, crates/core/src/rng.rs:18-21) leaves
// one GpuAccum per rank whose fields are all sums over that rank's samples,
// so the frame's accumulator is their field-wise sum
// (crates/gpu/tests/cpu_gpu_agreement.rs:119-168: progressive == one shot).
// The host gathers the ranks' accumulators into one array (torch.distributed
// over NCCL) and this kernel adds them in rank order — fixed order, so the
// merged image does not depend on the collective's reduction schedule.
#include <algorithm>
#include "ctx.cuh"

namespace luc {
namespace {
// One thread per float4 of the output (a GpuAccum is four): parts[0] + parts[1]
// + ... in rank order, 16-byte loads and stores.
__global__ void __launch_bounds__(256) k_accum_merge(const float4* __restrict__ parts, uint32_t nparts,
                                                     uint64_t n4, float4* __restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4; i += (uint64_t)gridDim.x * blockDim.x) {
        float4 a = __ldcs(parts + i);
        for (uint32_t r = 1; r < nparts; ++r) {
            const float4 b = __ldcs(parts + (uint64_t)r * n4 + i);
            a.x = a.x + b.x;
            a.y = a.y + b.y;
            a.z = a.z + b.z;
            a.w = a.w + b.w;
        }
        __stcs(out + i, a);
    }
}
}  // namespace
}  // namespace luc

extern "C" int32_t luc_accum_merge(luc_ctx* c, const void* parts_dev, uint32_t nparts, uint32_t pixels,
                                   void* out_dev) {
    using namespace luc;
    if (!c || nparts == 0 || (pixels && (!parts_dev || !out_dev)) || ((uintptr_t)parts_dev & 15u) ||
        ((uintptr_t)out_dev & 15u))
        return LUC_ERR_VALIDATION;
    if (pixels == 0) return LUC_OK;
    cudaSetDevice(c->device);
    const uint64_t n4 = (uint64_t)pixels * 4;
    const unsigned grid = (unsigned)std::min<uint64_t>((n4 + 255) / 256, 148ull * 16);
    k_accum_merge<<<grid, 256, 0, c->stream>>>((const float4*)parts_dev, nparts, n4, (float4*)out_dev);
    LUC_CUDA(c, cudaGetLastError(), "accumulator merge");
    return LUC_OK;
}
