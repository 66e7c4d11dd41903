// The guide MLP's forward pass on the 5th-generation tensor cores: tcgen05
// MMAs reading BF16 operands from shared memory and accumulating in FP32 in
// tensor memory (TMEM). Same network, numerics contract and feature
// encoding as the mma.sync forward in guide.cu (BF16 operands, FP32
// accumulation, bias + ReLU in FP32, BF16 activations between layers).
//
// One CTA of 128 threads owns 128-row tiles, one row per thread:
//   * the thread writes its row's 128 features (64 sin/cos pairs) into the
//     A tile in shared memory, BF16, in the canonical K-major no-swizzle
//     layout: 8 x 16-byte core matrices, 8-element K chunks LBO apart, 8-row
//     groups 128 B apart;
//   * one thread issues the layer's MMAs (M = 128, N = 64 or 48, K = 16
//     each) against the weights (B, same layout, loaded once per CTA) into
//     TMEM columns 0..63, and commits them to an mbarrier;
//   * every thread waits (bounded), reads its row of the accumulator from
//     TMEM (warp w reads lanes 32w..32w+31), adds the bias, applies ReLU and
//     writes the BF16 activations as the next layer's A tile;
//   * the last layer's 48 outputs (40 used) go to the caller's functor.
// A wait that runs out of iterations sets the CTA's error word (reported in
// *err), all threads leave the tile loop together and the TMEM is freed.
#include <cuda_bf16.h>

#include "ctx.cuh"
#include "guide.cuh"

namespace luc {
namespace tcg {

constexpr int kM = 128;
constexpr int kParts = 4, kThreads = kM * kParts;  // four threads per row
constexpr uint32_t kLboA = kM * 16;            // A tiles: 128 rows per 8-element K chunk
constexpr uint32_t kLboH = kGHid * 16;         // B tiles of 64 output units
constexpr uint32_t kLboO = kGOutPad * 16;      // B tile of the 48 (40 used) output units
constexpr uint32_t kSbo = 128;                 // 8 rows of 16 B
constexpr uint32_t kTmemCols = 64;
constexpr uint32_t kWaitLimit = 1u << 22;

struct Smem {
    // The features (A of the first layer) and, once that layer has run, the
    // tile's raw outputs (bias added) share the first 32 KB.
    union {
        uint8_t x[(kGIn / 8) * kLboA];    // features, 32 KB
        float o[kM][kGOutPad];           // 24 KB
    };
    uint8_t h[(kGHid / 8) * kLboA];   // hidden activations, 16 KB
    uint8_t w1[(kGIn / 8) * kLboH];   // 16 KB
    uint8_t w2[(kGHid / 8) * kLboH];  // 8 KB
    uint8_t w3[(kGHid / 8) * kLboH];  // 8 KB
    uint8_t w4[(kGHid / 8) * kLboO];  // 6 KB
    float b[kGBias];
    float in[kM][9];          // the tile's inputs (computed once per row)
    uint8_t valid[kM];
    unsigned long long mbar;
    uint32_t tmem;
};

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (Blackwell, version 1): start, leading
// and stride byte offsets >> 4, base offset 0, no swizzle.
__device__ __forceinline__ uint64_t desc(uint32_t a, uint32_t lbo) {
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((kSbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor, kind::f16: D F32, A and B BF16, both K-major.
__host__ __device__ constexpr uint32_t idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(d), "l"(a), "l"(b), "r"(id), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ bool wait_phase(uint32_t mbar, uint32_t phase) {
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(ok)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__device__ __forceinline__ float softplus_tc(float x) { return x > 20.0f ? x : log1pf(expf(x)); }

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

// Row r, K chunk c (8 elements, 16 B) of an A tile.
__device__ __forceinline__ uint4* chunk(uint8_t* tile, int c, int r) {
    return reinterpret_cast<uint4*>(tile + c * kLboA + (r >> 3) * kSbo + (r & 7) * 16);
}

// Weights (row = output unit, K contiguous, BF16) into the B layout.
__device__ void load_weights(Smem& S, const uint16_t* __restrict__ wbf, const float* __restrict__ bias) {
    auto load = [&](uint8_t* dst, const uint16_t* src, int n, int k, uint32_t lbo) {
        const int chunks = n * (k / 8);
        for (int i = threadIdx.x; i < chunks; i += blockDim.x) {
            const int row = i / (k / 8), c = i % (k / 8);
            const uint4 v = *reinterpret_cast<const uint4*>(src + row * k + c * 8);
            *reinterpret_cast<uint4*>(dst + c * lbo + (row >> 3) * kSbo + (row & 7) * 16) = v;
        }
    };
    load(S.w1, wbf, kGHid, kGIn, kLboH);
    load(S.w2, wbf + kGHid * kGIn, kGHid, kGHid, kLboH);
    load(S.w3, wbf + kGHid * kGIn + kGHid * kGHid, kGHid, kGHid, kLboH);
    load(S.w4, wbf + kGHid * kGIn + 2 * kGHid * kGHid, kGOutPad, kGHid, kLboO);
    for (int i = threadIdx.x; i < kGBias; i += blockDim.x) S.b[i] = bias[i];
}

// The 128 features of one row (position: 12 frequencies per axis of the
// box-normalised point; normal and outgoing direction: 4 each; sin/cos
// pairs, zero padding from 120) into row r of the feature tile.
__device__ __forceinline__ void write_features(Smem& S, int r, int part, const float (&in)[9], const GuideDev& g) {
#pragma unroll
    for (int cc = 0; cc < kGIn / 8 / kParts; ++cc) {
        const int c = part * (kGIn / 8 / kParts) + cc;
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int f = 8 * c + 2 * j;
            if (f >= kGFeatures) {
                w[j] = 0u;
                continue;
            }
            float arg;
            if (f < 72) {
                const int a = f / 24, k = (f % 24) / 2;
                const float q = fminf(fmaxf((in[a] - g.lo[a]) / g.ext[a], 0.0f), 1.0f);
                arg = q * (kPi * (float)(1 << k));
            } else {
                const int rr = f - 72, comp = 3 + 3 * (rr / 24) + (rr % 24) / 8, t = (rr % 8) / 2;
                arg = in[comp] * (kPi * (float)(1 << t));
            }
            float sn, cs;
            sincosf(arg, &sn, &cs);
            w[j] = pack2(sn, cs);
        }
        *chunk(S.x, c, r) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// bias + ReLU of this thread's 16 accumulator columns (16 part .. + 15)
// into row r of the hidden tile.
__device__ __forceinline__ void write_hidden(Smem& S, int r, int part, const float (&v)[16],
                                             const float* __restrict__ b) {
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k = 8 * cc + 2 * j, n = 16 * part + k;
            w[j] = pack2(fmaxf(v[k] + b[n], 0.0f), fmaxf(v[k + 1] + b[n + 1], 0.0f));
        }
        *chunk(S.h, 2 * part + cc, r) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// The tile loop. load(row, in) fills a row's 9 inputs (false: no row to
// evaluate); store(row, out) receives the 48 raw outputs (bias added) of
// every valid row. Thread (warp w, lane l) serves row 32 (w % 4) + l — the
// TMEM lane quadrant warp w may read — as part w / 4 of four: the part-0
// thread loads the inputs and later decodes; each part computes 16 feature
// pairs and reads 16 accumulator columns.
template <typename Load, typename Store>
__device__ void forward_tiles(uint32_t n, const GuideDev& g, uint32_t* err, Load load, Store store) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    Smem& S = *reinterpret_cast<Smem*>(smem_raw);
    const int t = threadIdx.x, warp = t >> 5, part = warp >> 2;
    const int r = 32 * (warp & 3) + (t & 31);
    load_weights(S, g.wbf, g.bias);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%1], %0;" ::"r"(1u), "r"(saddr(&S.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&S.tmem)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = S.tmem, mbar = saddr(&S.mbar);
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + 16 * part;
    uint32_t phase = 0;
    bool failed = false;
    // One layer: MMAs over K (k16 steps), commit, bounded wait; every thread
    // learns whether the CTA's wait completed.
    auto layer = [&](const uint8_t* a, uint32_t lba, const uint8_t* w, uint32_t lbw, int ksteps, int nout) {
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        if (t == 0) {
            for (int ks = 0; ks < ksteps; ++ks)
                mma(tmem, desc(saddr(a) + 2 * ks * lba, lba), desc(saddr(w) + 2 * ks * lbw, lbw), idesc(nout),
                    ks > 0 ? 1u : 0u);
            commit(mbar);
        }
        const bool ok = wait_phase(mbar, phase);
        phase ^= 1u;
        fence_after();
        return __syncthreads_and(ok) != 0;
    };
    for (uint32_t base = blockIdx.x * kM; base < n; base += gridDim.x * kM) {
        const uint32_t row = base + r;
        if (part == 0) {
            float in[9] = {0, 0, 0, 0, 0, 1, 0, 0, 1};
            const bool valid = row < n && load(row, in);
#pragma unroll
            for (int k = 0; k < 9; ++k) S.in[r][k] = in[k];
            S.valid[r] = valid ? 1 : 0;
        }
        __syncthreads();
        {
            float in[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) in[k] = S.in[r][k];
            write_features(S, r, part, in, g);
        }
        float v[16];
        if (!layer(S.x, kLboA, S.w1, kLboH, kGIn / 16, kGHid)) {
            failed = true;
            break;
        }
        ld16(lane_addr, v);
        write_hidden(S, r, part, v, S.b);
        if (!layer(S.h, kLboA, S.w2, kLboH, kGHid / 16, kGHid)) {
            failed = true;
            break;
        }
        ld16(lane_addr, v);
        write_hidden(S, r, part, v, S.b + kGHid);
        if (!layer(S.h, kLboA, S.w3, kLboH, kGHid / 16, kGHid)) {
            failed = true;
            break;
        }
        ld16(lane_addr, v);
        write_hidden(S, r, part, v, S.b + 2 * kGHid);
        if (!layer(S.h, kLboA, S.w4, kLboO, kGHid / 16, kGOutPad)) {
            failed = true;
            break;
        }
        ld16(lane_addr, v);  // part 3 reads columns 48..63, which the last layer does not write
        if (part < kGOutPad / 16) {
#pragma unroll
            for (int k = 0; k < 16; ++k) S.o[r][16 * part + k] = v[k] + S.b[3 * kGHid + 16 * part + k];
        }
        fence_before();
        __syncthreads();
        if (part == 0 && S.valid[r]) store(row, S.o[r]);
    }
    if (failed && t == 0) atomicOr(err, 1u);
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

// Raw outputs (bias added) of n rows of 9 inputs: the test-facing forward.
__global__ void __launch_bounds__(kThreads, 2) k_forward_tc(const float* __restrict__ in9, uint32_t n, GuideDev g,
                                                   float* __restrict__ out40, uint32_t* err) {
    forward_tiles(
        n, g, err,
        [&](uint32_t row, float (&in)[9]) {
#pragma unroll
            for (int k = 0; k < 9; ++k) in[k] = in9[9 * (size_t)row + k];
            return true;
        },
        [&](uint32_t row, const float* o) {
#pragma unroll
            for (int k = 0; k < kGOut; ++k) out40[kGOut * (size_t)row + k] = o[k];
        });
}

// Per bounce (as the mma.sync inference did): the decoded mixture of every
// queue position whose ray hit a surface, in SoA planes of ps.lobe_stride.
// Inputs are the hit point, the shading normal and the outgoing direction.
// The decode is the per-row form of the two-lane decode it replaces, in the
// same operation order (the softmax sum is the two half-sums added).
__global__ void __launch_bounds__(kThreads, 2) k_infer_tc(PathState ps, const __grid_constant__ DevScene sc,
                                                 const __grid_constant__ FrameParams fp, uint32_t depth) {
    const uint32_t len = depth == 0 ? (uint32_t)fp.num_paths : ps.ctr[depth * kCtrStride + kCtrQueue];
    const uint32_t* queue = ps.queue[depth & 1];
    forward_tiles(
        len, fp.guide, ps.gmisc + kGmTcError,
        [&](uint32_t i, float (&in)[9]) {
            const uint32_t q = depth == 0 ? i : queue[i];
            const float4 h4 = ps.hit[q];
            const uint32_t id = __float_as_uint(h4.w);
            if (id == kMiss) return false;
            const float4 o4 = ps.o_pdf[q], d4 = ps.dir[q];
            const V3 dir{d4.x, d4.y, d4.z};
            const SurfaceHit hit = surface_hit(sc, id, sc.num_instances ? ps.hinst[q] : 0u, h4.x, h4.y, h4.z,
                                               V3{o4.x, o4.y, o4.z}, dir);
            in[0] = hit.position.x;
            in[1] = hit.position.y;
            in[2] = hit.position.z;
            in[3] = hit.normal.x;
            in[4] = hit.normal.y;
            in[5] = hit.normal.z;
            in[6] = -dir.x;
            in[7] = -dir.y;
            in[8] = -dir.z;
            return true;
        },
        [&](uint32_t i, const float* o) {
            float mx = -INFINITY;
#pragma unroll
            for (int j = 0; j < kGLobes; ++j) mx = fmaxf(mx, o[5 * j + 4]);
            float e[kGLobes], half[2] = {0.f, 0.f};
#pragma unroll
            for (int j = 0; j < kGLobes; ++j) {
                e[j] = expf(o[5 * j + 4] - mx);
                half[j >> 2] += e[j];
            }
            const float sum = half[0] + half[1];
            const size_t st = ps.lobe_stride;
#pragma unroll
            for (int j = 0; j < kGLobes; ++j) {
                const float x = o[5 * j], y = o[5 * j + 1], z = o[5 * j + 2];
                const float ln = sqrtf(x * x + y * y + z * z);
                const float kappa = fminf(1.0f + softplus_tc(o[5 * j + 3]), kGKappaMax);
                ps.lobes[j * st + i] =
                    ln > 0.0f ? make_float4(x / ln, y / ln, z / ln, kappa) : make_float4(0.f, 0.f, 1.f, kappa);
            }
            ps.lobes[8 * st + i] = make_float4(e[0] / sum, e[1] / sum, e[2] / sum, e[3] / sum);
            ps.lobes[9 * st + i] = make_float4(e[4] / sum, e[5] / sum, e[6] / sum, e[7] / sum);
        });
}

}  // namespace tcg
}  // namespace luc

// Dynamic shared memory above 48 KB: opted into once per device, before any
// launch (never inside a stream capture).
cudaError_t guide_tc_setup() {
    using namespace luc;
    cudaError_t e = cudaFuncSetAttribute(tcg::k_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(tcg::Smem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(tcg::k_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(tcg::Smem));
    return e;
}

void launch_guide_infer_tc(const luc::RenderState& rs, const luc::DevScene& sc, const luc::FrameParams& fp,
                           uint32_t depth, cudaStream_t s) {
    using namespace luc;
    // Persistent tiles: two CTAs fit an SM (shared memory), each holding 64
    // TMEM columns.
    tcg::k_infer_tc<<<rs.num_sms * 2, tcg::kThreads, sizeof(tcg::Smem), s>>>(rs.ps, sc, fp, depth);
}

// Launch the tensor-core forward over n rows of 9 inputs (device arrays).
cudaError_t launch_guide_forward_tc(const float* in9, uint32_t n, const luc::GuideDev& g, float* out40, uint32_t* err,
                                    int num_sms, cudaStream_t s) {
    using namespace luc;
    static const cudaError_t attr = guide_tc_setup();
    if (attr != cudaSuccess) return attr;
    const int grid = (int)std::min<uint64_t>((n + tcg::kM - 1) / tcg::kM, (uint64_t)num_sms * 2);
    tcg::k_forward_tc<<<grid, tcg::kThreads, sizeof(tcg::Smem), s>>>(in9, n, g, out40, err);
    return cudaGetLastError();
}
