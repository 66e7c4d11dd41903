// The guide MLP's forward pass on the 5th-generation tensor cores: tcgen05
// MMAs reading BF16 operands from shared memory and accumulating in FP32 in
// tensor memory (TMEM). Same network, numerics contract and feature
// encoding as the mma.sync forward in guide.cu (BF16 operands, FP32
// accumulation, bias + ReLU in FP32, BF16 activations between layers).
//
// Eight teams per CTA (one CTA per SM), each a 128-row pipeline: four warps,
// one thread per row (its TMEM lane), a named barrier, an mbarrier, 64 TMEM
// columns and a 16 KB operand region:
//   * the thread writes its row's features (BF16, 64 sin/cos pairs) into the
//     region in the canonical K-major no-swizzle layout — 8 x 16-byte core
//     matrices, 8-element K chunks LBO apart, 8-row groups 128 B apart — in
//     two K halves, the first layer accumulating over both;
//   * one thread issues the layer's MMAs (M = 128, N = 64 or 48, K = 16
//     each) against the weights (B, same layout, loaded once per CTA) into
//     the team's TMEM columns and commits them to the team's mbarrier;
//   * every thread waits (bounded), reads its row of the accumulator
//     (tcgen05.ld, 16 columns at a time), adds the bias, applies ReLU and
//     writes the BF16 activations back into the region as the next A tile;
//   * the last layer's 48 outputs (40 used) go to the caller's functor.
// Eight tiles in flight per SM hide one another's MMA round trips. A wait
// that runs out of iterations sets the error word (*err); the team votes, so
// all its threads leave the tile loop together, and the TMEM is freed.
#include <cuda_bf16.h>

#include "ctx.cuh"
#include "guide.cuh"

namespace luc {
namespace tcg {

constexpr int kM = 128;
constexpr uint32_t kLboA = kM * 16;            // A tiles: 128 rows per 8-element K chunk
constexpr uint32_t kLboH = kGHid * 16;         // B tiles of 64 output units
constexpr uint32_t kLboO = kGOutPad * 16;      // B tile of the 48 (40 used) output units
constexpr uint32_t kSbo = 128;                 // 8 rows of 16 B
constexpr uint32_t kTmemCols = 64;

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (Blackwell, version 1): start, leading
// and stride byte offsets >> 4, base offset 0, no swizzle.
__device__ __forceinline__ uint64_t desc(uint32_t a, uint32_t lbo) {
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((kSbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// The same with an explicit stride byte offset: the stride between 8-row
// groups (K-major) or between 8-element MN groups (MN-major, where `lbo` is
// the stride between 8-row K groups).
__device__ __forceinline__ uint64_t desc2(uint32_t a, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor, kind::f16: D F32, A and B BF16, both K-major.
__host__ __device__ constexpr uint32_t idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
}
// With A and/or B read MN-major (bit 15: A, bit 16: B): the operand's
// elements are contiguous along M (N) instead of K, so a tile stored K-major
// for one product is read transposed by another.
__host__ __device__ constexpr uint32_t idesc_mn(int n, bool a_mn, bool b_mn) {
    return idesc(n) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16);
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
__device__ __forceinline__ bool wait_phase(uint32_t mbar, uint32_t phase, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i) {
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

// ---------------------------------------------------------------- teams
// Eight teams per CTA, each a complete 128-row pipeline of its own: four
// warps (one per TMEM lane quadrant, one thread per row), a 16 KB operand
// region (the first layer's features in two K halves, then the hidden
// activations), 64 TMEM columns, an mbarrier and a named barrier. The
// weights are shared. Eight tiles are in flight per SM, so one team's
// features and epilogues overlap the others' MMA round trips.
constexpr int kTeams = 8, kTeamThreads = kM, kTeamCta = kTeams * kTeamThreads;
constexpr uint32_t kRegion = (kGHid / 8) * kLboA;  // 16 KB: 128 rows x 64 BF16

struct TeamSmem {
    uint8_t a[kTeams][kRegion];
    uint8_t w1[(kGIn / 8) * kLboH], w2[(kGHid / 8) * kLboH], w3[(kGHid / 8) * kLboH], w4[(kGHid / 8) * kLboO];
    float b[kGBias];
    unsigned long long mbar[kTeams];
    uint32_t tmem;
};

__device__ __forceinline__ void team_sync(int team) {
    asm volatile("bar.sync %0, %1;" ::"r"(1 + team), "r"(kTeamThreads) : "memory");
}

// Feature pairs [32 h, 32 h + 32) of a row (the K half h of the first
// layer) as 8 chunks of the team's region.
__device__ __forceinline__ void write_feature_half(uint8_t* region, int r, int h, const float (&in)[9],
                                                   const GuideDev& g) {
#pragma unroll
    for (int cc = 0; cc < 8; ++cc) {
        const int c = 8 * h + cc;
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
        *chunk(region, cc, r) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

template <typename Load, typename Store>
__device__ void forward_teams(uint32_t n, const GuideDev& g, uint32_t* err, Load load, Store store) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TeamSmem& S = *reinterpret_cast<TeamSmem*>(smem_raw);
    const int t = threadIdx.x, warp = t >> 5, team = warp >> 2, tt = t & (kTeamThreads - 1);
    const int r = 32 * (warp & 3) + (t & 31);  // this thread's row = its TMEM lane
    {
        auto load_w = [&](uint8_t* dst, const uint16_t* src, int nn, int k, uint32_t lbo) {
            const int chunks = nn * (k / 8);
            for (int i = t; i < chunks; i += blockDim.x) {
                const int row = i / (k / 8), c = i % (k / 8);
                *reinterpret_cast<uint4*>(dst + c * lbo + (row >> 3) * kSbo + (row & 7) * 16) =
                    *reinterpret_cast<const uint4*>(src + row * k + c * 8);
            }
        };
        load_w(S.w1, g.wbf, kGHid, kGIn, kLboH);
        load_w(S.w2, g.wbf + kGHid * kGIn, kGHid, kGHid, kLboH);
        load_w(S.w3, g.wbf + kGHid * kGIn + kGHid * kGHid, kGHid, kGHid, kLboH);
        load_w(S.w4, g.wbf + kGHid * kGIn + 2 * kGHid * kGHid, kGOutPad, kGHid, kLboO);
        for (int i = t; i < kGBias; i += blockDim.x) S.b[i] = g.bias[i];
    }
    if (t < kTeams) {
        asm volatile("mbarrier.init.shared::cta.b64 [%1], %0;" ::"r"(1u), "r"(saddr(&S.mbar[t])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&S.tmem)),
                     "r"(kTeams * kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tcol = S.tmem + kTmemCols * team;  // this team's accumulator columns
    const uint32_t lane_addr = tcol + ((uint32_t)(32 * (warp & 3)) << 16);
    const uint32_t mbar = saddr(&S.mbar[team]);
    uint8_t* region = S.a[team];
    uint32_t phase = 0;
    bool failed = false;
    // MMAs over ksteps k16 steps from the region against w (first: whether D
    // starts fresh), commit, bounded wait; the whole team learns the outcome.
    auto mma_step = [&](const uint8_t* w, uint32_t lbw, int ksteps, int nout, bool fresh) {
        fence_async_smem();
        fence_before();
        team_sync(team);
        fence_after();
        if (tt == 0 && !g.tc_no_issue) {
            for (int ks = 0; ks < ksteps; ++ks)
                mma(tcol, desc(saddr(region) + 2 * ks * kLboA, kLboA), desc(saddr(w) + 2 * ks * lbw, lbw), idesc(nout),
                    (fresh && ks == 0) ? 0u : 1u);
            commit(mbar);
        }
        const bool ok = wait_phase(mbar, phase, g.tc_wait_limit);
        phase ^= 1u;
        fence_after();
        // The team votes on the outcome (threads time out independently),
        // so all of them leave the tile loop together or none does.
        uint32_t any_fail;
        asm volatile(
            "{\n\t.reg .pred q, p;\n\t"
            "setp.ne.u32 q, %1, 0;\n\t"
            "bar.red.or.pred p, %2, %3, q;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(any_fail)
            : "r"(ok ? 0u : 1u), "r"(1 + team), "r"(kTeamThreads)
            : "memory");
        return any_fail == 0u;
    };
    // bias + ReLU of 64 accumulator columns (16 at a time) into the region.
    auto epilogue = [&](const float* b) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float v[16];
            ld16(lane_addr + 16 * q, v);
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                uint32_t w[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int k = 8 * cc + 2 * j, nn = 16 * q + k;
                    w[j] = pack2(fmaxf(v[k] + b[nn], 0.0f), fmaxf(v[k + 1] + b[nn + 1], 0.0f));
                }
                *chunk(region, 2 * q + cc, r) = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
    };
    const uint32_t stride = gridDim.x * kTeams * kM;
    for (uint32_t base = (blockIdx.x * kTeams + team) * kM; base < n; base += stride) {
        const uint32_t row = base + r;
        float in[9] = {0, 0, 0, 0, 0, 1, 0, 0, 1};
        const bool valid = row < n && load(row, in);
        write_feature_half(region, r, 0, in, g);
        bool ok = mma_step(S.w1, kLboH, 4, kGHid, true);
        if (ok) {
            write_feature_half(region, r, 1, in, g);
            ok = mma_step(S.w1 + 8 * kLboH, kLboH, 4, kGHid, false);
        }
        if (ok) {
            epilogue(S.b);
            ok = mma_step(S.w2, kLboH, 4, kGHid, true);
        }
        if (ok) {
            epilogue(S.b + kGHid);
            ok = mma_step(S.w3, kLboH, 4, kGHid, true);
        }
        if (ok) {
            epilogue(S.b + 2 * kGHid);
            ok = mma_step(S.w4, kLboO, 4, kGOutPad, true);
        }
        if (!ok) {
            failed = true;
            break;
        }
        float o[kGOutPad];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            float v[16];
            ld16(lane_addr + 16 * q, v);
#pragma unroll
            for (int k = 0; k < 16; ++k) o[16 * q + k] = v[k] + S.b[3 * kGHid + 16 * q + k];
        }
        if (valid) store(row, o);
        fence_before();
    }
    if (failed && tt == 0) atomicOr(err, 1u);
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(S.tmem), "r"(kTeams * kTmemCols)
                     : "memory");
}

// Raw outputs (bias added) of n rows of 9 inputs: the test-facing forward.
__global__ void __launch_bounds__(kTeamCta, 1) k_forward_tc(const float* __restrict__ in9, uint32_t n, GuideDev g,
                                                   float* __restrict__ out40, uint32_t* err) {
    forward_teams(
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
__global__ void __launch_bounds__(kTeamCta, 1) k_infer_tc(PathState ps, const __grid_constant__ DevScene sc,
                                                 const __grid_constant__ FrameParams fp, uint32_t depth) {
    const uint32_t len = shaded_count(ps, fp, depth);
    forward_teams(
        len, fp.guide, ps.gmisc + kGmTcError,
        [&](uint32_t i, float (&in)[9]) {
            const uint32_t q = shaded_path(ps, fp, depth, i);
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

// ---------------------------------------------------------------- training
// One gradient evaluation on the tensor cores: the tcgen05 counterpart of
// k_guide_train (guide.cu) over the same records, with the same loss, output
// gradient and parameter-gradient layout. One CTA of 128 threads per SM (one
// thread per tile row, its TMEM lane) walks 128-row tiles of records:
//   forward   X -> H1 -> H2 -> H3 -> Y as inference computes it, the BF16
//             activations kept in shared memory in the canonical K-major
//             layout;
//   loss      each thread turns its row's outputs into dL/dY (row_loss_grad),
//             rounded to BF16;
//   backward  dH(l-1) = (dY(l) W(l)) * (H(l-1) > 0), the weights read
//             transposed through MN-major descriptors of their forward
//             layout, and dW(l)^T += H(l-1)^T dY(l) accumulated in TMEM over
//             all of the CTA's tiles, the activation and gradient tiles read
//             transposed the same way (the batch rows are the contraction).
// Bias gradients come out of the same products: each hidden activation tile
// carries a constant upper half (features 64..127) whose feature 64 is 1, so
// row 64 of dW(l)^T (l = 2, 3, 4) is the column sum of dY(l), the gradient
// of b(l); the input tile's padding feature 127 is 1, so row 127 of dW1^T is
// the gradient of b1 (W1's padding columns are zero, so the forward does not
// change). TMEM: columns 0-63 the layer product, 64-127 dW1^T, 128-191
// dW2^T, 192-255 dW3^T, 256-303 dW4^T. At the end each thread reads its
// rows of the gradients into the CTA's slice of `part` (k_guide_fold sums the
// slices in CTA order) and the bias gradients into `grad`.
// A wait that runs out sets gmisc[kGmTcError]; the CTA's slice is zeroed.
struct TrainTcSmem {
    uint8_t x[16 * kLboA];     // 128 rows x 128 features
    uint8_t h[3][16 * kLboA];  // 128 rows x (64 features + the constant half)
    uint8_t dy[6 * kLboA];     // 128 rows x 48 output gradients
    uint8_t dh[2][8 * kLboA];  // 128 rows x 64 hidden gradients, ping-pong
    uint8_t w1[(kGIn / 8) * kLboH], w2[(kGHid / 8) * kLboH], w3[(kGHid / 8) * kLboH], w4[(kGHid / 8) * kLboO];
    float b[kGBias];
    unsigned long long mbar;
    uint32_t tmem;
    float loss;
};
constexpr uint32_t kTrainTmemCols = 512;
constexpr uint32_t kColS = 0, kColW1 = 64, kColW2 = 128, kColW3 = 192, kColW4 = 256;

__global__ void __launch_bounds__(kM, 1) k_guide_train_tc(const float4* __restrict__ rec, uint32_t cap,
                                                          uint32_t* __restrict__ gmisc, GuideDev g,
                                                          float* __restrict__ grad, float* __restrict__ part) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TrainTcSmem& S = *reinterpret_cast<TrainTcSmem*>(smem_raw);
    const int t = threadIdx.x, warp = t >> 5, r = t;
    const uint32_t n = min(gmisc[kGmRecords], cap);
    const float wsum = __uint_as_float(gmisc[kGmWeightSum]);
    const float invS = wsum > 0.0f ? 1.0f / wsum : 0.0f;
    float* P = part + (size_t)blockIdx.x * kPartFloats;
    if (blockIdx.x * (uint32_t)kM >= n) {  // no tile: an all-zero slice
        for (int i = t; i < kPartFloats / 4; i += blockDim.x)
            reinterpret_cast<float4*>(P)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    {
        auto load_w = [&](uint8_t* dst, const uint16_t* src, int nn, int k, uint32_t lbo) {
            const int chunks = nn * (k / 8);
            for (int i = t; i < chunks; i += blockDim.x) {
                const int row = i / (k / 8), c = i % (k / 8);
                *reinterpret_cast<uint4*>(dst + c * lbo + (row >> 3) * kSbo + (row & 7) * 16) =
                    *reinterpret_cast<const uint4*>(src + row * k + c * 8);
            }
        };
        load_w(S.w1, g.wbf, kGHid, kGIn, kLboH);
        load_w(S.w2, g.wbf + kGHid * kGIn, kGHid, kGHid, kLboH);
        load_w(S.w3, g.wbf + kGHid * kGIn + kGHid * kGHid, kGHid, kGHid, kLboH);
        load_w(S.w4, g.wbf + kGHid * kGIn + 2 * kGHid * kGHid, kGOutPad, kGHid, kLboO);
        for (int i = t; i < kGBias; i += blockDim.x) S.b[i] = g.bias[i];
        // The hidden tiles' constant upper half: feature 64 = 1, 65..127 = 0.
        for (int l = 0; l < 3; ++l)
            for (int c = 8; c < 16; ++c)
                *chunk(S.h[l], c, r) = make_uint4(c == 8 ? 0x3F80u : 0u, 0u, 0u, 0u);
    }
    if (t == 0) {
        S.loss = 0.0f;
        asm volatile("mbarrier.init.shared::cta.b64 [%1], %0;" ::"r"(1u), "r"(saddr(&S.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&S.tmem)),
                     "r"(kTrainTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tm = S.tmem;
    const uint32_t lane_off = (uint32_t)(32 * warp) << 16;
    const uint32_t mbar = saddr(&S.mbar);
    uint32_t phase = 0;
    bool failed = false, first = true;
    float loss = 0.0f;
    // One product chain: D[M=128][N] (+)= sum over ksteps of A x B^T.
    auto chain = [&](uint32_t dcol, uint32_t a, uint32_t a_lbo, uint32_t a_sbo, uint32_t a_step, uint32_t b,
                     uint32_t b_lbo, uint32_t b_sbo, uint32_t b_step, int ksteps, uint32_t id, bool fresh) {
        for (int ks = 0; ks < ksteps; ++ks)
            mma(tm + dcol, desc2(a + ks * a_step, a_lbo, a_sbo), desc2(b + ks * b_step, b_lbo, b_sbo), id,
                (fresh && ks == 0) ? 0u : 1u);
    };
    // Issue (one thread), commit, bounded wait; the CTA learns the outcome.
    auto run = [&](auto issue) {
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        if (t == 0 && !g.tc_no_issue) {
            issue();
            commit(mbar);
        }
        const bool ok = wait_phase(mbar, phase, g.tc_wait_limit);
        phase ^= 1u;
        fence_after();
        return __syncthreads_or(ok ? 0 : 1) == 0;
    };
    // Forward products: A = activations (K-major), B = weights (K-major).
    auto fwd = [&](const uint8_t* act, int ksteps, const uint8_t* w, uint32_t lbw, int nout) {
        return run([&] {
            chain(kColS, saddr(act), kLboA, kSbo, 2 * kLboA, saddr(w), lbw, kSbo, 2 * lbw, ksteps, idesc(nout), true);
        });
    };
    // bias + ReLU of the 64 product columns into hidden tile `hout`.
    auto epi_hidden = [&](const float* b, uint8_t* hout) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float v[16];
            ld16(tm + kColS + lane_off + 16 * q, v);
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                uint32_t w[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int k = 8 * cc + 2 * j, nn = 16 * q + k;
                    w[j] = pack2(fmaxf(v[k] + b[nn], 0.0f), fmaxf(v[k + 1] + b[nn + 1], 0.0f));
                }
                *chunk(hout, 2 * q + cc, r) = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
    };
    // The product (dY W) masked by the forward activation (> 0), into `gout`.
    auto epi_grad = [&](const uint8_t* hprev, uint8_t* gout) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float v[16];
            ld16(tm + kColS + lane_off + 16 * q, v);
#pragma unroll
            for (int cc = 0; cc < 2; ++cc) {
                const uint4 hp = *chunk(const_cast<uint8_t*>(hprev), 2 * q + cc, r);
                const uint32_t hw[4] = {hp.x, hp.y, hp.z, hp.w};
                uint32_t w[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int k = 8 * cc + 2 * j;
                    const float h0 = __uint_as_float(hw[j] << 16), h1 = __uint_as_float(hw[j] & 0xFFFF0000u);
                    w[j] = pack2(h0 > 0.0f ? v[k] : 0.0f, h1 > 0.0f ? v[k + 1] : 0.0f);
                }
                *chunk(gout, 2 * q + cc, r) = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
    };
    const uint32_t sx = saddr(S.x), sh0 = saddr(S.h[0]), sh1 = saddr(S.h[1]), sh2 = saddr(S.h[2]);
    const uint32_t sdy = saddr(S.dy), sd0 = saddr(S.dh[0]), sd1 = saddr(S.dh[1]);
    // Backward pair: dH = dY x W (B = W read MN-major: K = output units in
    // 8-row groups 128 B apart, N = input units in groups lbw apart) and
    // dW^T += Hprev^T x dY (both read MN-major: M = Hprev's 128 features in
    // groups kLboA apart, N = dY's units, K = the 128 rows in groups 128 B
    // apart).
    auto back = [&](uint32_t g_tile, int gk, uint32_t w, uint32_t lbw, uint32_t hprev, uint32_t dwcol, int nout) {
        return run([&] {
            chain(kColS, g_tile, kLboA, kSbo, 2 * kLboA, w, kSbo, lbw, 2 * kSbo, gk, idesc_mn(kGHid, false, true),
                  true);
            chain(dwcol, hprev, kSbo, kLboA, 2 * kSbo, g_tile, kSbo, kLboA, 2 * kSbo, kM / 16,
                  idesc_mn(nout, true, true), first);
        });
    };
    for (uint32_t base = blockIdx.x * kM; base < n && !failed; base += gridDim.x * kM) {
        const uint32_t i = base + r;
        const bool mine = i < n;
        float in[9] = {0, 0, 0, 0, 0, 1, 0, 0, 1};
        float4 a4{0, 0, 0, 0}, d4{0, 0, 0, 0};
        if (mine) {
            a4 = rec[kGRecF4 * (size_t)i];
            const float4 b4 = rec[kGRecF4 * (size_t)i + 1], c4 = rec[kGRecF4 * (size_t)i + 2];
            d4 = rec[kGRecF4 * (size_t)i + 3];
            in[0] = a4.x;
            in[1] = a4.y;
            in[2] = a4.z;
            in[3] = b4.x;
            in[4] = b4.y;
            in[5] = b4.z;
            in[6] = c4.x;
            in[7] = c4.y;
            in[8] = c4.z;
        }
        write_feature_half(S.x, r, 0, in, g);               // features 0..63: chunks 0..7
        write_feature_half(S.x + 8 * kLboA, r, 1, in, g);   // features 64..127: chunks 8..15
        *chunk(S.x, 15, r) = make_uint4(0u, 0u, 0u, 0x3F800000u);  // feature 127 = 1 (bias gradient of b1)
        bool ok = fwd(S.x, 8, S.w1, kLboH, kGHid);
        if (ok) {
            epi_hidden(S.b, S.h[0]);
            ok = fwd(S.h[0], 4, S.w2, kLboH, kGHid);
        }
        if (ok) {
            epi_hidden(S.b + kGHid, S.h[1]);
            ok = fwd(S.h[1], 4, S.w3, kLboH, kGHid);
        }
        if (ok) {
            epi_hidden(S.b + 2 * kGHid, S.h[2]);
            ok = fwd(S.h[2], 4, S.w4, kLboO, kGOutPad);
        }
        if (ok) {
            // Loss epilogue: this row's outputs -> dL/dY (BF16) and its loss term.
            float o[kGOutPad], go[kGOut];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                float v[16];
                ld16(tm + kColS + lane_off + 16 * q, v);
#pragma unroll
                for (int k = 0; k < 16; ++k) o[16 * q + k] = v[k] + S.b[3 * kGHid + 16 * q + k];
            }
            if (mine && a4.w > 0.0f) loss += row_loss_grad(o, V3{d4.x, d4.y, d4.z}, a4.w, invS, go);
            else
#pragma unroll
                for (int k = 0; k < kGOut; ++k) go[k] = 0.0f;
#pragma unroll
            for (int c = 0; c < kGOutPad / 8; ++c) {
                uint32_t w[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int k = 8 * c + 2 * j;
                    w[j] = pack2(k < kGOut ? go[k] : 0.0f, k + 1 < kGOut ? go[k + 1] : 0.0f);
                }
                *chunk(S.dy, c, r) = make_uint4(w[0], w[1], w[2], w[3]);
            }
            ok = back(sdy, kGOutPad / 16, saddr(S.w4), kLboO, sh2, kColW4, kGOutPad);
        }
        if (ok) {
            epi_grad(S.h[2], S.dh[0]);
            ok = back(sd0, kGHid / 16, saddr(S.w3), kLboH, sh1, kColW3, kGHid);
        }
        if (ok) {
            epi_grad(S.h[1], S.dh[1]);
            ok = back(sd1, kGHid / 16, saddr(S.w2), kLboH, sh0, kColW2, kGHid);
        }
        if (ok) {
            epi_grad(S.h[0], S.dh[0]);
            ok = run([&] {
                chain(kColW1, sx, kSbo, kLboA, 2 * kSbo, sd0, kSbo, kLboA, 2 * kSbo, kM / 16,
                      idesc_mn(kGHid, true, true), first);
            });
        }
        if (!ok) failed = true;
        first = false;
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (!failed) {
        float* gb1 = grad + kGHid * kGIn;
        float* gb2 = gb1 + kGHid + kGHid * kGHid;
        float* gb3 = gb2 + kGHid + kGHid * kGHid;
        float* gb4 = gb3 + kGHid + kGOut * kGHid;
        // dW1^T: row r = input feature r; row 127 = the gradient of b1.
#pragma unroll 1
        for (int q = 0; q < 4; ++q) {
            float v[16];
            ld16(tm + kColW1 + lane_off + 16 * q, v);
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const int h = 16 * q + k;
                P[kPartW1 + h * kGIn + r] = r < kGFeatures ? v[k] : 0.0f;
                if (r == kGIn - 1) atomicAdd(gb1 + h, v[k]);
            }
        }
        // dW2^T, dW3^T, dW4^T: row r < 64 = input unit r; row 64 = the bias gradient.
        auto read_dw = [&](uint32_t col, int poff, int nout, int nreal, float* gb) {
#pragma unroll 1
            for (int q = 0; q < nout / 16; ++q) {
                float v[16];
                ld16(tm + col + lane_off + 16 * q, v);
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    const int o = 16 * q + k;
                    if (r < kGHid) P[poff + o * kGHid + r] = v[k];
                    else if (r == kGHid && o < nreal) atomicAdd(gb + o, v[k]);
                }
            }
        };
        read_dw(kColW2, kPartW2, kGHid, kGHid, gb2);
        read_dw(kColW3, kPartW3, kGHid, kGHid, gb3);
        read_dw(kColW4, kPartW4, kGOutPad, kGOut, gb4);
    } else {
        for (int i = t; i < kPartFloats / 4; i += blockDim.x)
            reinterpret_cast<float4*>(P)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (t == 0) atomicOr(gmisc + kGmTcError, 1u);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, off);
    if ((t & 31) == 0) atomicAdd(&S.loss, loss);
    fence_before();
    __syncthreads();
    fence_after();
    if (t == 0 && !failed) atomicAdd(reinterpret_cast<float*>(gmisc + kGmLoss), S.loss);
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(kTrainTmemCols)
                     : "memory");
}

}  // namespace tcg
}  // namespace luc

// Dynamic shared memory above 48 KB: opted into once per device, before any
// launch (never inside a stream capture).
cudaError_t guide_tc_setup() {
    using namespace luc;
    cudaError_t e = cudaFuncSetAttribute(tcg::k_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sizeof(tcg::TeamSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(tcg::k_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(tcg::TeamSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(tcg::k_guide_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(tcg::TrainTcSmem));
    return e;
}

// One gradient evaluation on the tensor cores: one CTA per SM at most (512
// TMEM columns and 211 KB of shared memory each), one per 128-row tile of
// `cap` records; returns the grid (the number of gradient slices to fold).
uint32_t launch_guide_gradient_tc(const float4* rec, uint32_t cap, uint32_t* gmisc, const luc::GuideDev& g,
                                  float* grad, float* part, int num_sms, cudaStream_t s) {
    using namespace luc;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>((cap + tcg::kM - 1) / tcg::kM, (uint64_t)num_sms));
    tcg::k_guide_train_tc<<<grid, tcg::kM, sizeof(tcg::TrainTcSmem), s>>>(rec, cap, gmisc, g, grad, part);
    return grid;
}

void launch_guide_infer_tc(const luc::RenderState& rs, const luc::DevScene& sc, const luc::FrameParams& fp,
                           uint32_t depth, cudaStream_t s) {
    using namespace luc;
    // Persistent: one CTA of eight teams per SM (all 512 TMEM columns).
    tcg::k_infer_tc<<<rs.num_sms, tcg::kTeamCta, sizeof(tcg::TeamSmem), s>>>(rs.ps, sc, fp, depth);
}

// Launch the tensor-core forward over n rows of 9 inputs (device arrays).
cudaError_t launch_guide_forward_tc(const float* in9, uint32_t n, const luc::GuideDev& g, float* out40, uint32_t* err,
                                    int num_sms, cudaStream_t s) {
    using namespace luc;
    static const cudaError_t attr = guide_tc_setup();
    if (attr != cudaSuccess) return attr;
    const uint64_t per_cta = (uint64_t)tcg::kTeams * tcg::kM;
    const int grid = (int)std::min<uint64_t>((n + per_cta - 1) / per_cta, (uint64_t)num_sms);
    tcg::k_forward_tc<<<grid, tcg::kTeamCta, sizeof(tcg::TeamSmem), s>>>(in9, n, g, out40, err);
    return cudaGetLastError();
}
