// Learned path-guiding proposal on sm_100a: fused BF16 tensor-core MLP
// kernels (inference per bounce over the path queue; forward + backward +
// weight-gradient accumulation for training), record finalisation and Adam.
// The model and the record layout are described in guide.cuh.
//
// Matrix products use mma.sync m16n8k16 (BF16 inputs, FP32 accumulate). The
// forward pass (inference and training alike) runs a warp's 16 rows entirely
// in registers, layer to layer, with the weights in shared memory fed by
// ldmatrix. Training stores the forward activations as row-major BF16 tiles;
// the backward products read them through ldmatrix (.trans where the product
// needs the transposed operand), so one copy of every tile serves the
// input-gradient and weight-gradient products. A training CTA of 4 warps owns
// a 64-row tile; weight gradients accumulate in shared-memory FP32 across all
// the tiles a persistent CTA processes and reach global memory once per CTA.
//
// Every kernel reads its row count and normalisers from device memory, so the
// per-batch training step (finalise -> train -> Adam -> pack) is captured in
// the frame's CUDA graph with the rest of the batch.
#include <cmath>
#include <cstring>
#include <random>
#include <cuda_bf16.h>
#include "ctx.cuh"

namespace luc {

// Shared-memory row strides (elements), padded by 8 bf16 (16 B) so the eight
// row addresses of an ldmatrix fall in distinct banks.
constexpr int kSIn = kGIn + 8, kSHid = kGHid + 8, kSOut = kGOutPad + 8;
constexpr int kTileRows = 64;
constexpr int kGuideThreads = 128;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x2(uint32_t (&r)[2], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n" : "=r"(r[0]), "=r"(r[1]) : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x2_t(uint32_t (&r)[2], const void* p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ uint16_t to_bf16(float x) {
    __nv_bfloat16 h = __float2bfloat16_rn(x);
    return *reinterpret_cast<uint16_t*>(&h);
}
__device__ __forceinline__ float bf16_to_f(uint16_t h) { return __uint_as_float(((uint32_t)h) << 16); }
__device__ __forceinline__ float u2f(uint32_t u) { return __uint_as_float(u); }

// Shared-memory image of the network (weight row = output unit).
struct NetSmem {
    uint16_t w1[kGHid * kSIn], w2[kGHid * kSHid], w3[kGHid * kSHid], w4[kGOutPad * kSHid];
    float b[kGBias];
};

__device__ __forceinline__ void load_net(NetSmem& s, const uint16_t* __restrict__ wbf, const float* __restrict__ bias) {
    const int t = threadIdx.x, nt = blockDim.x;
    for (int i = t; i < kGHid * kGIn; i += nt) s.w1[(i / kGIn) * kSIn + i % kGIn] = wbf[i];
    const uint16_t* w2 = wbf + kGHid * kGIn;
    for (int i = t; i < kGHid * kGHid; i += nt) s.w2[(i / kGHid) * kSHid + i % kGHid] = w2[i];
    const uint16_t* w3 = w2 + kGHid * kGHid;
    for (int i = t; i < kGHid * kGHid; i += nt) s.w3[(i / kGHid) * kSHid + i % kGHid] = w3[i];
    const uint16_t* w4 = w3 + kGHid * kGHid;
    for (int i = t; i < kGOutPad * kGHid; i += nt) s.w4[(i / kGHid) * kSHid + i % kGHid] = w4[i];
    for (int i = t; i < kGBias; i += nt) s.b[i] = bias[i];
}


// Raw outputs -> (mu, kappa) x 8 and softmax weights.
__device__ __forceinline__ void decode_row(const float* __restrict__ o, float4* __restrict__ lobes, float* __restrict__ w) {
    float mx = -INFINITY;
    for (int j = 0; j < kGLobes; ++j) mx = fmaxf(mx, o[5 * j + 4]);
    float s = 0.0f;
    for (int j = 0; j < kGLobes; ++j) {
        w[j] = expf(o[5 * j + 4] - mx);
        s += w[j];
    }
    for (int j = 0; j < kGLobes; ++j) {
        w[j] /= s;
        float x = o[5 * j], y = o[5 * j + 1], z = o[5 * j + 2];
        float ln = sqrtf(x * x + y * y + z * z);
        float kappa = fminf(1.0f + softplus_f(o[5 * j + 3]), kGKappaMax);
        lobes[j] = ln > 0.0f ? make_float4(x / ln, y / ln, z / ln, kappa) : make_float4(0.f, 0.f, 1.f, kappa);
    }
}

// ---------------------------------------------------------------- inference
// Inference keeps a warp's 16 rows in registers from the features to the
// outputs: the m16n8 accumulator fragments of n-tiles 2j and 2j+1 are, after
// bias, ReLU and BF16 packing, exactly the m16k16 A fragment of k-tile j of
// the next layer, so hidden activations never touch shared memory. The
// features are computed straight into the first layer's A fragments: lane
// (g = lane / 4, t = lane % 4) holds feature pairs 16 kt + 8 h + 2 t of rows g
// and g + 8, and every pair is (sin, cos) of one argument. Only the weights
// (shared by the CTA) and a 16 x 48 FP32 output tile per warp live in shared
// memory.
constexpr int kInferWarps = 8;

struct InferSmem {
    NetSmem net;
    float o[kInferWarps][16 * kGOutPad];
};

// (sin, cos) of feature pair f0 + 2t of one row, packed as bf16x2. f0 is a
// multiple of 8 known at compile time after unrolling, so the input component
// each feature reads is a constant index.
template <int F0>
__device__ __forceinline__ uint32_t feature_pair(const float (&in)[9], const GuideDev& g, int t) {
    if (F0 >= kGFeatures) return 0u;
    float arg;
    if (F0 < 72) {
        constexpr int a = F0 / 24, k0 = (F0 % 24) / 2;
        float q = fminf(fmaxf((in[a] - g.lo[a]) / g.ext[a], 0.0f), 1.0f);
        arg = q * (kPi * (float)(1 << (k0 + t)));
    } else {
        constexpr int r = F0 - 72, comp = 3 + 3 * (r / 24) + (r % 24) / 8;
        arg = in[comp] * (kPi * (float)(1 << t));
    }
    float sn, cs;
    sincosf(arg, &sn, &cs);
    return pack_bf16(sn, cs);
}

template <int KT>
__device__ __forceinline__ void features_kt(uint32_t (&a)[4], const float (&r0)[9], const float (&r1)[9],
                                            const GuideDev& g, int t) {
    a[0] = feature_pair<16 * KT>(r0, g, t);
    a[1] = feature_pair<16 * KT>(r1, g, t);
    a[2] = feature_pair<16 * KT + 8>(r0, g, t);
    a[3] = feature_pair<16 * KT + 8>(r1, g, t);
}

// One hidden layer from register A fragments (KT k-tiles) to the next
// layer's A fragments (N / 16 k-tiles), with bias and ReLU.
template <int KT, int N, int SW>
__device__ __forceinline__ void layer_regs(const uint32_t (&a)[KT][4], const uint16_t* __restrict__ W,
                                           const float* __restrict__ b, uint32_t (&out)[N / 16][4], int lane) {
    const int t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < N / 8; ++nt) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kt = 0; kt < KT; ++kt) {
            uint32_t bf[2];
            ldsm_x2(bf, W + (nt * 8 + (lane & 7)) * SW + kt * 16 + 8 * ((lane >> 3) & 1));
            mma16816(c, a[kt], bf);
        }
        const int n = nt * 8 + 2 * t;
        const float b0 = b[n], b1 = b[n + 1];
        out[nt >> 1][(nt & 1) * 2] = pack_bf16(fmaxf(c[0] + b0, 0.f), fmaxf(c[1] + b1, 0.f));
        out[nt >> 1][(nt & 1) * 2 + 1] = pack_bf16(fmaxf(c[2] + b0, 0.f), fmaxf(c[3] + b1, 0.f));
    }
}

// Store an A-fragment set (KT k-tiles) of rows g, g + 8 as a row-major bf16
// tile (row stride SX), the layout the backward pass reads.
template <int KT, int SX>
__device__ __forceinline__ void store_frags(const uint32_t (&a)[KT][4], uint16_t* __restrict__ x, int lane) {
    const int t = lane & 3, gr = lane >> 2;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
        *reinterpret_cast<uint32_t*>(x + gr * SX + 16 * kt + 2 * t) = a[kt][0];
        *reinterpret_cast<uint32_t*>(x + (gr + 8) * SX + 16 * kt + 2 * t) = a[kt][1];
        *reinterpret_cast<uint32_t*>(x + gr * SX + 16 * kt + 8 + 2 * t) = a[kt][2];
        *reinterpret_cast<uint32_t*>(x + (gr + 8) * SX + 16 * kt + 8 + 2 * t) = a[kt][3];
    }
}

// The warp's forward pass: rows g and g + 8 of this lane's fragments have
// inputs r0 and r1; raw outputs (+ bias) land in o[16][kGOutPad]. With kStore
// the features and the three hidden activations are also written, row-major
// BF16, to x (stride kSIn) and h1, h2, h3 (stride kSHid) for the backward pass.
template <bool kStore>
__device__ __forceinline__ void warp_forward(const NetSmem& net, const GuideDev& g, const float (&r0)[9],
                                             const float (&r1)[9], float* __restrict__ o, int lane,
                                             uint16_t* x = nullptr, uint16_t* h1 = nullptr, uint16_t* h2 = nullptr,
                                             uint16_t* h3 = nullptr) {
    const int t = lane & 3, gr = lane >> 2;
    uint32_t a1[kGIn / 16][4];
    features_kt<0>(a1[0], r0, r1, g, t);
    features_kt<1>(a1[1], r0, r1, g, t);
    features_kt<2>(a1[2], r0, r1, g, t);
    features_kt<3>(a1[3], r0, r1, g, t);
    features_kt<4>(a1[4], r0, r1, g, t);
    features_kt<5>(a1[5], r0, r1, g, t);
    features_kt<6>(a1[6], r0, r1, g, t);
    features_kt<7>(a1[7], r0, r1, g, t);
    if (kStore) store_frags<kGIn / 16, kSIn>(a1, x, lane);
    uint32_t a2[kGHid / 16][4], a3[kGHid / 16][4];
    layer_regs<kGIn / 16, kGHid, kSIn>(a1, net.w1, net.b, a2, lane);
    if (kStore) store_frags<kGHid / 16, kSHid>(a2, h1, lane);
    layer_regs<kGHid / 16, kGHid, kSHid>(a2, net.w2, net.b + kGHid, a3, lane);
    if (kStore) store_frags<kGHid / 16, kSHid>(a3, h2, lane);
    layer_regs<kGHid / 16, kGHid, kSHid>(a3, net.w3, net.b + 2 * kGHid, a2, lane);
    if (kStore) store_frags<kGHid / 16, kSHid>(a2, h3, lane);
    const float* b4 = net.b + 3 * kGHid;
#pragma unroll
    for (int nt = 0; nt < kGOutPad / 8; ++nt) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kt = 0; kt < kGHid / 16; ++kt) {
            uint32_t bf[2];
            ldsm_x2(bf, net.w4 + (nt * 8 + (lane & 7)) * kSHid + kt * 16 + 8 * ((lane >> 3) & 1));
            mma16816(c, a2[kt], bf);
        }
        const int n = nt * 8 + 2 * t;
        *reinterpret_cast<float2*>(o + gr * kGOutPad + n) = make_float2(c[0] + b4[n], c[1] + b4[n + 1]);
        *reinterpret_cast<float2*>(o + (gr + 8) * kGOutPad + n) = make_float2(c[2] + b4[n], c[3] + b4[n + 1]);
    }
}

// Rows g and g + 8 of the inputs held by lanes 0..15 (one row each).
__device__ __forceinline__ void gather_rows(const float (&mine)[9], float (&r0)[9], float (&r1)[9], int lane) {
    const int gr = lane >> 2;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        r0[k] = __shfl_sync(0xFFFFFFFFu, mine[k], gr);
        r1[k] = __shfl_sync(0xFFFFFFFFu, mine[k], gr + 8);
    }
}

// Per bounce: the decoded mixture at every queue position whose ray hit a
// surface (SoA planes of ps.lobe_stride). Inputs are the hit point, the
// shading normal and the outgoing direction -dir, as SHADE computes them.
// Each warp takes 32 queue positions at a time (every lane fetches one hit, so
// the dependent loads of all 32 overlap), then runs them through the network
// as two groups of 16 rows; two lanes decode a row (four lobes each, softmax
// across the pair).
__global__ void __launch_bounds__(kInferWarps * 32) k_guide_infer(PathState ps, DevScene sc, FrameParams fp,
                                                                   uint32_t depth) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    InferSmem& S = *reinterpret_cast<InferSmem*>(smem_raw);
    load_net(S.net, fp.guide.wbf, fp.guide.bias);
    __syncthreads();
    const uint32_t len = shaded_count(ps, fp, depth);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* o = S.o[warp];
    const uint32_t nwarps = gridDim.x * kInferWarps;
    for (uint32_t base = (blockIdx.x * kInferWarps + warp) * 32u; base < len; base += nwarps * 32u) {
        float in[9] = {0, 0, 0, 0, 0, 1, 0, 0, 1};
        bool hit_row = false;
        if (base + lane < len) {
            const uint32_t i = base + lane;
            const uint32_t q = shaded_path(ps, fp, depth, i);
            const float4 h4 = ps.hit[q];
            const uint32_t id = __float_as_uint(h4.w);
            if (id != kMiss) {
                hit_row = true;
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
            }
        }
        const uint32_t hits = __ballot_sync(0xFFFFFFFFu, hit_row);
#pragma unroll 1
        for (int half = 0; half < 2; ++half) {
            const uint32_t hh = (hits >> (16 * half)) & 0xFFFFu;
            if (hh == 0) continue;  // uniform across the warp
            float r0[9], r1[9];
            const int gr = (lane >> 2) + 16 * half;
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                r0[k] = __shfl_sync(0xFFFFFFFFu, in[k], gr);
                r1[k] = __shfl_sync(0xFFFFFFFFu, in[k], gr + 8);
            }
            warp_forward<false>(S.net, fp.guide, r0, r1, o, lane);
            __syncwarp();
            // Decode: lanes 2r and 2r + 1 share row r, lobes 4h .. 4h + 3.
            const int r = lane >> 1, h = lane & 1;
            const float* orow = o + r * kGOutPad + 20 * h;
            float lg[4], mx = -INFINITY;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                lg[j] = orow[5 * j + 4];
                mx = fmaxf(mx, lg[j]);
            }
            mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, 1));
            float e[4], sum = 0.f;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                e[j] = expf(lg[j] - mx);
                sum += e[j];
            }
            sum += __shfl_xor_sync(0xFFFFFFFFu, sum, 1);
            if ((hh >> r) & 1u) {
                const size_t st = ps.lobe_stride, i = base + 16 * half + r;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float x = orow[5 * j], y = orow[5 * j + 1], z = orow[5 * j + 2];
                    const float ln = sqrtf(x * x + y * y + z * z);
                    const float kappa = fminf(1.0f + softplus_f(orow[5 * j + 3]), kGKappaMax);
                    ps.lobes[(4 * h + j) * st + i] =
                        ln > 0.0f ? make_float4(x / ln, y / ln, z / ln, kappa) : make_float4(0.f, 0.f, 1.f, kappa);
                }
                ps.lobes[(8 + h) * st + i] = make_float4(e[0] / sum, e[1] / sum, e[2] / sum, e[3] / sum);
            }
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------- training
// Under 113 KB, so two CTAs (8 warps) share an SM: the weight gradients
// accumulate in each CTA's slice of a global buffer (kPartFloats per CTA,
// L2-resident; each warp owns its rows, so plain read-modify-write), and the
// raw outputs share the input-gradient planes (outputs are dead once the
// loss epilogue has turned them into dy).
struct TrainSmem {
    NetSmem net;
    float db[kGBias];
    uint16_t x[kTileRows * kSIn];
    uint16_t h[3][kTileRows * kSHid];
    uint16_t dy[kTileRows * kSOut];
    union {
        uint16_t dh[2][kTileRows * kSHid];
        float o[kTileRows * kGOutPad];
    };
    float loss;
};
static_assert(sizeof(TrainSmem) <= 113 * 1024, "two training CTAs per SM");

// dW[m][n] += sum_r G[r][m] H[r][n] over the tile's 64 rows for the 16 output
// rows m0..m0+15. G is [64][SG] (m contiguous), H is [64][SH]; both operands
// come through ldmatrix.trans, so neither is ever stored transposed.
template <int NIN, int SH, int SG>
__device__ void acc_weight_grad(const uint16_t* __restrict__ G, const uint16_t* __restrict__ H, float* __restrict__ dW,
                                int m0, int lane) {
    const int g = lane >> 2, t = lane & 3;
    uint32_t af[kTileRows / 16][4];
#pragma unroll
    for (int kt = 0; kt < kTileRows / 16; ++kt)
        ldsm_x4_t(af[kt], G + (kt * 16 + (lane & 7) + 8 * (lane >> 4)) * SG + m0 + 8 * ((lane >> 3) & 1));
#pragma unroll 4
    for (int nt = 0; nt < NIN / 8; ++nt) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kt = 0; kt < kTileRows / 16; ++kt) {
            uint32_t bf[2];
            ldsm_x2_t(bf, H + (kt * 16 + (lane & 7) + 8 * ((lane >> 3) & 1)) * SH + nt * 8);
            mma16816(c, af[kt], bf);
        }
        const int n = nt * 8 + 2 * t;
        float2* d0 = reinterpret_cast<float2*>(dW + (m0 + g) * NIN + n);
        float2* d1 = reinterpret_cast<float2*>(dW + (m0 + g + 8) * NIN + n);
        float2 a0 = *d0, a1 = *d1;
        *d0 = make_float2(a0.x + c[0], a0.y + c[1]);
        *d1 = make_float2(a1.x + c[2], a1.y + c[3]);
    }
}

// dH[r][k] = (sum_n G[r][n] W[n][k]) * (Hprev[r][k] > 0) for the warp's 16
// rows, and db[k] += the column sums of that FP32 value.
template <int NOUT, int SG>
__device__ void input_grad(const uint16_t* __restrict__ G, const uint16_t* __restrict__ W, const uint16_t* __restrict__ Hp,
                           uint16_t* __restrict__ dH, float* __restrict__ db, int r0, int lane) {
    const int g = lane >> 2, t = lane & 3;
    uint32_t af[NOUT / 16][4];
#pragma unroll
    for (int kt = 0; kt < NOUT / 16; ++kt)
        ldsm_x4(af[kt], G + (r0 + (lane & 7) + 8 * ((lane >> 3) & 1)) * SG + kt * 16 + 8 * (lane >> 4));
#pragma unroll
    for (int nt = 0; nt < kGHid / 8; ++nt) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kt = 0; kt < NOUT / 16; ++kt) {
            uint32_t bf[2];
            ldsm_x2_t(bf, W + (kt * 16 + (lane & 7) + 8 * ((lane >> 3) & 1)) * kSHid + nt * 8);
            mma16816(c, af[kt], bf);
        }
        const int n = nt * 8 + 2 * t;
        const uint16_t* h0 = Hp + (r0 + g) * kSHid + n;
        const uint16_t* h1 = Hp + (r0 + g + 8) * kSHid + n;
        float v0 = bf16_to_f(h0[0]) > 0.f ? c[0] : 0.f, v1 = bf16_to_f(h0[1]) > 0.f ? c[1] : 0.f;
        float v2 = bf16_to_f(h1[0]) > 0.f ? c[2] : 0.f, v3 = bf16_to_f(h1[1]) > 0.f ? c[3] : 0.f;
        *reinterpret_cast<uint32_t*>(dH + (r0 + g) * kSHid + n) = pack_bf16(v0, v1);
        *reinterpret_cast<uint32_t*>(dH + (r0 + g + 8) * kSHid + n) = pack_bf16(v2, v3);
        float s0 = v0 + v2, s1 = v1 + v3;
#pragma unroll
        for (int off = 4; off < 32; off <<= 1) {
            s0 += __shfl_xor_sync(0xFFFFFFFFu, s0, off);
            s1 += __shfl_xor_sync(0xFFFFFFFFu, s1, off);
        }
        if (g == 0) {
            atomicAdd(db + n, s0);
            atomicAdd(db + n + 1, s1);
        }
    }
}

// One gradient evaluation over the records (count gmisc[kGmRecords], capped
// at `cap`; normaliser 1 / gmisc[kGmWeightSum]) added into grad (FP32, master
// layout), and the loss into gmisc[kGmLoss].
__global__ void __launch_bounds__(kGuideThreads, 2) k_guide_train(const float4* __restrict__ rec, uint32_t cap,
                                                                   uint32_t* __restrict__ gmisc, GuideDev g,
                                                                   float* __restrict__ grad, float* __restrict__ part) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
    const uint32_t n = min(gmisc[kGmRecords], cap);
    const float wsum = u2f(gmisc[kGmWeightSum]);
    const float invS = wsum > 0.0f ? 1.0f / wsum : 0.0f;
    // This CTA's gradient slice starts at zero, tiles or not (k_guide_fold
    // sums every slice).
    float* P = part + (size_t)blockIdx.x * kPartFloats;
    for (int i = threadIdx.x; i < kPartFloats / 4; i += blockDim.x)
        reinterpret_cast<float4*>(P)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (blockIdx.x * kTileRows >= n) return;
    load_net(S.net, g.wbf, g.bias);
    for (int i = threadIdx.x; i < kGBias; i += blockDim.x) S.db[i] = 0.f;
    if (threadIdx.x == 0) S.loss = 0.f;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, r0 = warp * 16;
    for (uint32_t base = blockIdx.x * kTileRows; base < n; base += gridDim.x * kTileRows) {
        const uint32_t i = base + r0 + lane;
        const bool mine = lane < 16 && i < n;
        float in[9] = {0, 0, 0, 0, 0, 1, 0, 0, 1};
        float4 a4{0, 0, 0, 0}, d4{0, 0, 0, 0};
        if (mine) {
            a4 = rec[kGRecF4 * (size_t)i];
            float4 b4 = rec[kGRecF4 * (size_t)i + 1], c4 = rec[kGRecF4 * (size_t)i + 2];
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
        float ra[9], rb[9];
        gather_rows(in, ra, rb, lane);
        warp_forward<true>(S.net, g, ra, rb, S.o + r0 * kGOutPad, lane, S.x + r0 * kSIn, S.h[0] + r0 * kSHid,
                           S.h[1] + r0 * kSHid, S.h[2] + r0 * kSHid);
        __syncwarp();
        // Loss epilogue: lanes 0..15, one row each.
        if (lane < 16) {
            const int r = r0 + lane;
            float go[kGOut];
            float lrow = 0.f;
            if (mine && a4.w > 0.0f) {
                lrow = row_loss_grad(S.o + r * kGOutPad, V3{d4.x, d4.y, d4.z}, a4.w, invS, go);
            } else {
                for (int k = 0; k < kGOut; ++k) go[k] = 0.f;
            }
#pragma unroll
            for (int k = 0; k < kGOutPad; k += 2) {
                float v0 = k < kGOut ? go[k] : 0.f, v1 = k + 1 < kGOut ? go[k + 1] : 0.f;
                *reinterpret_cast<uint32_t*>(S.dy + r * kSOut + k) = pack_bf16(v0, v1);
            }
            // Output-bias gradient: reduce over the 16 rows, then one atomic.
#pragma unroll
            for (int k = 0; k < kGOut; ++k) {
                float v = go[k];
                for (int off = 8; off > 0; off >>= 1) v += __shfl_xor_sync(0x0000FFFFu, v, off);
                if (lane == 0) atomicAdd(S.db + 3 * kGHid + k, v);
            }
            for (int off = 8; off > 0; off >>= 1) lrow += __shfl_xor_sync(0x0000FFFFu, lrow, off);
            if (lane == 0) atomicAdd(&S.loss, lrow);
        }
        __syncthreads();
        // Layer 4: dW4 (48 rows: warps 0..2, 16 each) and dH3.
        if (warp < 3) acc_weight_grad<kGHid, kSHid, kSOut>(S.dy, S.h[2], P + kPartW4, warp * 16, lane);
        input_grad<kGOutPad, kSOut>(S.dy, S.net.w4, S.h[2], S.dh[0], S.db + 2 * kGHid, r0, lane);
        __syncthreads();
        acc_weight_grad<kGHid, kSHid, kSHid>(S.dh[0], S.h[1], P + kPartW3, warp * 16, lane);
        input_grad<kGHid, kSHid>(S.dh[0], S.net.w3, S.h[1], S.dh[1], S.db + kGHid, r0, lane);
        __syncthreads();
        acc_weight_grad<kGHid, kSHid, kSHid>(S.dh[1], S.h[0], P + kPartW2, warp * 16, lane);
        input_grad<kGHid, kSHid>(S.dh[1], S.net.w2, S.h[0], S.dh[0], S.db, r0, lane);
        __syncthreads();
        acc_weight_grad<kGIn, kSIn, kSHid>(S.dh[0], S.x, P + kPartW1, warp * 16, lane);
        __syncthreads();
    }
    // Bias gradients and loss into the global FP32 gradient (layout W1 b1 W2
    // b2 W3 b3 W4 b4); the weight gradients stay in this CTA's slice for
    // k_guide_fold.
    float* gb1 = grad + kGHid * kGIn;
    float* gb2 = gb1 + kGHid + kGHid * kGHid;
    float* gb3 = gb2 + kGHid + kGHid * kGHid;
    float* gb4 = gb3 + kGHid + kGOut * kGHid;
    for (int i = threadIdx.x; i < kGHid; i += blockDim.x) {
        atomicAdd(gb1 + i, S.db[i]);
        atomicAdd(gb2 + i, S.db[kGHid + i]);
        atomicAdd(gb3 + i, S.db[2 * kGHid + i]);
    }
    for (int i = threadIdx.x; i < kGOut; i += blockDim.x) atomicAdd(gb4 + i, S.db[3 * kGHid + i]);
    if (threadIdx.x == 0) atomicAdd(reinterpret_cast<float*>(gmisc + kGmLoss), S.loss);
}

// Sum of the CTAs' weight-gradient slices into the FP32 gradient (added to
// what the training kernel put there: the bias gradients). One thread per
// weight, slices in CTA order: the sum is deterministic.
__global__ void k_guide_fold(const float* __restrict__ part, uint32_t nparts, float* __restrict__ grad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kPartFloats) return;
    int dst;
    if (i < kPartW2) dst = i;                                        // W1
    else if (i < kPartW3) dst = kGHid * kGIn + kGHid + (i - kPartW2);  // W2
    else if (i < kPartW4) dst = kGHid * kGIn + 2 * kGHid + kGHid * kGHid + (i - kPartW3);  // W3
    else if (i - kPartW4 < kGOut * kGHid)
        dst = kGHid * kGIn + 3 * kGHid + 2 * kGHid * kGHid + (i - kPartW4);  // W4 (padding rows dropped)
    else return;
    float s = 0.f;
    for (uint32_t c = 0; c < nparts; ++c) s += part[(size_t)c * kPartFloats + i];
    grad[dst] += s;
}

// The training kernel's grid: one CTA per 64-row tile, at most two per SM.
uint32_t guide_train_grid(uint32_t cap, int num_sms) {
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((cap + kTileRows - 1) / kTileRows, 2ull * num_sms));
}
size_t guide_part_bytes(int num_sms) { return (size_t)2 * num_sms * kPartFloats * sizeof(float); }

// One gradient evaluation over records rec[0, min(count, cap)) into grad
// (zeroed here) and the loss word.
// tc: the tcgen05 kernel (guide_tc.cu), else the mma.sync one.
void launch_guide_gradient(const float4* rec, uint32_t cap, uint32_t* gmisc, const GuideDev& g, float* grad,
                           float* part, int num_sms, bool tc, cudaStream_t s) {
    cudaMemsetAsync(grad, 0, kGParams * sizeof(float), s);
    uint32_t grid;
    if (tc) {
        grid = launch_guide_gradient_tc(rec, cap, gmisc, g, grad, part, num_sms, s);
    } else {
        grid = guide_train_grid(cap, num_sms);
        k_guide_train<<<grid, kGuideThreads, sizeof(TrainSmem), s>>>(rec, cap, gmisc, g, grad, part);
    }
    k_guide_fold<<<(kPartFloats + 255) / 256, 256, 0, s>>>(part, grid, grad);
}

// Records of a rendered batch: F = luminance of the radiance that arrived
// along the sampled direction (the path radiance gained after the vertex,
// divided per channel by the throughput after scattering) over the mixture
// pdf, into rec[0].w; the sum of F into gmisc[kGmWeightSum].
__global__ void k_guide_finalize(PathState ps, uint32_t cap) {
    const uint32_t n = min(ps.gmisc[kGmRecords], cap);
    float s = 0.f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4* r = ps.rec + kGRecF4 * (size_t)i;
        float4 a = r[0], b = r[1], c = r[2], d = r[3], e = r[4];
        const uint32_t p = __float_as_uint(a.w);
        float4 rf = ps.rad[p];
        const float T[3] = {b.w, c.w, d.w};
        const float dR[3] = {rf.x - e.x, rf.y - e.y, rf.z - e.z};
        const float lw[3] = {0.2126f, 0.7152f, 0.0722f};
        float L = 0.f;
        for (int k = 0; k < 3; ++k)
            if (T[k] > 0.f) L += lw[k] * dR[k] / T[k];
        float F = L > 0.f && e.w > 0.f ? L / e.w : 0.f;
        if (!isfinite(F)) F = 0.f;
        r[0].w = F;
        s += F;
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, off);
    if ((threadIdx.x & 31) == 0 && s != 0.f) atomicAdd(reinterpret_cast<float*>(ps.gmisc + kGmWeightSum), s);
}

// Sum of F over host-given records.
__global__ void k_guide_weight_sum(const float4* __restrict__ rec, uint32_t n, uint32_t* __restrict__ gmisc) {
    float s = 0.f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        s += fmaxf(rec[kGRecF4 * (size_t)i].w, 0.f);
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xFFFFFFFFu, s, off);
    if ((threadIdx.x & 31) == 0 && s != 0.f) atomicAdd(reinterpret_cast<float*>(gmisc + kGmWeightSum), s);
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the FP32 master; the step
// number comes from gmisc[kGmStep] (advanced by k_guide_pack).
__global__ void k_guide_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                             const float* __restrict__ grad, const uint32_t* __restrict__ gmisc, float lr) {
    const float t = (float)(gmisc[kGmStep] + 1u);
    const float c1 = 1.0f - powf(0.9f, t), c2 = 1.0f - powf(0.999f, t);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGParams; i += gridDim.x * blockDim.x) {
        float gi = grad[i];
        float mi = 0.9f * m[i] + 0.1f * gi;
        float vi = 0.999f * v[i] + 0.001f * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
    }
}

// Pack the master into BF16 weights (W4 zero-padded to 48 rows) and FP32
// biases. With `advance`, block 0 thread 0 also closes the step: step count,
// last loss and record count, the recording threshold for the next batch
// (aiming at `cap` records from this batch's candidate count) and the
// per-batch counters reset.
__global__ void k_guide_pack(const float* __restrict__ p, uint16_t* __restrict__ wbf, float* __restrict__ bias,
                             uint32_t* __restrict__ gmisc, uint32_t cap, uint32_t advance) {
    const float* W1 = p;
    const float* b1 = W1 + kGHid * kGIn;
    const float* W2 = b1 + kGHid;
    const float* b2 = W2 + kGHid * kGHid;
    const float* W3 = b2 + kGHid;
    const float* b3 = W3 + kGHid * kGHid;
    const float* W4 = b3 + kGHid;
    const float* b4 = W4 + kGOut * kGHid;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGBf16; i += gridDim.x * blockDim.x) {
        float x;
        if (i < kGHid * kGIn) x = W1[i];
        else if (i < kGHid * kGIn + kGHid * kGHid) x = W2[i - kGHid * kGIn];
        else if (i < kGHid * kGIn + 2 * kGHid * kGHid) x = W3[i - kGHid * kGIn - kGHid * kGHid];
        else {
            int j = i - kGHid * kGIn - 2 * kGHid * kGHid;
            x = j < kGOut * kGHid ? W4[j] : 0.0f;
        }
        wbf[i] = to_bf16(x);
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGBias; i += gridDim.x * blockDim.x) {
        float x;
        if (i < kGHid) x = b1[i];
        else if (i < 2 * kGHid) x = b2[i - kGHid];
        else if (i < 3 * kGHid) x = b3[i - 2 * kGHid];
        else x = (i - 3 * kGHid) < kGOut ? b4[i - 3 * kGHid] : 0.0f;
        bias[i] = x;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && advance) {
        gmisc[kGmStep] += 1u;
        gmisc[kGmLastLoss] = gmisc[kGmLoss];
        gmisc[kGmLastRecords] = min(gmisc[kGmRecords], cap);
        const uint32_t cand = gmisc[kGmCandidates];
        if (cand > 0) {
            uint64_t t = (uint64_t)65536 * cap * 15 / 16 / cand;
            gmisc[kGmThreshold] = (uint32_t)(t > 65536 ? 65536 : (t == 0 ? 1 : t));
        }
        gmisc[kGmCandidates] = 0;
        gmisc[kGmRecords] = 0;
    }
}

// Raw outputs for host-given inputs (x, n, wo per row): the inference
// kernel's forward pass, without the decode.
__global__ void __launch_bounds__(kInferWarps * 32) k_guide_forward(const float* __restrict__ in9, uint32_t n,
                                                                     GuideDev g, float* __restrict__ out40) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    InferSmem& S = *reinterpret_cast<InferSmem*>(smem_raw);
    load_net(S.net, g.wbf, g.bias);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float* o = S.o[warp];
    const uint32_t nwarps = gridDim.x * kInferWarps;
    for (uint32_t base = (blockIdx.x * kInferWarps + warp) * 16u; base < n; base += nwarps * 16u) {
        float in[9] = {0, 0, 0, 0, 0, 1, 0, 0, 1};
        if (lane < 16 && base + lane < n)
            for (int k = 0; k < 9; ++k) in[k] = in9[9 * (size_t)(base + lane) + k];
        float r0[9], r1[9];
        gather_rows(in, r0, r1, lane);
        warp_forward<false>(S.net, g, r0, r1, o, lane);
        __syncwarp();
        for (int k = lane; k < 16 * kGOut; k += 32) {
            const int r = k / kGOut, c = k % kGOut;
            if (base + r < n) out40[(size_t)(base + r) * kGOut + c] = o[r * kGOutPad + c];
        }
        __syncwarp();
    }
}

// Mixture sampling (mode 0: in3 = uniforms; out dir3 and pdf) and density
// (mode 1: in3 = directions; out pdf) for given raw outputs.
__global__ void k_guide_mixture_eval(const float* __restrict__ raw40, const float* __restrict__ in3, uint32_t n, int mode,
                                     float* __restrict__ dir3, float* __restrict__ pdf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 lobes[kGLobes];
    float w[kGLobes];
    decode_row(raw40 + (size_t)i * kGOut, lobes, w);
    Mixture m;
    for (int j = 0; j < kGLobes; ++j) {
        m.lobe[j] = lobes[j];
        m.w[j] = w[j];
    }
    V3 d;
    if (mode == 0) {
        d = mixture_sample(m, in3[3 * i], in3[3 * i + 1], in3[3 * i + 2]);
        dir3[3 * i] = d.x;
        dir3[3 * i + 1] = d.y;
        dir3[3 * i + 2] = d.z;
    } else {
        d = V3{in3[3 * i], in3[3 * i + 1], in3[3 * i + 2]};
    }
    pdf[i] = mixture_pdf(m, d);
}

static int g_infer_blocks = 1;

// Dynamic shared memory above 48 KB needs an opt-in per kernel; done once
// per device, before any launch (never inside a stream capture).
static cudaError_t guide_kernel_setup(int device) {
    static bool done[64] = {false};
    if (device >= 0 && device < 64 && done[device]) return cudaSuccess;
    cudaError_t e =
        cudaFuncSetAttribute(k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(InferSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guide_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(InferSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guide_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_guide_train, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess) e = guide_tc_setup();
    if (e != cudaSuccess) return e;
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_guide_infer, kInferWarps * 32, sizeof(InferSmem));
    g_infer_blocks = b > 0 ? b : 1;
    if (device >= 0 && device < 64) done[device] = true;
    return cudaSuccess;
}

// Per bounce: the guide's mixtures for the queued paths, by default on the
// tcgen05 team kernel (guide_tc.cu: 1.14 ms per 1-spp 1024^2 guided frame);
// LUC_GUIDE_TC=0 selects the register-chained mma.sync kernel (1.45 ms)
// per context. Both give the same mixtures bit for bit.
void launch_guide_infer(const RenderState& rs, const DevScene& sc, const FrameParams& fp, uint32_t depth,
                        cudaStream_t s) {
    if (rs.guide_tc) launch_guide_infer_tc(rs, sc, fp, depth, s);
    else k_guide_infer<<<rs.num_sms * g_infer_blocks, kInferWarps * 32, sizeof(InferSmem), s>>>(rs.ps, sc, fp, depth);
}

void launch_guide_finalize(const RenderState& rs, const FrameParams& fp, cudaStream_t s) {
    cudaMemsetAsync(rs.ps.gmisc + kGmWeightSum, 0, 2 * sizeof(uint32_t), s);  // weight sum, loss
    k_guide_finalize<<<rs.num_sms * 4, 256, 0, s>>>(rs.ps, fp.rec_cap);
}

void launch_guide_step(const RenderState& rs, uint32_t cap, const GuideDev& g, const GuideTrain& gt, cudaStream_t s) {
    launch_guide_gradient(rs.ps.rec, cap, rs.ps.gmisc, g, gt.grad, gt.part, rs.num_sms, rs.guide_tc, s);
    k_guide_adam<<<(kGParams + 255) / 256, 256, 0, s>>>(gt.params, gt.m, gt.v, gt.grad, rs.ps.gmisc, gt.lr);
    k_guide_pack<<<(kGBf16 + 255) / 256, 256, 0, s>>>(gt.params, gt.wbf, gt.bias, rs.ps.gmisc, cap, 1u);
}

void launch_guide_train(const RenderState& rs, const FrameParams& fp, const GuideTrain& gt, cudaStream_t s) {
    launch_guide_finalize(rs, fp, s);
    launch_guide_step(rs, fp.rec_cap, fp.guide, gt, s);
}

}  // namespace luc

using namespace luc;

// ------------------------------------------------------------------ context side
static int32_t require_guide(luc_ctx* c) {
    if (!c->guide_ready) return luc_fail(c, LUC_ERR_VALIDATION, "guide not initialised (luc_guide_init)");
    return LUC_OK;
}

GuideDev luc_guide_dev(const luc_ctx* c) {
    GuideDev g{};
    g.wbf = c->g_wbf.as<uint16_t>();
    g.bias = c->g_bias.as<float>();
    g.tc_wait_limit = kTcWaitLimit;
    g.tc_no_issue = 0;
    for (int a = 0; a < 3; ++a) {
        g.lo[a] = c->guide_lo[a];
        g.ext[a] = c->guide_hi[a] > c->guide_lo[a] ? c->guide_hi[a] - c->guide_lo[a] : 1.0f;
    }
    return g;
}

GuideTrain luc_guide_train_state(luc_ctx* c) {
    GuideTrain gt{};
    gt.params = c->g_params.as<float>();
    gt.m = c->g_m.as<float>();
    gt.v = c->g_v.as<float>();
    gt.grad = c->g_grad.as<float>();
    gt.wbf = c->g_wbf.as<uint16_t>();
    gt.bias = c->g_bias.as<float>();
    gt.part = c->g_part.as<float>();
    gt.lr = c->guide_lr;
    gt.train = c->guide_train;
    return gt;
}

// A gradient step left pending by a guided frame (GuideTrain::defer) runs
// now, on the context's stream, before anything reads or changes the guide.
int32_t luc_guide_flush(luc_ctx* c) {
    if (!c->guide_pending) return LUC_OK;
    c->guide_pending = false;
    cudaSetDevice(c->device);
    launch_guide_step(c->rs, c->guide_pending_cap, luc_guide_dev(c), luc_guide_train_state(c), c->stream);
    LUC_CUDA(c, cudaGetLastError(), "guide step");
    return LUC_OK;
}

int32_t luc_guide_prepare_frame(luc_ctx* c, uint64_t paths) {
    if (int32_t rc = require_guide(c)) return rc;
    LUC_CUDA(c, guide_kernel_setup(c->device), "guide kernel attributes");
    LUC_CUDA(c, c->g_lobes.ensure(paths * kGLobeF4 * sizeof(float4)), "allocate guide lobes");
    LUC_CUDA(c, c->g_rec.ensure((size_t)std::max<uint32_t>(c->guide_rec_cap, 1) * kGRecF4 * sizeof(float4)),
             "allocate guide records");
    LUC_CUDA(c, c->g_part.ensure(guide_part_bytes(c->num_sms)), "allocate guide gradient slices");
    return LUC_OK;
}

// ------------------------------------------------------------------ C ABI
extern "C" {

int32_t luc_guide_init(luc_ctx* c, const float* params, uint64_t seed, const float* lo, const float* hi) {
    if (!c) return LUC_ERR_VALIDATION;
    cudaSetDevice(c->device);
    if ((lo == nullptr) != (hi == nullptr)) return luc_fail(c, LUC_ERR_VALIDATION, "give both lo and hi or neither");
    if (!lo && !c->has_scene) return luc_fail(c, LUC_ERR_VALIDATION, "no scene bounds: upload a scene or give lo/hi");
    for (int a = 0; a < 3; ++a) {
        c->guide_lo[a] = lo ? lo[a] : c->scene_lo[a];
        c->guide_hi[a] = hi ? hi[a] : c->scene_hi[a];
        if (!std::isfinite(c->guide_lo[a]) || !std::isfinite(c->guide_hi[a]))
            return luc_fail(c, LUC_ERR_VALIDATION, "guide bounds must be finite");
    }
    LUC_CUDA(c, guide_kernel_setup(c->device), "guide kernel attributes");
    std::vector<float> p(kGParams, 0.0f);
    if (params) {
        std::memcpy(p.data(), params, kGParams * sizeof(float));
        // W1's padding columns multiply features that are always zero; they
        // are held at zero (the tensor-core training kernel sets padding
        // feature 127 to 1 to read b1's gradient out of its dW1 product).
        for (int r = 0; r < kGHid; ++r)
            for (int k = kGFeatures; k < kGIn; ++k) p[(size_t)r * kGIn + k] = 0.0f;
    } else {
        // Uniform +-sqrt(6 / (fan_in + fan_out)) weights, zero biases, W1's
        // padding columns zero.
        std::mt19937_64 rng(seed);
        const int fan[4][2] = {{kGHid, kGIn}, {kGHid, kGHid}, {kGHid, kGHid}, {kGOut, kGHid}};
        size_t o = 0;
        for (int l = 0; l < 4; ++l) {
            float lim = std::sqrt(6.0f / (float)(fan[l][0] + fan[l][1]));
            std::uniform_real_distribution<float> U(-lim, lim);
            for (int r = 0; r < fan[l][0]; ++r)
                for (int k = 0; k < fan[l][1]; ++k)
                    p[o + (size_t)r * fan[l][1] + k] = (l == 0 && k >= kGFeatures) ? 0.0f : U(rng);
            o += (size_t)fan[l][0] * fan[l][1] + fan[l][0];
        }
    }
    for (float x : p)
        if (!std::isfinite(x)) return luc_fail(c, LUC_ERR_VALIDATION, "guide parameters must be finite");
    cudaStream_t s = c->stream;
    c->guide_pending = false;  // a step of the guide being replaced
    LUC_CUDA(c, c->g_params.ensure(kGParams * sizeof(float)), "allocate guide");
    LUC_CUDA(c, c->g_m.ensure(kGParams * sizeof(float)), "allocate guide");
    LUC_CUDA(c, c->g_v.ensure(kGParams * sizeof(float)), "allocate guide");
    LUC_CUDA(c, c->g_grad.ensure(kGParams * sizeof(float)), "allocate guide");
    LUC_CUDA(c, c->g_wbf.ensure(kGBf16 * sizeof(uint16_t)), "allocate guide");
    LUC_CUDA(c, c->g_bias.ensure(kGBias * sizeof(float)), "allocate guide");
    LUC_CUDA(c, c->g_misc.ensure(kGmWords * sizeof(uint32_t)), "allocate guide");
    LUC_CUDA(c, cudaMemcpyAsync(c->g_params.p, p.data(), kGParams * sizeof(float), cudaMemcpyHostToDevice, s),
             "upload guide");
    LUC_CUDA(c, cudaMemsetAsync(c->g_m.p, 0, kGParams * sizeof(float), s), "clear guide");
    LUC_CUDA(c, cudaMemsetAsync(c->g_v.p, 0, kGParams * sizeof(float), s), "clear guide");
    uint32_t misc[kGmWords] = {0};
    misc[kGmThreshold] = 65536;
    LUC_CUDA(c, cudaMemcpyAsync(c->g_misc.p, misc, sizeof(misc), cudaMemcpyHostToDevice, s), "upload guide");
    k_guide_pack<<<(kGBf16 + 255) / 256, 256, 0, s>>>(c->g_params.as<float>(), c->g_wbf.as<uint16_t>(),
                                                      c->g_bias.as<float>(), c->g_misc.as<uint32_t>(), 0, 0);
    LUC_CUDA(c, cudaGetLastError(), "pack guide");
    LUC_CUDA(c, cudaStreamSynchronize(s), "guide init");
    c->guide_ready = true;
    return LUC_OK;
}

int32_t luc_guide_configure(luc_ctx* c, uint32_t train, uint32_t records_per_step, float lr) {
    if (!c) return LUC_ERR_VALIDATION;
    if (records_per_step == 0 || records_per_step > (1u << 24))
        return luc_fail(c, LUC_ERR_VALIDATION, "records_per_step must be in 1..=2^24");
    if (!(lr > 0.0f) || !std::isfinite(lr)) return luc_fail(c, LUC_ERR_VALIDATION, "lr must be positive and finite");
    if (int32_t rc = luc_guide_flush(c)) return rc;  // with the settings it was recorded under
    c->guide_train = train != 0;
    c->guide_rec_cap = records_per_step;
    c->guide_lr = lr;
    return LUC_OK;
}

int32_t luc_guide_get_params(luc_ctx* c, float* out) {
    if (!c || !out) return LUC_ERR_VALIDATION;
    if (int32_t rc = require_guide(c)) return rc;
    if (int32_t rc = luc_guide_flush(c)) return rc;
    cudaSetDevice(c->device);
    LUC_CUDA(c, cudaMemcpyAsync(out, c->g_params.p, kGParams * sizeof(float), cudaMemcpyDeviceToHost, c->stream),
             "read guide");
    LUC_CUDA(c, cudaStreamSynchronize(c->stream), "read guide");
    return LUC_OK;
}

int32_t luc_guide_stats(luc_ctx* c, luc_guide_info* out) {
    if (!c || !out) return LUC_ERR_VALIDATION;
    if (int32_t rc = require_guide(c)) return rc;
    if (int32_t rc = luc_guide_flush(c)) return rc;
    cudaSetDevice(c->device);
    uint32_t misc[kGmWords];
    LUC_CUDA(c, cudaMemcpyAsync(misc, c->g_misc.p, sizeof(misc), cudaMemcpyDeviceToHost, c->stream), "read guide");
    LUC_CUDA(c, cudaStreamSynchronize(c->stream), "read guide");
    out->steps = misc[kGmStep];
    out->last_records = misc[kGmLastRecords];
    std::memcpy(&out->last_loss, &misc[kGmLastLoss], 4);
    out->threshold = misc[kGmThreshold];
    out->num_params = kGParams;
    out->tc_error = misc[kGmTcError];
    return LUC_OK;
}

int32_t luc_guide_forward_ex(luc_ctx* c, const float* in9, uint32_t n, int32_t path, float* out40) {
    if (!c || (n && (!in9 || !out40))) return LUC_ERR_VALIDATION;
    if (path != 0 && path != 1) return luc_fail(c, LUC_ERR_VALIDATION, "path: 0 tcgen05, 1 mma.sync");
    if (int32_t rc = require_guide(c)) return rc;
    if (int32_t rc = luc_guide_flush(c)) return rc;
    if (n == 0) return LUC_OK;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    LUC_CUDA(c, c->g_io.ensure((size_t)n * (9 + kGOut) * sizeof(float)), "allocate guide io");
    float* din = c->g_io.as<float>();
    float* dout = din + (size_t)n * 9;
    LUC_CUDA(c, cudaMemcpyAsync(din, in9, (size_t)n * 9 * sizeof(float), cudaMemcpyHostToDevice, s), "upload");
    uint32_t* err = c->g_misc.as<uint32_t>() + kGmTcError;
    if (path == 0) {
        GuideDev g = luc_guide_dev(c);
        if (c->dbg_mode == LUC_DEBUG_TC_NO_COMMIT) {  // test hook: a wait that runs out
            g.tc_no_issue = 1;
            g.tc_wait_limit = c->dbg_limit;
            c->dbg_mode = 0;
        }
        LUC_CUDA(c, cudaMemsetAsync(err, 0, 4, s), "clear error word");
        LUC_CUDA(c, launch_guide_forward_tc(din, n, g, dout, err, c->num_sms, s), "guide forward");
    } else {
        int grid = (int)std::min<uint64_t>((n + 16 * kInferWarps - 1) / (16 * kInferWarps), (uint64_t)c->num_sms * 2);
        k_guide_forward<<<grid, kInferWarps * 32, sizeof(InferSmem), s>>>(din, n, luc_guide_dev(c), dout);
        LUC_CUDA(c, cudaGetLastError(), "guide forward");
    }
    uint32_t h_err = 0;
    LUC_CUDA(c, cudaMemcpyAsync(out40, dout, (size_t)n * kGOut * sizeof(float), cudaMemcpyDeviceToHost, s), "readback");
    LUC_CUDA(c, cudaMemcpyAsync(&h_err, err, 4, cudaMemcpyDeviceToHost, s), "read error word");
    LUC_CUDA(c, cudaStreamSynchronize(s), "guide forward");
    if (path == 0 && h_err) return luc_fail(c, LUC_ERR_LAUNCH, "guide forward: a tensor-core wait ran out");
    return LUC_OK;
}

int32_t luc_guide_forward(luc_ctx* c, const float* in9, uint32_t n, float* out40) {
    return luc_guide_forward_ex(c, in9, n, 0, out40);
}

int32_t luc_guide_train_records(luc_ctx* c, const float* records, uint32_t n, uint32_t steps, float* grad_out,
                                float* loss_out) {
    if (!c || (n && !records)) return LUC_ERR_VALIDATION;
    if (int32_t rc = require_guide(c)) return rc;
    if (int32_t rc = luc_guide_flush(c)) return rc;
    if (n == 0) return luc_fail(c, LUC_ERR_VALIDATION, "no records");
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    LUC_CUDA(c, c->g_io.ensure((size_t)n * kGRecF4 * sizeof(float4)), "allocate guide io");
    float4* rec = c->g_io.as<float4>();
    LUC_CUDA(c, cudaMemcpyAsync(rec, records, (size_t)n * kGRecF4 * sizeof(float4), cudaMemcpyHostToDevice, s),
             "upload records");
    uint32_t* gm = c->g_misc.as<uint32_t>();
    const uint32_t rounds = steps == 0 ? 1 : steps;
    LUC_CUDA(c, c->g_part.ensure(guide_part_bytes(c->num_sms)), "allocate guide gradient slices");
    const uint32_t count = n;
    for (uint32_t it = 0; it < rounds; ++it) {
        LUC_CUDA(c, cudaMemcpyAsync(gm + kGmRecords, &count, sizeof(count), cudaMemcpyHostToDevice, s), "upload count");
        LUC_CUDA(c, cudaMemsetAsync(gm + kGmWeightSum, 0, 2 * sizeof(uint32_t), s), "clear sums");
        k_guide_weight_sum<<<c->num_sms * 2, 256, 0, s>>>(rec, n, gm);
        launch_guide_gradient(rec, n, gm, luc_guide_dev(c), c->g_grad.as<float>(), c->g_part.as<float>(),
                              c->num_sms, c->rs.guide_tc, s);
        if (steps > 0) {
            k_guide_adam<<<(kGParams + 255) / 256, 256, 0, s>>>(c->g_params.as<float>(), c->g_m.as<float>(),
                                                                c->g_v.as<float>(), c->g_grad.as<float>(), gm,
                                                                c->guide_lr);
            k_guide_pack<<<(kGBf16 + 255) / 256, 256, 0, s>>>(c->g_params.as<float>(), c->g_wbf.as<uint16_t>(),
                                                              c->g_bias.as<float>(), gm, n, 1u);
        }
        LUC_CUDA(c, cudaGetLastError(), "guide train");
    }
    uint32_t misc[kGmWords];
    LUC_CUDA(c, cudaMemcpyAsync(misc, gm, sizeof(misc), cudaMemcpyDeviceToHost, s), "read guide");
    if (grad_out)
        LUC_CUDA(c, cudaMemcpyAsync(grad_out, c->g_grad.p, kGParams * sizeof(float), cudaMemcpyDeviceToHost, s),
                 "read gradient");
    LUC_CUDA(c, cudaStreamSynchronize(s), "guide train");
    if (loss_out) std::memcpy(loss_out, &misc[steps > 0 ? kGmLastLoss : kGmLoss], 4);
    return LUC_OK;
}

int32_t luc_guide_mixture(luc_ctx* c, const float* raw40, const float* in3, uint32_t n, int32_t mode, float* dir3,
                          float* pdf) {
    if (!c || (n && (!raw40 || !in3 || !pdf || (mode == 0 && !dir3)))) return LUC_ERR_VALIDATION;
    if (mode != 0 && mode != 1) return luc_fail(c, LUC_ERR_VALIDATION, "mode must be 0 (sample) or 1 (pdf)");
    if (n == 0) return LUC_OK;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    LUC_CUDA(c, c->g_io.ensure((size_t)n * (kGOut + 3 + 3 + 1) * sizeof(float)), "allocate guide io");
    float* draw = c->g_io.as<float>();
    float* din = draw + (size_t)n * kGOut;
    float* ddir = din + (size_t)n * 3;
    float* dpdf = ddir + (size_t)n * 3;
    LUC_CUDA(c, cudaMemcpyAsync(draw, raw40, (size_t)n * kGOut * 4, cudaMemcpyHostToDevice, s), "upload");
    LUC_CUDA(c, cudaMemcpyAsync(din, in3, (size_t)n * 3 * 4, cudaMemcpyHostToDevice, s), "upload");
    k_guide_mixture_eval<<<(n + 255) / 256, 256, 0, s>>>(draw, din, n, mode, ddir, dpdf);
    LUC_CUDA(c, cudaGetLastError(), "guide mixture");
    if (mode == 0) LUC_CUDA(c, cudaMemcpyAsync(dir3, ddir, (size_t)n * 3 * 4, cudaMemcpyDeviceToHost, s), "readback");
    LUC_CUDA(c, cudaMemcpyAsync(pdf, dpdf, (size_t)n * 4, cudaMemcpyDeviceToHost, s), "readback");
    LUC_CUDA(c, cudaStreamSynchronize(s), "guide mixture");
    return LUC_OK;
}

}  // extern "C"
