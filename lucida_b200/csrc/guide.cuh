// Learned path-guiding proposal: shared definitions (network shape, device
// state, vMF-mixture sampling and density used by SHADE).
//
// The proposal is a small MLP — frequency-encoded position (12 frequencies
// per axis, normalised to the scene box), shading normal and outgoing
// direction (4 each); 120 features padded to 128 -> 64 -> 64 -> 64 -> 40 with
// ReLU — whose 40 outputs are 8 von Mises-Fisher lobes: direction
// normalize(o[0:3]), concentration min(1 + softplus(o[3]), 1e4), weight
// softmax(o[4]). Weights are BF16 in the matrix multiplies with FP32
// accumulation; the master copy, gradients and Adam moments are FP32.
#pragma once
#include <cstdint>
#include "device_math.cuh"

namespace luc {

constexpr int kGIn = 128, kGHid = 64, kGOut = 40, kGOutPad = 48, kGLobes = 8;
constexpr int kGFeatures = 120;
constexpr int kGParams = kGHid * kGIn + kGHid + kGHid * kGHid + kGHid + kGHid * kGHid + kGHid + kGOut * kGHid + kGOut;
constexpr int kGBf16 = kGHid * kGIn + 2 * kGHid * kGHid + kGOutPad * kGHid;  // packed W1..W4 (row = output)
constexpr int kGBias = 3 * kGHid + kGOutPad;
constexpr float kGKappaMax = 1.0e4f;
constexpr int kGLobeF4 = 10;  // per queued path: 8 x (mu, kappa) + 2 x 4 weights
constexpr int kGRecF4 = 5;    // per training record, see below
// Vertices are guided when opaque and not near-specular; sharper lobes and
// transmission stay BSDF-sampled.
constexpr float kGuideMinRoughness = 0.2f;

// Device bookkeeping words (u32, floats stored as bits).
constexpr int kGmRecords = 0;     // records appended this batch
constexpr int kGmStep = 1;        // Adam steps taken
constexpr int kGmWeightSum = 2;   // sum of F over the batch's records (f32)
constexpr int kGmLoss = 3;        // loss accumulated by the training kernel (f32)
constexpr int kGmCandidates = 4;  // guided, surviving vertices this batch
constexpr int kGmThreshold = 5;   // recording threshold, 16-bit fraction
constexpr int kGmLastLoss = 6;    // loss of the last step (f32)
constexpr int kGmLastRecords = 7; // records used by the last step
constexpr int kGmTcError = 8;     // a tensor-core kernel's bounded wait ran out (nonzero)
constexpr int kGmWords = 16;

// Training record, 5 float4 per guided vertex:
//   [0] position, F (written by the finalize kernel; path id bits before)
//   [1] shading normal, throughput after scattering .x
//   [2] outgoing direction (world), throughput .y
//   [3] sampled direction (world), throughput .z
//   [4] path radiance when the continuation started, mixture pdf p(wi)

// Polls of a tensor-core kernel's mbarrier before its wait gives up.
constexpr uint32_t kTcWaitLimit = 1u << 22;

struct GuideDev {
    const uint16_t* wbf;   // packed bf16 weights
    const float* bias;     // packed fp32 biases
    float lo[3], ext[3];  // scene box for the position encoding (ext = hi - lo, or 1)
    uint32_t tc_wait_limit;  // kTcWaitLimit (a test hook lowers it)
    uint32_t tc_no_issue;    // test hook: issue no MMA and no commit, so the wait runs out
};

// 32-bit integer mix (Wellons' "lowbias32" constants) for record selection.
LUC_D uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Decoded mixture of one vertex, as stored for SHADE.
struct Mixture {
    float4 lobe[kGLobes];  // mu.xyz, kappa
    float w[kGLobes];
};

LUC_D void load_mixture(const float4* __restrict__ p, Mixture& m) {
#pragma unroll
    for (int j = 0; j < kGLobes; ++j) m.lobe[j] = p[j];
    float4 a = p[8], b = p[9];
    m.w[0] = a.x; m.w[1] = a.y; m.w[2] = a.z; m.w[3] = a.w;
    m.w[4] = b.x; m.w[5] = b.y; m.w[6] = b.z; m.w[7] = b.w;
}

// kappa / (2 pi (1 - e^{-2 kappa})) e^{kappa (c - 1)}. For kappa >= 9,
// 1 - e^{-2 kappa} rounds to 1 in f32, so the exponential is skipped.
LUC_D float vmf_pdf(float kappa, float c) {
    float e = kappa < 9.0f ? expf(-2.0f * kappa) : 0.0f;
    float norm = kappa / (2.0f * kPi * (1.0f - e));
    return norm * expf(kappa * (c - 1.0f));
}

LUC_D float mixture_pdf(const Mixture& m, V3 d) {
    float p = 0.0f;
#pragma unroll
    for (int j = 0; j < kGLobes; ++j) {
        float4 l = m.lobe[j];
        p += m.w[j] * vmf_pdf(l.w, l.x * d.x + l.y * d.y + l.z * d.z);
    }
    return p;
}

// Sample one vMF lobe (Wood 1994 inversion of the cosine's CDF, in the
// Duff et al. frame around the lobe direction).
LUC_D V3 vmf_sample(float4 l, float u1, float u2) {
    float kappa = l.w;
    float W = 1.0f + logf(u1 + (1.0f - u1) * expf(-2.0f * kappa)) / kappa;
    W = fminf(fmaxf(W, -1.0f), 1.0f);
    float s = sqrtf(fmaxf(1.0f - W * W, 0.0f));
    float sp, cp;
    sincosf(2.0f * kPi * u2, &sp, &cp);
    V3 local{s * cp, s * sp, W};
    return normalize(to_world(local, V3{l.x, l.y, l.z}));
}

// Pick a lobe with u0 by weight, then sample it with (u1, u2).
LUC_D V3 mixture_sample(const Mixture& m, float u0, float u1, float u2) {
    int j = kGLobes - 1;
    float acc = 0.0f;
#pragma unroll
    for (int k = 0; k < kGLobes; ++k) {
        acc += m.w[k];
        if (u0 < acc) {
            j = k;
            break;
        }
    }
    return vmf_sample(m.lobe[j], u1, u2);
}

// The same two operations on a stored mixture: SoA by queue position, lobe j
// (mu.xyz, kappa) at L[j * stride], the weights at L[8 * stride] (lobes
// 0..3) and L[9 * stride] (4..7), so a warp's loads coalesce and SHADE holds
// no mixture in registers.
LUC_D float mixture_pdf_mem(const float4* __restrict__ L, size_t stride, V3 d) {
    const float4 wa = L[8 * stride], wb = L[9 * stride];
    const float w[kGLobes] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
    float p = 0.0f;
#pragma unroll
    for (int j = 0; j < kGLobes; ++j) {
        float4 l = L[j * stride];
        p += w[j] * vmf_pdf(l.w, l.x * d.x + l.y * d.y + l.z * d.z);
    }
    return p;
}
LUC_D V3 mixture_sample_mem(const float4* __restrict__ L, size_t stride, float u0, float u1, float u2) {
    const float4 wa = L[8 * stride], wb = L[9 * stride];
    const float w[kGLobes] = {wa.x, wa.y, wa.z, wa.w, wb.x, wb.y, wb.z, wb.w};
    int j = kGLobes - 1;
    float acc = 0.0f;
#pragma unroll
    for (int k = 0; k < kGLobes; ++k) {
        acc += w[k];
        if (u0 < acc) {
            j = k;
            break;
        }
    }
    return vmf_sample(L[j * stride], u1, u2);
}

}  // namespace luc
