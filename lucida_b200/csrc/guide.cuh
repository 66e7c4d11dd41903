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

// Per-CTA weight-gradient slice of the training kernels (mma.sync and
// tcgen05 alike): dW1 | dW2 | dW3 | dW4 (kGOutPad rows), each [out][in].
constexpr int kPartW1 = 0, kPartW2 = kGHid * kGIn, kPartW3 = kPartW2 + kGHid * kGHid,
              kPartW4 = kPartW3 + kGHid * kGHid, kPartFloats = kPartW4 + kGOutPad * kGHid;

// Polls of a tensor-core kernel's mbarrier before its wait gives up.
constexpr uint32_t kTcWaitLimit = 1u << 22;

struct GuideDev {
    const uint16_t* wbf;   // packed bf16 weights
    const float* bias;     // packed fp32 biases
    float lo[3], ext[3];  // scene box for the position encoding (ext = hi - lo, or 1)
    uint32_t tc_wait_limit;  // kTcWaitLimit (a test hook lowers it)
    uint32_t tc_no_issue;    // test hook: issue no MMA and no commit, so the wait runs out
};

LUC_D float softplus_f(float x) { return x > 20.0f ? x : log1pf(expf(x)); }

// Loss term of one row, -F/S log q(d), and its gradient w.r.t. the raw
// outputs (the same closed forms as the oracle).
LUC_D float row_loss_grad(const float* __restrict__ o, V3 d, float F, float invS, float* __restrict__ go) {
    float mx = -INFINITY;
    for (int j = 0; j < kGLobes; ++j) mx = fmaxf(mx, o[5 * j + 4]);
    float w[kGLobes], pj[kGLobes];
    float ws = 0.f;
    for (int j = 0; j < kGLobes; ++j) {
        w[j] = expf(o[5 * j + 4] - mx);
        ws += w[j];
    }
    float q = 0.f;
    for (int j = 0; j < kGLobes; ++j) {
        w[j] /= ws;
        float x = o[5 * j], y = o[5 * j + 1], z = o[5 * j + 2];
        float ln = fmaxf(sqrtf(x * x + y * y + z * z), 1e-30f);
        float c = (x * d.x + y * d.y + z * d.z) / ln;
        float kap = fminf(1.0f + softplus_f(o[5 * j + 3]), kGKappaMax);
        pj[j] = kap / (2.0f * kPi * (1.0f - expf(-2.0f * kap))) * expf(kap * (c - 1.0f));
        q += w[j] * pj[j];
    }
    q = fmaxf(q, 1e-30f);
    const float scale = -F * invS;
    for (int j = 0; j < kGLobes; ++j) {
        float x = o[5 * j], y = o[5 * j + 1], z = o[5 * j + 2];
        float ln = fmaxf(sqrtf(x * x + y * y + z * z), 1e-30f);
        float mu[3] = {x / ln, y / ln, z / ln};
        float c = mu[0] * d.x + mu[1] * d.y + mu[2] * d.z;
        float kr = 1.0f + softplus_f(o[5 * j + 3]);
        float kap = fminf(kr, kGKappaMax);
        float ex = expf(-2.0f * kap);
        float r = w[j] * pj[j] / q;
        go[5 * j + 4] = scale * (r - w[j]);
        float dk = r * (1.0f / kap - 2.0f * ex / (1.0f - ex) + c - 1.0f);
        float sig = 1.0f / (1.0f + expf(-fminf(fmaxf(o[5 * j + 3], -60.f), 60.f)));
        go[5 * j + 3] = kr >= kGKappaMax ? 0.0f : scale * dk * sig;
        float gm[3] = {r * kap * d.x, r * kap * d.y, r * kap * d.z};
        float dotm = gm[0] * mu[0] + gm[1] * mu[1] + gm[2] * mu[2];
        for (int a = 0; a < 3; ++a) go[5 * j + a] = scale * (gm[a] - dotm * mu[a]) / ln;
    }
    return scale * logf(q);
}

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
