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
constexpr int kGLobeF4 = 10;  // per path: 8 x (mu, kappa) + 2 x 4 weights

struct GuideDev {
    const uint16_t* wbf;   // packed bf16 weights
    const float* bias;     // packed fp32 biases
    float lo[3], inv_ext[3];  // scene box for the position encoding
};

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

// kappa / (2 pi (1 - e^{-2 kappa})) e^{kappa (c - 1)}
LUC_D float vmf_pdf(float kappa, float c) {
    float norm = kappa / (2.0f * kPi * (1.0f - expf(-2.0f * kappa)));
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

// Pick a lobe with u0, then sample it (Wood 1994 inversion in the lobe frame).
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
    float4 l = m.lobe[j];
    float kappa = l.w;
    float W = 1.0f + logf(u1 + (1.0f - u1) * expf(-2.0f * kappa)) / kappa;
    W = fminf(fmaxf(W, -1.0f), 1.0f);
    float s = sqrtf(fmaxf(1.0f - W * W, 0.0f));
    float sp, cp;
    __sincosf(2.0f * kPi * u2, &sp, &cp);
    V3 local{s * cp, s * sp, W};
    return normalize(to_world(local, V3{l.x, l.y, l.z}));
}

}  // namespace luc
