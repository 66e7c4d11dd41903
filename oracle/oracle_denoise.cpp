// ORACLE — test infrastructure only (see oracle_core.hpp). Restates the
// edge-avoiding à-trous filter of crates/core/src/denoise.rs:101-228.
#include "oracle_scene.hpp"

namespace oracle {

static const float KERNEL[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};

// denoise.rs:111-128
static float local_deviation(const std::vector<Vec3>& data, uint32_t width, uint32_t height, uint32_t x,
                             uint32_t y) {
    int32_t w = (int32_t)width, h = (int32_t)height;
    float sum = 0.0f, sum_sq = 0.0f, n = 0.0f;
    for (int32_t dy = -1; dy <= 1; ++dy) {
        for (int32_t dx = -1; dx <= 1; ++dx) {
            int32_t px = (int32_t)x + dx, py = (int32_t)y + dy;
            if (px < 0 || py < 0 || px >= w || py >= h) continue;
            float l = luminance(data[(size_t)(py * w + px)]);
            sum += l;
            sum_sq += l * l;
            n += 1.0f;
        }
    }
    float mean = sum / n;
    return std::sqrt(fmax_(sum_sq / n - mean * mean, 0.0f));
}

// denoise.rs:134-228
void denoise(const std::vector<Vec3>& film, const std::vector<Vec3>& albedo, const std::vector<Vec3>& normal,
             const std::vector<float>& depth, uint32_t width, uint32_t height, const DenoiseParams& p,
             std::vector<Vec3>& out) {
    int32_t w = (int32_t)width, h = (int32_t)height;
    size_t n = (size_t)w * (size_t)h;
    if (n == 0 || albedo.size() != n) {
        out = film;
        return;
    }
    std::vector<Vec3> cur(n), nxt;
    for (size_t i = 0; i < n; ++i) cur[i] = film[i] / albedo[i].max(Vec3::splat(1.0e-3f));
    nxt = cur;
    std::vector<float> dev(n);
    for (size_t i = 0; i < n; ++i) dev[i] = local_deviation(cur, width, height, (uint32_t)(i % width), (uint32_t)(i / width));
    for (uint32_t level = 0; level < p.iterations; ++level) {
        int32_t stride = 1 << level;
        for (int32_t y = 0; y < h; ++y) {
            for (int32_t x = 0; x < w; ++x) {
                size_t ci = (size_t)(y * w + x);
                Vec3 cn = normal[ci];
                float cd = depth[ci];
                float cl = luminance(cur[ci]);
                float ca = fmax_(luminance(albedo[ci]), 1.0e-3f);
                float lum_scale = p.sigma_luminance * fmax_(dev[ci], 1.0e-4f);
                Vec3 sum;
                float wsum = 0.0f;
                for (int32_t ky = 0; ky < 5; ++ky) {
                    for (int32_t kx = 0; kx < 5; ++kx) {
                        int32_t px = x + (kx - 2) * stride, py = y + (ky - 2) * stride;
                        if (px < 0 || py < 0 || px >= w || py >= h) continue;
                        size_t qi = (size_t)(py * w + px);
                        float nd = fmax_(cn.dot(normal[qi]), 0.0f);
                        float w_n = std::pow(nd, p.sigma_normal);
                        float dd = std::fabs(cd - depth[qi]);
                        float w_d = std::exp(-dd / (p.sigma_depth * fmax_(std::fabs(cd), 1.0e-3f)));
                        float dl = std::fabs(cl - luminance(cur[qi]));
                        float w_l = std::exp(-dl / lum_scale);
                        float da = std::fabs(ca - luminance(albedo[qi]));
                        float w_a = std::exp(-da / (p.sigma_albedo * ca));
                        float weight = KERNEL[kx] * KERNEL[ky] * w_n * w_d * w_l * w_a;
                        sum += cur[qi] * weight;
                        wsum += weight;
                    }
                }
                nxt[ci] = wsum > 0.0f ? sum / wsum : cur[ci];
            }
        }
        std::swap(cur, nxt);
    }
    out.resize(n);
    for (size_t i = 0; i < n; ++i) out[i] = cur[i] * albedo[i].max(Vec3::splat(1.0e-3f));
}

}  // namespace oracle
