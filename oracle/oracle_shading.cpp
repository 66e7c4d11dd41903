// ORACLE — test infrastructure only (see oracle_core.hpp). Restates
// crates/core/src/{bsdf,light,envmap}.rs.
#include "oracle_core.hpp"
#include <mutex>

namespace oracle {

const SobolTable& sobol_table() {
    static const SobolTable t;
    return t;
}

// bsdf.rs:760-777 — midpoint-rule quadrature over the VNDF parameter square.
float specular_directional_albedo_grid(float alpha, float cos_theta_o, uint32_t grid) {
    float sin_theta = std::sqrt(fmax_(1.0f - cos_theta_o * cos_theta_o, 0.0f));
    Vec3 wo(sin_theta, 0.0f, cos_theta_o);
    double sum = 0.0;
    float n = (float)grid;
    for (uint32_t i = 0; i < grid; ++i) {
        for (uint32_t j = 0; j < grid; ++j) {
            Vec2 u(((float)i + 0.5f) / n, ((float)j + 0.5f) / n);
            BsdfSample s = specular_sample_single(alpha, Vec3::splat(1.0f), wo, u);
            if (s.valid()) sum += (double)s.weight.x;
        }
    }
    return (float)(sum / ((double)grid * (double)grid));
}

// bsdf.rs:1210-1225
std::vector<float> compute_energy_table() {
    const int n = ENERGY_TABLE_SIZE;
    std::vector<float> t(n * n);
    for (int ri = 0; ri < n; ++ri) {
        float roughness = (float)ri / (float)(n - 1);
        float alpha = roughness_to_alpha(roughness);
        for (int ci = 0; ci < n; ++ci) {
            float root_mu = (float)ci / (float)(n - 1);
            float mu = fmax_(root_mu * root_mu, 1.0e-4f);
            t[ri * n + ci] = specular_directional_albedo_grid(alpha, mu, 128);
        }
    }
    return t;
}

const float* energy_table() {
    static std::once_flag once;
    static std::vector<float> table;
    std::call_once(once, [] { table = compute_energy_table(); });
    return table.data();
}

// surface::eval (bsdf.rs:1493-1540)
Vec3 surface_eval(const Surface& s, Vec3 wo, Vec3 wi) {
    if (wo.z <= 0.0f) return Vec3();
    float alpha = roughness_to_alpha(s.roughness);
    if (wi.z < 0.0f) {
        if (s.transmission <= 0.0f) return Vec3();
        float t = dielectric_eval(alpha, s.relative_ior, wo, wi);
        return Vec3::splat(t) * s.transmission * s.transmission_tint;
    }
    if (wi.z <= 0.0f) return Vec3();
    Vec3 transmitted = Vec3::splat(1.0f) - s.specular_albedo(wo.z);
    // diffuse::eval (bsdf.rs:425-430)
    Vec3 diff = wi.z <= 0.0f ? Vec3() : s.diffuse_albedo * INV_PI;
    Vec3 f = diff * transmitted * (1.0f - s.transmission);
    Vec3 h = (wo + wi).normalize_or_zero();
    if (h != Vec3()) {
        float d = ggx_d(alpha, h.z);
        float g2 = smith_g2(alpha, wo.z, wi.z);
        Vec3 fr = s.reflection_fresnel(fmax_(wo.dot(h), 0.0f));
        Vec3 single = fr * (d * g2 / (4.0f * wo.z * wi.z));
        f += s.transmission > 0.0f ? single
                                   : single * compensation(s.roughness, wo.z, s.normal_reflectance());
    }
    return f;
}

// surface::pdf (bsdf.rs:1543-1562)
float surface_pdf(const Surface& s, Vec3 wo, Vec3 wi) {
    if (wo.z <= 0.0f) return 0.0f;
    float p_spec = s.specular_probability(wo.z);
    float alpha = roughness_to_alpha(s.roughness);
    float rest = 1.0f - p_spec;
    if (wi.z < 0.0f) {
        if (s.transmission <= 0.0f) return 0.0f;
        return rest * s.transmission * dielectric_pdf(alpha, s.relative_ior, wo, wi);
    }
    if (wi.z <= 0.0f) return 0.0f;
    // specular::pdf (bsdf.rs:476-485)
    float spec = 0.0f;
    {
        Vec3 h = (wo + wi).normalize_or_zero();
        if (wo.z > 0.0f && wi.z > 0.0f && h != Vec3()) spec = ggx_vndf_pdf(alpha, wo, h);
    }
    float diff = wi.z <= 0.0f ? 0.0f : wi.z * INV_PI;  // diffuse::pdf
    return p_spec * spec + rest * (1.0f - s.transmission) * diff;
}

// surface::sample (bsdf.rs:1571-1661)
BsdfSample surface_sample(const Surface& s, Vec3 wo, float u_lobe, Vec2 u) {
    if (wo.z <= 0.0f) return BsdfSample::invalid();
    float p_spec = s.specular_probability(wo.z);
    float alpha = roughness_to_alpha(s.roughness);
    Vec3 wi;
    if (u_lobe < p_spec) {
        sig_event(3, 0);
        Vec3 m = sample_ggx_vndf(wo, alpha, u);
        Vec3 r = reflect(wo, m);
        if (r.z <= 0.0f) return sig_event(4, 1), BsdfSample::invalid();
        wi = r;
    } else if (u_lobe < p_spec + (1.0f - p_spec) * s.transmission) {
        sig_event(3, 1);
        Vec3 m = sample_ggx_vndf(wo, alpha, u);
        Vec3 wt;
        if (!refract(wo, m, s.relative_ior, wt)) return sig_event(4, 2), BsdfSample::invalid();
        if (wt.z >= 0.0f) return sig_event(4, 3), BsdfSample::invalid();
        wi = wt;
    } else {
        sig_event(3, 2);
        wi = sample_cosine_hemisphere(u);
    }
    if (wi.z == 0.0f || wi == Vec3()) return sig_event(4, 4), BsdfSample::invalid();
    if (wi.z < 0.0f && s.transmission <= 0.0f) return sig_event(4, 5), BsdfSample::invalid();
    Vec3 f = surface_eval(s, wo, wi);
    float pdf = surface_pdf(s, wo, wi);
    if (pdf <= 0.0f) return sig_event(4, 6), BsdfSample::invalid();
    return BsdfSample{wi, f * (std::fabs(wi.z) / pdf), pdf};
}

// light.rs:62-123
std::vector<GpuLight> build_lights(const std::vector<GpuMaterial>& mats,
                                   const std::vector<GpuPrimitive>& prims,
                                   const std::vector<GpuTriangle>& tris,
                                   const std::vector<float>& pos) {
    std::vector<GpuLight> lights;
    auto emits = [&](uint32_t m) {
        const float* e = mats[m].emissive;
        return e[0] > 0.0f || e[1] > 0.0f || e[2] > 0.0f;
    };
    for (const GpuPrimitive& p : prims) {
        if (p.kind != PRIM_KIND_QUAD || !emits(p.material)) continue;
        Vec3 eu = Vec3::from(p.edge_u), ev = Vec3::from(p.edge_v);
        Vec3 cr = eu.cross(ev);
        GpuLight l;
        std::memset(&l, 0, sizeof(l));
        std::memcpy(l.origin, p.position, 12);
        l.area = cr.length();
        std::memcpy(l.edge_u, p.edge_u, 12);
        l.kind = LIGHT_KIND_QUAD;
        std::memcpy(l.edge_v, p.edge_v, 12);
        l.material = p.material;
        std::memcpy(l.normal, p.normal, 12);
        lights.push_back(l);
    }
    for (const GpuTriangle& t : tris) {
        if (!emits(t.material)) continue;
        auto P = [&](uint32_t i) { return Vec3(pos[4 * i], pos[4 * i + 1], pos[4 * i + 2]); };
        Vec3 p0 = P(t.i0), p1 = P(t.i1), p2 = P(t.i2);
        Vec3 e1 = p1 - p0, e2 = p2 - p0;
        Vec3 cr = e1.cross(e2);
        float len = cr.length();
        if (len <= 0.0f) continue;
        GpuLight l;
        std::memset(&l, 0, sizeof(l));
        p0.to(l.origin);
        l.area = 0.5f * len;
        e1.to(l.edge_u);
        l.kind = LIGHT_KIND_TRIANGLE;
        e2.to(l.edge_v);
        l.material = t.material;
        (cr / len).to(l.normal);
        lights.push_back(l);
    }
    return lights;
}

// ---------------------------------------------------------------- envmap.rs
Vec3 EnvMap::direction_from_uv(float u, float v) {  // envmap.rs:93-99
    float theta = v * PI;
    float phi = u * TAU;
    float st = m_sin(theta), ct = m_cos(theta);
    return Vec3(st * m_cos(phi), ct, st * m_sin(phi));
}
Vec2 EnvMap::uv_from_direction(Vec3 d) {  // :103-111
    float theta = m_acos(clampf(d.y, -1.0f, 1.0f));
    float a = m_atan2(d.z, d.x);
    float r = std::fmod(a, TAU);  // rem_euclid
    float phi = r < 0.0f ? r + std::fabs(TAU) : r;
    return Vec2(phi / TAU, theta / PI);
}
EnvMap EnvMap::build(uint32_t width, uint32_t height, std::vector<float> px) {  // :114-178
    EnvMap e;
    e.width = width;
    e.height = height;
    size_t w = width, h = height;
    e.conditional.assign((w + 1) * h, 0.0f);
    e.marginal.assign(h + 1, 0.0f);
    std::vector<float> row_weight(h, 0.0f);
    for (size_t j = 0; j < h; ++j) {
        float theta = ((float)j + 0.5f) / (float)h * PI;
        float sin_theta = std::sin(theta);
        size_t base = j * (w + 1);
        float running = 0.0f;
        for (size_t i = 0; i < w; ++i) {
            const float* p = &px[4 * (j * w + i)];
            float weight = fmax_(luminance(Vec3(p[0], p[1], p[2])), 0.0f) * sin_theta;
            running += weight;
            e.conditional[base + i + 1] = running;
        }
        row_weight[j] = running;
        if (running > 0.0f) {
            float inv = 1.0f / running;
            for (size_t k = 1; k <= w; ++k) e.conditional[base + k] *= inv;
            e.conditional[base + w] = 1.0f;
        }
    }
    float running = 0.0f;
    for (size_t j = 0; j < h; ++j) {
        running += row_weight[j];
        e.marginal[j + 1] = running;
    }
    e.total_weight = running;
    if (running > 0.0f) {
        float inv = 1.0f / running;
        for (size_t k = 1; k <= h; ++k) e.marginal[k] *= inv;
        e.marginal[h] = 1.0f;
    }
    e.pixels = std::move(px);
    return e;
}
void EnvMap::texel_of(Vec2 uv, uint64_t& i, uint64_t& j) const {  // :199-203
    int64_t ii = f2i64(uv.x * (float)width);
    int64_t jj = f2i64(uv.y * (float)height);
    ii = std::min<int64_t>(std::max<int64_t>(ii, 0), (int64_t)width - 1);
    jj = std::min<int64_t>(std::max<int64_t>(jj, 0), (int64_t)height - 1);
    i = (uint64_t)ii;
    j = (uint64_t)jj;
}
Vec3 EnvMap::radiance(Vec3 d) const {  // :188-196
    if (pixels.empty()) return Vec3();
    Vec2 uv = uv_from_direction(d);
    uint64_t i, j;
    texel_of(uv, i, j);
    const float* p = &pixels[4 * (j * width + i)];
    return Vec3(p[0], p[1], p[2]);
}
float EnvMap::pdf(Vec3 d) const {  // :211-232
    if (is_empty()) return 0.0f;
    Vec2 uv = uv_from_direction(d);
    uint64_t i, j;
    texel_of(uv, i, j);
    float theta = ((float)j + 0.5f) / (float)height * PI;
    float st = std::sin(theta);
    if (st <= 0.0f) return 0.0f;
    const float* p = &pixels[4 * (j * width + i)];
    float weight = fmax_(luminance(Vec3(p[0], p[1], p[2])), 0.0f) * st;
    float pdf_uv = weight / total_weight * (float)((uint64_t)width * height);
    return pdf_uv / (2.0f * PI * PI * st);
}
// envmap.rs:290-317
static void sample_cdf(const std::vector<float>& cdf, size_t base, size_t n, float x,
                       size_t& cell, float& frac) {
    size_t lo = 0, len = n;
    while (len > 0) {
        size_t half = len / 2;
        size_t mid = lo + half;
        if (cdf[base + mid] <= x) {
            lo = mid + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    cell = std::min<size_t>(lo == 0 ? 0 : lo - 1, n - 1);
    float c0 = cdf[base + cell], c1 = cdf[base + cell + 1];
    float span = c1 - c0;
    frac = span > 0.0f ? clampf((x - c0) / span, 0.0f, 1.0f) : 0.0f;
}
EnvSample EnvMap::sample(Vec2 u) const {  // :235-275
    EnvSample invalid{Vec3(0, 1, 0), Vec3(), 0.0f};
    if (is_empty()) return invalid;
    size_t w = width, h = height;
    size_t j, i;
    float dv, du;
    sample_cdf(marginal, 0, h, u.y, j, dv);
    sample_cdf(conditional, j * (w + 1), w, u.x, i, du);
    Vec2 uv(((float)i + du) / (float)w, ((float)j + dv) / (float)h);
    Vec3 direction = direction_from_uv(uv.x, uv.y);
    float theta = ((float)j + 0.5f) / (float)h * PI;
    float st = std::sin(theta);
    if (st <= 0.0f) return invalid;
    const float* p = &pixels[4 * (j * w + i)];
    Vec3 rad(p[0], p[1], p[2]);
    float weight = fmax_(luminance(rad), 0.0f) * st;
    float pdf_uv = weight / total_weight * (float)(w * h);
    float pdf = pdf_uv / (2.0f * PI * PI * st);
    if (pdf <= 0.0f) return invalid;
    return EnvSample{direction, rad, pdf};
}

// envmap.rs:343-408
EnvMap procedural_sky(uint32_t width, uint32_t height, Vec3 sun_direction, float sun_intensity,
                      float sun_radius_degrees) {
    Vec3 sun = sun_direction.normalize_or(Vec3(0, 1, 0));
    float texel = fmax_(PI / (float)height, TAU / (float)width);
    float requested = sun_radius_degrees * (PI / 180.0f);
    float radius = fmax_(requested, texel);
    float area_ratio = (1.0f - std::cos(requested)) / fmax_(1.0f - std::cos(radius), 1e-20f);
    float intensity = sun_intensity * fmin_(area_ratio, 1.0f);
    float cos_sun_radius = std::cos(radius);
    std::vector<float> px;
    px.reserve((size_t)width * height * 4);
    for (uint32_t j = 0; j < height; ++j) {
        float v = ((float)j + 0.5f) / (float)height;
        for (uint32_t i = 0; i < width; ++i) {
            float u = ((float)i + 0.5f) / (float)width;
            Vec3 d = EnvMap::direction_from_uv(u, v);
            Vec3 c;
            if (d.y >= 0.0f) {
                float t = std::pow(d.y, 0.45f);
                c = Vec3(0.75f, 0.86f, 1.00f) * t + Vec3(0.85f, 0.70f, 0.55f) * (1.0f - t);
            } else {
                c = Vec3::splat(0.12f);
            }
            c *= 0.40f;
            if (d.dot(sun) >= cos_sun_radius) c += Vec3(1.0f, 0.92f, 0.78f) * intensity;
            px.push_back(c.x);
            px.push_back(c.y);
            px.push_back(c.z);
            px.push_back(0.0f);
        }
    }
    return EnvMap::build(width, height, std::move(px));
}

}  // namespace oracle
