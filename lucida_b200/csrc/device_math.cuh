// Device math for the Lucida light-transport path on sm_100a.
//
// Numerical contract: this translation unit is compiled with --fmad=false,
// -prec-div=true and -prec-sqrt=true, so every f32 add/mul/div/sqrt is one
// IEEE-rounded operation, the way Rust evaluates the reference (which never
// contracts a*b+c). Vector operations keep glam 0.33's evaluation order:
// dot = ((x*x') + (y*y')) + (z*z'), cross = (y*z'-y'*z, z*x'-z'*x, x*y'-x'*y),
// normalize = v * (1/sqrt(dot)). Transcendentals are evaluated in double and
// rounded once to f32 (correctly rounded up to double rounding); the
// reference's glibc f32 functions round the last bit differently on a small
// fraction of inputs, which the parity tests measure.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/lucida_layout.h"

#define LUC_D __device__ __forceinline__
#define LUC_HD __host__ __device__ __forceinline__

namespace luc {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTau = 6.28318530717958647692f;
constexpr float kInvPi = 0.318309886183790671538f;

struct V3 {
    float x, y, z;
};
LUC_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
LUC_HD V3 splat(float s) { return V3{s, s, s}; }
LUC_HD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
LUC_HD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
LUC_HD V3 operator*(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
LUC_HD V3 operator/(V3 a, V3 b) { return V3{a.x / b.x, a.y / b.y, a.z / b.z}; }
LUC_HD V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
LUC_HD V3 operator*(float s, V3 a) { return V3{s * a.x, s * a.y, s * a.z}; }
LUC_HD V3 operator/(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
LUC_HD V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
LUC_HD bool operator==(V3 a, V3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
LUC_HD float dot(V3 a, V3 b) { return ((a.x * b.x) + (a.y * b.y)) + (a.z * b.z); }
LUC_HD V3 cross(V3 a, V3 b) {
    return V3{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
LUC_HD float fmax_(float a, float b) { return fmaxf(a, b); }
LUC_HD float fmin_(float a, float b) { return fminf(a, b); }
LUC_HD V3 vmin(V3 a, V3 b) { return V3{fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)}; }
LUC_HD V3 vmax(V3 a, V3 b) { return V3{fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
LUC_HD float max_elem(V3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
LUC_HD float min_elem(V3 a) { return fminf(a.x, fminf(a.y, a.z)); }
LUC_HD float length(V3 a) { return sqrtf(dot(a, a)); }
LUC_HD V3 normalize(V3 a) { return a * (1.0f / length(a)); }
LUC_HD V3 normalize_or(V3 a, V3 fb) {
    float r = 1.0f / length(a);
    return (isfinite(r) && r > 0.0f) ? a * r : fb;
}
LUC_HD float clampf(float x, float lo, float hi) {
    x = x < lo ? lo : x;
    return x > hi ? hi : x;
}
LUC_HD V3 vclamp01(V3 a) { return vmin(vmax(a, splat(0.0f)), splat(1.0f)); }
LUC_HD V3 ld3(const float* p) { return V3{p[0], p[1], p[2]}; }
LUC_HD float luminance(V3 c) { return dot(c, V3{0.2126f, 0.7152f, 0.0722f}); }

// Rust `f32 as u32` (saturating; NaN -> 0).
LUC_HD uint32_t f2u(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}
LUC_HD int32_t f2i(float x) {
    if (x != x) return 0;
    if (x <= -2147483648.0f) return INT32_MIN;
    if (x >= 2147483648.0f) return INT32_MAX;
    return (int32_t)x;
}

// Transcendentals: one rounding from a double evaluation. Not inlined: the
// double-precision routines are long, and one copy per kernel keeps the
// shading kernels' instruction footprint inside the instruction cache.
#define LUC_DN static __device__ __noinline__
LUC_DN float dsin(float x) { return (float)sin((double)x); }
LUC_DN float dcos(float x) { return (float)cos((double)x); }
LUC_DN float2 dsincos2(float x) {
    double sd, cd;
    sincos((double)x, &sd, &cd);
    return make_float2((float)sd, (float)cd);
}
LUC_D void dsincos(float x, float& s, float& c) {
    float2 r = dsincos2(x);
    s = r.x;
    c = r.y;
}
LUC_DN float dacos(float x) { return (float)acos((double)x); }
LUC_DN float datan2(float y, float x) { return (float)atan2((double)y, (double)x); }
LUC_DN float dexp(float x) { return (float)exp((double)x); }
LUC_DN float dpow(float x, float y) { return (float)pow((double)x, (double)y); }

// ------------------------------------------------------------------ samplers
// PCG-RXS-M-XS with counter seeding (crates/core/src/rng.rs:28-86).
LUC_HD uint32_t pcg_hash(uint32_t input) {
    uint32_t state = input * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}
LUC_HD uint32_t pcg_seed(uint32_t frame_seed, uint32_t pixel, uint32_t sample) {
    uint32_t h = pcg_hash(frame_seed);
    h = pcg_hash(h + pixel);
    return pcg_hash(h + sample);
}
LUC_HD uint32_t pcg_next(uint32_t& state) {
    state = state * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}
LUC_HD float u32_to_unit(uint32_t v) { return (float)(v >> 8) * (1.0f / 16777216.0f); }

// Owen-scrambled Sobol (crates/core/src/sobol.rs:147-235). Dimension 0's
// generator is the bit reversal; dimension 1's direction numbers follow
// V[0] = 2^31, V[k] = V[k-1] ^ (V[k-1] >> 1).
LUC_D uint32_t sobol_dim1_loop(uint32_t index) {
    uint32_t x = 0, v = 0x80000000u;
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        x ^= ((index >> k) & 1u) ? v : 0u;
        v ^= v >> 1;
    }
    return x;
}
// The same product by bytes: g_sobol_dim1_bytes[256 * j + b] is the XOR of
// the direction numbers V[8j + i] over the set bits i of b (4 KB, filled once
// per device by luc_init_sobol_tables), so a draw costs four L1-resident
// loads instead of a 32-step loop; the result is the same XOR sum.
extern __device__ uint32_t g_sobol_dim1_bytes[1024];
LUC_D uint32_t sobol_dim1(uint32_t index) {
    return __ldg(g_sobol_dim1_bytes + (index & 255u)) ^ __ldg(g_sobol_dim1_bytes + 256 + ((index >> 8) & 255u)) ^
           __ldg(g_sobol_dim1_bytes + 512 + ((index >> 16) & 255u)) ^ __ldg(g_sobol_dim1_bytes + 768 + (index >> 24));
}
LUC_HD uint32_t hash_u32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
LUC_D uint32_t lk_perm(uint32_t x, uint32_t seed) {
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
LUC_D uint32_t owen_scramble(uint32_t x, uint32_t seed) { return __brev(lk_perm(__brev(x), seed)); }
LUC_D float sobol_sample(uint32_t index, uint32_t dim, uint32_t seed) {
    uint32_t group = dim >> 1, base = dim & 1u;
    uint32_t gseed = hash_u32(seed ^ (group * 0x9e3779b9u));
    uint32_t shuffled = owen_scramble(index, gseed);
    uint32_t v = base == 0 ? __brev(shuffled) : sobol_dim1(shuffled);
    uint32_t scr = owen_scramble(v, hash_u32(gseed + (base + 1u)));
    return u32_to_unit(scr);
}
LUC_HD uint32_t sobol_pixel_seed(uint32_t pixel, uint32_t frame_seed) {
    return hash_u32(pixel + frame_seed * 0x9e3779b9u);
}

// The per-path sampler (sobol.rs:287-361). `state` is the PCG state for the
// independent sampler and the next dimension for Sobol; index and seed are
// rederived from the path's (pixel, sample).
struct Sampler {
    uint32_t kind, state, index, seed;
    LUC_D float next_f32() {
        if (kind == LUC_SAMPLER_INDEPENDENT) return u32_to_unit(pcg_next(state));
        float v = sobol_sample(index, state, seed);
        state += 1u;
        return v;
    }
    LUC_D void next_vec2(float& x, float& y) {
        if (kind == LUC_SAMPLER_INDEPENDENT) {
            x = u32_to_unit(pcg_next(state));
            y = u32_to_unit(pcg_next(state));
            return;
        }
        // Dimensions 2g and 2g+1 (even-aligned) share the group seed and the
        // scrambled index: sobol_sample for both, with those computed once.
        state = (state + 1u) & ~1u;
        const uint32_t gseed = hash_u32(seed ^ ((state >> 1) * 0x9e3779b9u));
        const uint32_t shuffled = owen_scramble(index, gseed);
        x = u32_to_unit(owen_scramble(__brev(shuffled), hash_u32(gseed + 1u)));
        y = u32_to_unit(owen_scramble(sobol_dim1(shuffled), hash_u32(gseed + 2u)));
        state += 2u;
    }
};
LUC_D Sampler make_sampler(uint32_t kind, uint32_t frame_seed, uint32_t pixel, uint32_t sample) {
    Sampler s;
    s.kind = kind;
    s.index = sample;
    s.seed = sobol_pixel_seed(pixel, frame_seed);
    s.state = kind == LUC_SAMPLER_INDEPENDENT ? pcg_seed(frame_seed, pixel, sample) : 0u;
    return s;
}

// ------------------------------------------------------------------ frames
// Duff et al. ONB (crates/core/src/math.rs:22-47).
LUC_D void onb(V3 n, V3& t, V3& b) {
    float sign = copysignf(1.0f, n.z);
    float a = -1.0f / (sign + n.z);
    float bb = n.x * n.y * a;
    t = V3{1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x};
    b = V3{bb, sign + n.y * n.y * a, -n.y};
}
LUC_D V3 to_world(V3 l, V3 n) {
    V3 t, b;
    onb(n, t, b);
    return t * l.x + b * l.y + n * l.z;
}
LUC_D V3 to_local(V3 w, V3 n) {
    V3 t, b;
    onb(n, t, b);
    return V3{dot(w, t), dot(w, b), dot(w, n)};
}
// Shirley–Chiu concentric map (math.rs:87-99).
LUC_D void concentric_disk(float ux, float uy, float& dx, float& dy) {
    float ox = 2.0f * ux - 1.0f, oy = 2.0f * uy - 1.0f;
    if (ox == 0.0f && oy == 0.0f) {
        dx = 0.0f;
        dy = 0.0f;
        return;
    }
    float r, theta;
    if (fabsf(ox) > fabsf(oy)) {
        r = ox;
        theta = (kPi / 4.0f) * (oy / ox);
    } else {
        r = oy;
        theta = kPi / 2.0f - (kPi / 4.0f) * (ox / oy);
    }
    float s, c;
    dsincos(theta, s, c);
    dx = r * c;
    dy = r * s;
}
LUC_D V3 cosine_hemisphere(float ux, float uy) {
    float dx, dy;
    concentric_disk(ux, uy, dx, dy);
    float z = sqrtf(fmaxf(1.0f - dx * dx - dy * dy, 0.0f));
    return V3{dx, dy, z};
}
// Wächter–Binder ULP offset (math.rs:118-167).
LUC_D V3 offset_ray_origin(V3 p, V3 n) {
    const float ORIGIN = 1.0f / 32.0f, FLOAT_SCALE = 1.0f / 65536.0f, INT_SCALE = 256.0f;
    int32_t ox = f2i(INT_SCALE * n.x), oy = f2i(INT_SCALE * n.y), oz = f2i(INT_SCALE * n.z);
    float px = __int_as_float(__float_as_int(p.x) + (p.x < 0.0f ? -ox : ox));
    float py = __int_as_float(__float_as_int(p.y) + (p.y < 0.0f ? -oy : oy));
    float pz = __int_as_float(__float_as_int(p.z) + (p.z < 0.0f ? -oz : oz));
    return V3{fabsf(p.x) < ORIGIN ? p.x + FLOAT_SCALE * n.x : px,
              fabsf(p.y) < ORIGIN ? p.y + FLOAT_SCALE * n.y : py,
              fabsf(p.z) < ORIGIN ? p.z + FLOAT_SCALE * n.z : pz};
}

// ------------------------------------------------------------------ BSDF
// crates/core/src/bsdf.rs — GGX with VNDF sampling, Smith height-correlated
// G2, Schlick / exact dielectric / exact conductor Fresnel, Walter BTDF,
// Turquin energy compensation, Fresnel-weighted lobe selection.
constexpr float kMinAlpha = 2.0e-3f;
LUC_D float rough_to_alpha(float r) { return fmaxf(r * r, kMinAlpha); }
LUC_D float ggx_d(float alpha, float c) {
    if (c <= 0.0f) return 0.0f;
    float a2 = alpha * alpha, c2 = c * c;
    float sin2 = fmaxf(1.0f - c2, 0.0f);
    float denom = a2 * c2 + sin2;
    return a2 / (kPi * denom * denom);
}
LUC_D float smith_lambda(float alpha, float ct) {
    float c = fabsf(ct);
    if (c >= 1.0f) return 0.0f;
    float c2 = c * c;
    float tan2 = (1.0f - c2) / fmaxf(c2, 1.0e-12f);
    return 0.5f * (-1.0f + sqrtf(1.0f + alpha * alpha * tan2));
}
LUC_D float smith_g1(float alpha, float c) { return 1.0f / (1.0f + smith_lambda(alpha, c)); }
LUC_D float smith_g2(float alpha, float co, float ci) {
    return 1.0f / (1.0f + smith_lambda(alpha, co) + smith_lambda(alpha, ci));
}
LUC_D V3 sample_vndf(V3 wo, float alpha, float ux, float uy) {
    V3 v = normalize(V3{alpha * wo.x, alpha * wo.y, wo.z});
    float lensq = v.x * v.x + v.y * v.y;
    V3 t1 = lensq > 0.0f ? V3{-v.y, v.x, 0.0f} / sqrtf(lensq) : V3{1.0f, 0.0f, 0.0f};
    V3 t2 = cross(v, t1);
    float r = sqrtf(ux);
    float phi = 2.0f * kPi * uy;
    float sp, cp;
    dsincos(phi, sp, cp);
    float p1 = r * cp;
    float p2 = r * sp;
    float s = 0.5f * (1.0f + v.z);
    p2 = (1.0f - s) * sqrtf(fmaxf(1.0f - p1 * p1, 0.0f)) + s * p2;
    V3 nh = p1 * t1 + p2 * t2 + sqrtf(fmaxf(1.0f - p1 * p1 - p2 * p2, 0.0f)) * v;
    return normalize(V3{alpha * nh.x, alpha * nh.y, fmaxf(nh.z, 0.0f)});
}
LUC_D float vndf_pdf(float alpha, V3 wo, V3 m) {
    float co = wo.z;
    if (co <= 0.0f) return 0.0f;
    return smith_g1(alpha, co) * ggx_d(alpha, m.z) / (4.0f * co);
}
LUC_D float vndf_half_pdf(float alpha, V3 wo, V3 m) {
    float co = wo.z, com = dot(wo, m);
    if (co <= 0.0f || com <= 0.0f) return 0.0f;
    return smith_g1(alpha, co) * ggx_d(alpha, fabsf(m.z)) * com / co;
}
LUC_D V3 schlick(V3 f0, float c) {
    float m = clampf(1.0f - c, 0.0f, 1.0f);
    float m2 = m * m;
    return f0 + (splat(1.0f) - f0) * (m2 * m2 * m);
}
LUC_D float fresnel_dielectric(float ci, float eta) {
    float c = fabsf(clampf(ci, -1.0f, 1.0f));
    float sin2_t = (1.0f - c * c) / (eta * eta);
    if (sin2_t >= 1.0f) return 1.0f;
    float ct = sqrtf(fmaxf(1.0f - sin2_t, 0.0f));
    float rpa = (eta * c - ct) / (eta * c + ct);
    float rpe = (c - eta * ct) / (c + eta * ct);
    return 0.5f * (rpa * rpa + rpe * rpe);
}
// The reference's powf(x, 0.5) is taken as the correctly rounded square root:
// for a float x >= 0, sqrt(x) never lies within 2^-50 (relative) of a float
// rounding midpoint, so a pow evaluated to double precision (error <= 2 ulp)
// rounds to the same float as IEEE sqrtf.
LUC_D V3 fresnel_conductor(float ci, V3 eta, V3 k) {
    float c = clampf(ci, 0.0f, 1.0f);
    float c2 = c * c, sin2 = 1.0f - c2;
    V3 eta2 = eta * eta, k2 = k * k;
    V3 t0 = eta2 - k2 - splat(sin2);
    V3 q = vmax(t0 * t0 + 4.0f * eta2 * k2, splat(0.0f));
    V3 a2pb2 = V3{sqrtf(q.x), sqrtf(q.y), sqrtf(q.z)};
    V3 t1 = a2pb2 + splat(c2);
    V3 qa = vmax(0.5f * (a2pb2 + t0), splat(0.0f));
    V3 a = V3{sqrtf(qa.x), sqrtf(qa.y), sqrtf(qa.z)};
    V3 t2 = 2.0f * c * a;
    V3 rs = (t1 - t2) / (t1 + t2);
    V3 t3 = c2 * a2pb2 + splat(sin2 * sin2);
    V3 t4 = t2 * sin2;
    V3 rp = rs * (t3 - t4) / (t3 + t4);
    return 0.5f * (rs + rp);
}
LUC_D V3 reflect(V3 v, V3 n) { return -v + 2.0f * dot(v, n) * n; }

// Turquin energy compensation (bsdf.rs:1236-1272): bilinear lookup of the
// white-Fresnel directional albedo table (32x32, roughness x sqrt(cos)).
LUC_D float energy_lookup(const float* __restrict__ table, float roughness, float cos_o) {
    const int n = 32;
    float fx = clampf(roughness, 0.0f, 1.0f) * (float)(n - 1);
    float fy = sqrtf(clampf(cos_o, 0.0f, 1.0f)) * (float)(n - 1);
    uint32_t x0 = min(f2u(fx), (uint32_t)(n - 1)), y0 = min(f2u(fy), (uint32_t)(n - 1));
    uint32_t x1 = min(x0 + 1u, (uint32_t)(n - 1)), y1 = min(y0 + 1u, (uint32_t)(n - 1));
    float tx = fx - (float)x0, ty = fy - (float)y0;
    float a = __ldg(table + x0 * n + y0), b = __ldg(table + x0 * n + y1);
    float c = __ldg(table + x1 * n + y0), d = __ldg(table + x1 * n + y1);
    float top = a + (b - a) * ty;
    float bot = c + (d - c) * ty;
    return clampf(top + (bot - top) * tx, 1.0e-3f, 1.0f);
}
LUC_D V3 fresnel_average(V3 f0) { return f0 + (splat(1.0f) - f0) * (1.0f / 21.0f); }

struct Surface {
    V3 diffuse_albedo, f0, eta, k, tint;
    float roughness, transmission, relative_ior;
    bool conductor;
};
LUC_D Surface make_surface(const GpuMaterial& m, bool front) {  // bsdf.rs:1345-1375
    V3 base = ld3(m.base_color);
    float metallic = clampf(m.metallic, 0.0f, 1.0f);
    Surface s;
    s.diffuse_albedo = base * (1.0f - metallic);
    float r = (fmaxf(m.ior, 1.0f) - 1.0f) / (fmaxf(m.ior, 1.0f) + 1.0f);
    V3 df0 = splat(r * r);
    s.transmission = clampf(m.transmission, 0.0f, 1.0f) * (1.0f - metallic);
    float ior = fmaxf(m.ior, 1.0f);
    s.roughness = clampf(m.roughness, 0.0f, 1.0f);
    s.f0 = df0 * (1.0f - metallic) + base * metallic;  // glam lerp
    s.eta = ld3(m.eta);
    s.k = ld3(m.k);
    s.conductor = m.k[0] > 0.0f || m.k[1] > 0.0f || m.k[2] > 0.0f;
    s.tint = (base == splat(0.0f)) ? splat(1.0f) : base;
    s.relative_ior = front ? ior : 1.0f / ior;
    return s;
}
LUC_D V3 surf_fresnel(const Surface& s, float c) {
    return s.conductor ? fresnel_conductor(c, s.eta, s.k) : schlick(s.f0, c);
}
LUC_D V3 normal_reflectance(const Surface& s) {
    return s.conductor ? fresnel_conductor(1.0f, s.eta, s.k) : s.f0;
}
LUC_D V3 reflection_fresnel(const Surface& s, float c) {
    if (s.transmission > 0.0f && !s.conductor) return splat(fresnel_dielectric(c, s.relative_ior));
    return surf_fresnel(s, c);
}
LUC_D bool transmission_half(V3 wo, V3 wi, float eta, V3& h) {
    V3 hh = normalize_or(wo + eta * wi, splat(0.0f));
    if (hh == splat(0.0f)) return false;
    h = hh.z < 0.0f ? -hh : hh;
    return true;
}
LUC_D float dielectric_eval(float alpha, float eta, V3 wo, V3 wi) {
    if (wo.z * wi.z >= 0.0f) return 0.0f;
    V3 h;
    if (!transmission_half(wo, wi, eta, h)) return 0.0f;
    float woh = dot(wo, h), wih = dot(wi, h);
    if (woh <= 0.0f || wih >= 0.0f) return 0.0f;
    float denom = woh + eta * wih;
    if (fabsf(denom) < 1.0e-9f) return 0.0f;
    float f = fresnel_dielectric(woh, eta);
    float d = ggx_d(alpha, fabsf(h.z));
    float g2 = smith_g2(alpha, fabsf(wo.z), fabsf(wi.z));
    return ((1.0f - f) * d * g2 * fabsf(wih * woh)) / (fabsf(wo.z) * fabsf(wi.z) * denom * denom);
}
LUC_D float dielectric_pdf(float alpha, float eta, V3 wo, V3 wi) {
    if (wo.z * wi.z >= 0.0f) return 0.0f;
    V3 h;
    if (!transmission_half(wo, wi, eta, h)) return 0.0f;
    float woh = dot(wo, h), wih = dot(wi, h);
    if (woh <= 0.0f || wih >= 0.0f) return 0.0f;
    float denom = woh + eta * wih;
    if (fabsf(denom) < 1.0e-9f) return 0.0f;
    float jac = fabsf(eta * eta * wih) / (denom * denom);
    return vndf_half_pdf(alpha, wo, h) * jac;
}
// What surface::eval, surface::pdf and surface::sample compute from wo alone
// (valid for wo.z > 0), evaluated once per vertex and shared by every
// direction evaluated there. Same operations as the per-call forms, so the
// same values.
struct SurfWo {
    float alpha;      // rough_to_alpha(roughness)
    float p_spec;     // specular_probability(wo.z)
    float e;          // energy_lookup(roughness, wo.z)
    V3 transmitted;   // 1 - specular_albedo(wo.z)
    V3 fav;           // fresnel_average(normal_reflectance)
};
LUC_D SurfWo surf_wo(const Surface& s, const float* table, float cos_o) {
    SurfWo w;
    w.alpha = rough_to_alpha(s.roughness);
    w.e = energy_lookup(table, s.roughness, fabsf(cos_o));
    w.fav = fresnel_average(normal_reflectance(s));
    const V3 sa = vclamp01(surf_fresnel(s, fabsf(cos_o)) * w.e + w.fav * (1.0f - w.e));  // specular_albedo
    w.transmitted = splat(1.0f) - sa;
    if (s.transmission > 0.0f) {
        float f = fresnel_dielectric(fabsf(cos_o), s.relative_ior);
        w.p_spec = f >= 1.0f ? 1.0f : clampf(f, 0.05f, 0.95f);
    } else {
        float spec = luminance(sa);
        float diff = luminance(s.diffuse_albedo * w.transmitted);
        w.p_spec = spec + diff <= 0.0f ? 1.0f : clampf(spec / (spec + diff), 0.1f, 0.9f);
    }
    return w;
}
// surface::eval (bsdf.rs:1493-1540) for wo.z > 0. Returns f.
LUC_D V3 bsdf_eval_w(const Surface& s, const SurfWo& w, V3 wo, V3 wi) {
    if (wi.z < 0.0f) {
        if (s.transmission <= 0.0f) return splat(0.0f);
        float t = dielectric_eval(w.alpha, s.relative_ior, wo, wi);
        return splat(t) * s.transmission * s.tint;
    }
    if (wi.z <= 0.0f) return splat(0.0f);
    V3 f = s.diffuse_albedo * kInvPi * w.transmitted * (1.0f - s.transmission);
    V3 h = normalize_or(wo + wi, splat(0.0f));
    if (!(h == splat(0.0f))) {
        float d = ggx_d(w.alpha, h.z);
        float g2 = smith_g2(w.alpha, wo.z, wi.z);
        V3 fr = reflection_fresnel(s, fmaxf(dot(wo, h), 0.0f));
        V3 single = fr * (d * g2 / (4.0f * wo.z * wi.z));
        if (s.transmission > 0.0f) {
            f = f + single;
        } else {
            V3 comp = splat(1.0f) + w.fav * ((1.0f - w.e) / w.e);
            f = f + single * comp;
        }
    }
    return f;
}
LUC_D V3 bsdf_eval(const Surface& s, const float* table, V3 wo, V3 wi) {
    if (wo.z <= 0.0f) return splat(0.0f);
    return bsdf_eval_w(s, surf_wo(s, table, wo.z), wo, wi);
}
// surface::pdf (bsdf.rs:1543-1562) for wo.z > 0.
LUC_D float bsdf_pdf_w(const Surface& s, const SurfWo& w, V3 wo, V3 wi) {
    float rest = 1.0f - w.p_spec;
    if (wi.z < 0.0f) {
        if (s.transmission <= 0.0f) return 0.0f;
        return rest * s.transmission * dielectric_pdf(w.alpha, s.relative_ior, wo, wi);
    }
    if (wi.z <= 0.0f) return 0.0f;
    float spec = 0.0f;
    V3 h = normalize_or(wo + wi, splat(0.0f));
    if (!(h == splat(0.0f))) spec = vndf_pdf(w.alpha, wo, h);
    float diff = wi.z * kInvPi;
    return w.p_spec * spec + rest * (1.0f - s.transmission) * diff;
}
LUC_D float bsdf_pdf(const Surface& s, const float* table, V3 wo, V3 wi) {
    if (wo.z <= 0.0f) return 0.0f;
    return bsdf_pdf_w(s, surf_wo(s, table, wo.z), wo, wi);
}
struct BsdfSample {
    V3 wi, weight;
    float pdf;
};
// The direction half of surface::sample (bsdf.rs:1571-1661) for wo.z > 0:
// lobe choice by u_lobe, then GGX reflection (VNDF), rough transmission or
// cosine-weighted diffuse. False where surface::sample returns no sample.
LUC_D bool bsdf_sample_dir_w(const Surface& s, const SurfWo& w, V3 wo, float u_lobe, float ux, float uy, V3& wi) {
    const float p_spec = w.p_spec, alpha = w.alpha;
    if (u_lobe < p_spec) {
        V3 m = sample_vndf(wo, alpha, ux, uy);
        V3 r = reflect(wo, m);
        if (r.z <= 0.0f) return false;
        wi = r;
    } else if (u_lobe < p_spec + (1.0f - p_spec) * s.transmission) {
        V3 m = sample_vndf(wo, alpha, ux, uy);
        float eta = s.relative_ior;
        float ci = dot(wo, m);
        float sin2_i = fmaxf(1.0f - ci * ci, 0.0f);
        float sin2_t = sin2_i / (eta * eta);
        if (sin2_t >= 1.0f) return false;
        float ct = sqrtf(1.0f - sin2_t);
        V3 wt = normalize_or(-wo / eta + (ci / eta - copysignf(ct, ci)) * m, splat(0.0f));
        if (wt.z >= 0.0f) return false;
        wi = wt;
    } else {
        wi = cosine_hemisphere(ux, uy);
    }
    if (wi.z == 0.0f || wi == splat(0.0f)) return false;
    if (wi.z < 0.0f && s.transmission <= 0.0f) return false;
    return true;
}
LUC_D bool bsdf_sample_dir(const Surface& s, const float* table, V3 wo, float u_lobe, float ux, float uy, V3& wi) {
    if (wo.z <= 0.0f) return false;
    return bsdf_sample_dir_w(s, surf_wo(s, table, wo.z), wo, u_lobe, ux, uy, wi);
}

// surface::sample (bsdf.rs:1571-1661): direction, then f and the pdf there.
LUC_D BsdfSample bsdf_sample(const Surface& s, const float* table, V3 wo, float u_lobe, float ux, float uy) {
    BsdfSample bad{V3{0.0f, 0.0f, 1.0f}, splat(0.0f), 0.0f};
    if (wo.z <= 0.0f) return bad;
    const SurfWo w = surf_wo(s, table, wo.z);
    V3 wi;
    if (!bsdf_sample_dir_w(s, w, wo, u_lobe, ux, uy, wi)) return bad;
    V3 f = bsdf_eval_w(s, w, wo, wi);
    float pdf = bsdf_pdf_w(s, w, wo, wi);
    if (pdf <= 0.0f) return bad;
    return BsdfSample{wi, f * (fabsf(wi.z) / pdf), pdf};
}

LUC_D float power_heuristic(float a, float b) {
    if (a <= 0.0f) return 0.0f;
    float r = b / a;
    return 1.0f / (1.0f + r * r);
}

// ------------------------------------------------------------------ geometry
constexpr float kTMax = 1.0e30f;
constexpr float kTMin = 1.0e-4f;

// scene.rs:76-97
LUC_D bool hit_sphere(V3 c, float radius, V3 o, V3 d, float tmin, float tmax, float& out) {
    V3 oc = o - c;
    float a = dot(d, d);
    float h = dot(oc, d);
    float cc = dot(oc, oc) - radius * radius;
    float disc = h * h - a * cc;
    if (disc < 0.0f) return false;
    float sd = sqrtf(disc);
    float t = (-h - sd) / a;
    if (t < tmin || t > tmax) {
        t = (-h + sd) / a;
        if (t < tmin || t > tmax) return false;
    }
    out = t;
    return true;
}
// scene.rs:120-148
LUC_D bool hit_quad(V3 org, V3 eu, V3 ev, V3 n, V3 o, V3 d, float tmin, float tmax, float& out) {
    float denom = dot(n, d);
    if (fabsf(denom) < 1.0e-8f) return false;
    float t = (dot(n, org) - dot(n, o)) / denom;
    if (t < tmin || t > tmax) return false;
    V3 p = o + t * d;
    V3 q = p - org;
    V3 nr = cross(eu, ev);
    V3 w = nr / dot(nr, nr);
    float a = dot(w, cross(q, ev));
    float b = dot(w, cross(eu, q));
    if (!(a >= 0.0f && a <= 1.0f) || !(b >= 0.0f && b <= 1.0f)) return false;
    out = t;
    return true;
}
// Möller–Trumbore, double-sided (bvh.rs:930-968).
LUC_D bool hit_triangle(V3 p0, V3 p1, V3 p2, V3 o, V3 d, float tmin, float tmax, float& tout, float& uout,
                        float& vout) {
    V3 e1 = p1 - p0, e2 = p2 - p0;
    V3 pv = cross(d, e2);
    float det = dot(e1, pv);
    if (fabsf(det) < 1.0e-12f) return false;
    float inv_det = 1.0f / det;
    V3 tv = o - p0;
    float u = dot(tv, pv) * inv_det;
    if (!(u >= 0.0f && u <= 1.0f)) return false;
    V3 qv = cross(tv, e1);
    float v = dot(d, qv) * inv_det;
    if (v < 0.0f || u + v > 1.0f) return false;
    float t = dot(e2, qv) * inv_det;
    if (t < tmin || t > tmax) return false;
    tout = t;
    uout = u;
    vout = v;
    return true;
}
// bvh.rs:165-178
LUC_D V3 safe_inv_dir(V3 d) {
    const float BIG = 1.0e16f, SMALL = 1.0f / BIG;
    return V3{fabsf(d.x) > SMALL ? 1.0f / d.x : copysignf(BIG, d.x),
              fabsf(d.y) > SMALL ? 1.0f / d.y : copysignf(BIG, d.y),
              fabsf(d.z) > SMALL ? 1.0f / d.z : copysignf(BIG, d.z)};
}

}  // namespace luc
