// ORACLE — test infrastructure only. This is a CPU restatement of Lucida's
// Rust reference tracer (crates/core/src), used by tests/, by the smoke check
// and by bench.py's CPU-baseline leg as the checker. The product path never
// links or calls it.
//
// Arithmetic conventions (the reference's, restated):
//   * every f32 operation is a separate IEEE operation — Rust never contracts
//     a*b+c into an FMA, so this file is compiled with -ffp-contract=off;
//   * glam 0.33's Vec3 is scalar: dot is ((x*x')+(y*y'))+(z*z'), cross is
//     (y*z' - y'*z, z*x' - z'*x, x*y' - x'*y), normalize is v * (1/len);
//   * transcendentals are glibc's sinf/cosf/tanf/acosf/asinf/atan2f/expf/powf,
//     which is what Rust's f32 methods call on Linux;
//   * `f32 as u32/i32/usize` is Rust's saturating cast (NaN -> 0).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include "../include/lucida_layout.h"

namespace oracle {

static const float PI = 3.14159265358979323846f;
static const float TAU = 6.28318530717958647692f;
static const float INV_PI = 0.318309886183790671538f;

// ---------------------------------------------------------------- casts
inline uint32_t f2u(float x) {  // Rust `x as u32`
    if (!(x > 0.0f)) return 0u;  // NaN, 0, negatives
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}
inline int32_t f2i(float x) {  // Rust `x as i32`
    if (x != x) return 0;
    if (x <= -2147483648.0f) return INT32_MIN;
    if (x >= 2147483648.0f) return INT32_MAX;
    return (int32_t)x;
}
inline int64_t f2i64(float x) {  // Rust `x as i64`
    if (x != x) return 0;
    if (x <= -9.2233720368547758e18f) return INT64_MIN;
    if (x >= 9.2233720368547758e18f) return INT64_MAX;
    return (int64_t)x;
}
inline uint64_t f2usize(float x) {  // Rust `x as usize`
    if (!(x > 0.0f)) return 0u;
    if (x >= 1.8446744073709552e19f) return UINT64_MAX;
    return (uint64_t)x;
}
// Rust f32::max / f32::min: NaN-ignoring.
inline float fmax_(float a, float b) { return std::fmax(a, b); }
inline float fmin_(float a, float b) { return std::fmin(a, b); }
// Rust f32::clamp: NaN passes through.
inline float clampf(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
inline uint32_t bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

// ---------------------------------------------------------------- libm mode
// How the render-time transcendentals round. 0 (the default): glibc's f32
// functions, what the reference's Rust calls. 1: evaluated in double and
// rounded once to f32, the rounding the CUDA integrator uses. Scene
// construction and the tables the device receives from the host (energy
// table, environment row sines, camera uniforms) always use glibc. Set only
// between renders (orc_set_libm_mode); render threads read it.
extern int g_libm_mode;
inline float m_sin(float x) { return g_libm_mode ? (float)std::sin((double)x) : std::sin(x); }
inline float m_cos(float x) { return g_libm_mode ? (float)std::cos((double)x) : std::cos(x); }
inline float m_acos(float x) { return g_libm_mode ? (float)std::acos((double)x) : std::acos(x); }
inline float m_atan2(float y, float x) {
    return g_libm_mode ? (float)std::atan2((double)y, (double)x) : std::atan2(y, x);
}
inline float m_pow(float x, float y) { return g_libm_mode ? (float)std::pow((double)x, (double)y) : std::pow(x, y); }

// ---------------------------------------------------------------- path signature
// A per-thread hash of a path's discrete events (which primitive each ray
// hit, each shadow ray's outcome, each BSDF lobe choice and rejection, each
// light pick), filled only while g_path_sig points somewhere. Two traces of
// one sample with equal signatures took the same branches everywhere; their
// radiance can differ only by rounding carried along the same path.
extern thread_local uint64_t* g_path_sig;
inline void sig_event(uint32_t kind, uint64_t value) {
    if (!g_path_sig) return;
    uint64_t h = *g_path_sig ^ (((uint64_t)kind << 56) + value + 0x9E3779B97F4A7C15ull);
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    *g_path_sig = h;
}
inline float from_bits(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t reverse_bits(uint32_t x) {
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
    x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
    return (x >> 16) | (x << 16);
}
inline int leading_zeros(uint32_t x) { return x == 0 ? 32 : __builtin_clz(x); }

// ---------------------------------------------------------------- Vec2/Vec3
struct Vec2 {
    float x, y;
    Vec2() : x(0), y(0) {}
    Vec2(float a, float b) : x(a), y(b) {}
};

struct Vec3 {
    float x, y, z;
    Vec3() : x(0), y(0), z(0) {}
    Vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    static Vec3 splat(float v) { return Vec3(v, v, v); }
    static Vec3 from(const float* a) { return Vec3(a[0], a[1], a[2]); }
    void to(float* a) const { a[0] = x; a[1] = y; a[2] = z; }
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    float& at(int i) { return i == 0 ? x : (i == 1 ? y : z); }
    Vec3 operator+(Vec3 o) const { return Vec3(x + o.x, y + o.y, z + o.z); }
    Vec3 operator-(Vec3 o) const { return Vec3(x - o.x, y - o.y, z - o.z); }
    Vec3 operator*(Vec3 o) const { return Vec3(x * o.x, y * o.y, z * o.z); }
    Vec3 operator/(Vec3 o) const { return Vec3(x / o.x, y / o.y, z / o.z); }
    Vec3 operator*(float s) const { return Vec3(x * s, y * s, z * s); }
    Vec3 operator/(float s) const { return Vec3(x / s, y / s, z / s); }
    Vec3 operator-() const { return Vec3(-x, -y, -z); }
    Vec3& operator+=(Vec3 o) { x = x + o.x; y = y + o.y; z = z + o.z; return *this; }
    Vec3& operator*=(Vec3 o) { x = x * o.x; y = y * o.y; z = z * o.z; return *this; }
    Vec3& operator*=(float s) { x = x * s; y = y * s; z = z * s; return *this; }
    bool operator==(Vec3 o) const { return x == o.x && y == o.y && z == o.z; }
    bool operator!=(Vec3 o) const { return !(*this == o); }
    float dot(Vec3 o) const { return ((x * o.x) + (y * o.y)) + (z * o.z); }
    Vec3 cross(Vec3 o) const {
        return Vec3(y * o.z - o.y * z, z * o.x - o.z * x, x * o.y - o.x * y);
    }
    float length_squared() const { return dot(*this); }
    float length() const { return std::sqrt(dot(*this)); }
    float length_recip() const { return 1.0f / length(); }
    Vec3 normalize() const { return *this * length_recip(); }
    Vec3 normalize_or(Vec3 fb) const {
        float r = length_recip();
        if (std::isfinite(r) && r > 0.0f) return *this * r;
        return fb;
    }
    Vec3 normalize_or_zero() const { return normalize_or(Vec3()); }
    Vec3 min(Vec3 o) const { return Vec3(fmin_(x, o.x), fmin_(y, o.y), fmin_(z, o.z)); }
    Vec3 max(Vec3 o) const { return Vec3(fmax_(x, o.x), fmax_(y, o.y), fmax_(z, o.z)); }
    float max_element() const { return fmax_(x, fmax_(y, z)); }
    float min_element() const { return fmin_(x, fmin_(y, z)); }
    Vec3 clamp(Vec3 lo, Vec3 hi) const { return max(lo).min(hi); }
    Vec3 abs() const { return Vec3(std::fabs(x), std::fabs(y), std::fabs(z)); }
    // glam 0.33: self * (1 - s) + rhs * s
    Vec3 lerp(Vec3 o, float s) const { return *this * (1.0f - s) + o * s; }
    Vec3 powf(float e) const { return Vec3(m_pow(x, e), m_pow(y, e), m_pow(z, e)); }
    bool is_finite() const { return std::isfinite(x) && std::isfinite(y) && std::isfinite(z); }
};
inline Vec3 operator*(float s, Vec3 v) { return Vec3(s * v.x, s * v.y, s * v.z); }

// ---------------------------------------------------------------- rng.rs
// rng.rs:28-32
inline uint32_t pcg_hash(uint32_t input) {
    uint32_t state = input * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
    return (word >> 22) ^ word;
}

// rng.rs:34-86
struct Rng {
    uint32_t state;
    Rng() : state(0) {}
    Rng(uint32_t frame_seed, uint32_t pixel, uint32_t sample) {
        uint32_t h = pcg_hash(frame_seed);
        h = pcg_hash(h + pixel);
        h = pcg_hash(h + sample);
        state = h;
    }
    uint32_t next_u32() {
        state = state * 747796405u + 2891336453u;
        uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
        return (word >> 22) ^ word;
    }
    float next_f32() { return (float)(next_u32() >> 8) * (1.0f / 16777216.0f); }
    Vec2 next_vec2() {
        float x = next_f32();
        float y = next_f32();
        return Vec2(x, y);
    }
};

// ---------------------------------------------------------------- sobol.rs
// sobol.rs:88-130: dimension 0 is bit reversal; dimension 1 from the
// degree-1 polynomial with m = [1] (V-recurrence V[i] = V[i-1] ^ V[i-1] >> 1).
struct SobolTable {
    uint32_t v[2][32];
    SobolTable() {
        for (int k = 0; k < 32; ++k) v[0][k] = 1u << (31 - k);
        uint32_t vv[33] = {0};
        vv[1] = 1u << 31;
        for (int i = 2; i <= 32; ++i) vv[i] = vv[i - 1] ^ (vv[i - 1] >> 1);
        for (int k = 0; k < 32; ++k) v[1][k] = vv[k + 1];
    }
};
const SobolTable& sobol_table();

inline uint32_t sobol(uint32_t index, uint32_t dim) {  // sobol.rs:147-156
    const uint32_t* v = sobol_table().v[dim];
    uint32_t x = 0;
    for (int k = 0; k < 32; ++k)
        if ((index >> k) & 1u) x ^= v[k];
    return x;
}
inline uint32_t laine_karras_permutation(uint32_t x, uint32_t seed) {  // :171-178
    x = x + seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
inline uint32_t owen_scramble(uint32_t x, uint32_t seed) {  // :187-189
    return reverse_bits(laine_karras_permutation(reverse_bits(x), seed));
}
inline uint32_t hash_u32(uint32_t x) {  // :197-204
    x ^= x >> 16;
    x = x * 0x7feb352du;
    x ^= x >> 15;
    x = x * 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
inline float sobol_sample(uint32_t index, uint32_t dim, uint32_t seed) {  // :221-235
    uint32_t group = dim / 2u;
    uint32_t base = dim % 2u;
    uint32_t group_seed = hash_u32(seed ^ (group * 0x9e3779b9u));
    uint32_t shuffled = owen_scramble(index, group_seed);
    uint32_t v = sobol(shuffled, base);
    uint32_t scrambled = owen_scramble(v, hash_u32(group_seed + (base + 1u)));
    return (float)(scrambled >> 8) * (1.0f / 16777216.0f);
}

// sobol.rs:287-361
struct Sampler {
    uint32_t kind;  // LUC_SAMPLER_*
    Rng rng;
    uint32_t index, seed, dim;
    Sampler(uint32_t kind_, uint32_t frame_seed, uint32_t pixel, uint32_t sample)
        : kind(kind_), rng(frame_seed, pixel, sample), index(sample),
          seed(hash_u32(pixel + frame_seed * 0x9e3779b9u)), dim(0) {}
    float next_f32() {
        if (kind == LUC_SAMPLER_INDEPENDENT) return rng.next_f32();
        float v = sobol_sample(index, dim, seed);
        dim += 1;
        return v;
    }
    Vec2 next_vec2() {
        if (kind == LUC_SAMPLER_INDEPENDENT) return rng.next_vec2();
        dim = (dim + 1u) & ~1u;
        float x = sobol_sample(index, dim, seed);
        float y = sobol_sample(index, dim + 1u, seed);
        dim += 2;
        return Vec2(x, y);
    }
};

// ---------------------------------------------------------------- math.rs
inline void onb(Vec3 n, Vec3& t, Vec3& b) {  // math.rs:22-30
    float sign = std::copysign(1.0f, n.z);
    float a = -1.0f / (sign + n.z);
    float bb = n.x * n.y * a;
    t = Vec3(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    b = Vec3(bb, sign + n.y * n.y * a, -n.y);
}
inline Vec3 to_world(Vec3 l, Vec3 n) {  // :34-37
    Vec3 t, b;
    onb(n, t, b);
    return t * l.x + b * l.y + n * l.z;
}
inline Vec3 to_local(Vec3 w, Vec3 n) {  // :44-47
    Vec3 t, b;
    onb(n, t, b);
    return Vec3(w.dot(t), w.dot(b), w.dot(n));
}
inline Vec2 concentric_sample_disk(Vec2 u) {  // :87-99
    Vec2 o(2.0f * u.x - 1.0f, 2.0f * u.y - 1.0f);
    if (o.x == 0.0f && o.y == 0.0f) return Vec2(0, 0);
    float r, theta;
    if (std::fabs(o.x) > std::fabs(o.y)) {
        r = o.x;
        theta = (PI / 4.0f) * (o.y / o.x);
    } else {
        r = o.y;
        theta = PI / 2.0f - (PI / 4.0f) * (o.x / o.y);
    }
    return Vec2(r * m_cos(theta), r * m_sin(theta));
}
inline Vec3 sample_cosine_hemisphere(Vec2 u) {  // :68-74
    Vec2 d = concentric_sample_disk(u);
    float z = std::sqrt(fmax_(1.0f - d.x * d.x - d.y * d.y, 0.0f));
    return Vec3(d.x, d.y, z);
}
inline float cosine_hemisphere_pdf(float c) { return fmax_(c * INV_PI, 0.0f); }
inline Vec3 offset_ray_origin(Vec3 p, Vec3 n) {  // :118-167
    const float ORIGIN = 1.0f / 32.0f, FLOAT_SCALE = 1.0f / 65536.0f, INT_SCALE = 256.0f;
    int32_t of[3] = {f2i(INT_SCALE * n.x), f2i(INT_SCALE * n.y), f2i(INT_SCALE * n.z)};
    float pi_[3];
    for (int a = 0; a < 3; ++a) {
        float pa = p[a];
        int32_t o = pa < 0.0f ? -of[a] : of[a];
        pi_[a] = from_bits((uint32_t)((int32_t)bits(pa) + o));
    }
    return Vec3(std::fabs(p.x) < ORIGIN ? p.x + FLOAT_SCALE * n.x : pi_[0],
                std::fabs(p.y) < ORIGIN ? p.y + FLOAT_SCALE * n.y : pi_[1],
                std::fabs(p.z) < ORIGIN ? p.z + FLOAT_SCALE * n.z : pi_[2]);
}
inline float luminance(Vec3 c) { return c.dot(Vec3(0.2126f, 0.7152f, 0.0722f)); }

// ---------------------------------------------------------------- camera.rs
struct Ray {
    Vec3 origin, dir;
};
struct Camera {  // camera.rs:302-366
    Vec3 eye, look_at, up;
    float vfov_deg, aperture, focus_distance;
    static Camera make(Vec3 eye, Vec3 at, float vfov) {
        Camera c;
        c.eye = eye;
        c.look_at = at;
        c.up = Vec3(0, 1, 0);
        c.vfov_deg = vfov;
        c.aperture = 0.0f;
        c.focus_distance = (at - eye).length();
        return c;
    }
    void basis(Vec3& right, Vec3& down, Vec3& forward) const {
        forward = (look_at - eye).normalize();
        right = forward.cross(up).normalize();
        Vec3 upv = right.cross(forward);
        down = -upv;
    }
    void write_uniforms(GpuUniforms& u, float aspect) const {
        Vec3 right, down, forward;
        basis(right, down, forward);
        float rad = vfov_deg * (PI / 180.0f);  // f32::to_radians
        float half_height = std::tan(rad * 0.5f) * focus_distance;
        float half_width = half_height * aspect;
        Vec3 horizontal = right * (2.0f * half_width);
        Vec3 vertical = down * (2.0f * half_height);
        Vec3 upper_left = eye + forward * focus_distance - right * half_width - down * half_height;
        eye.to(u.cam_origin);
        upper_left.to(u.cam_upper_left);
        horizontal.to(u.cam_horizontal);
        vertical.to(u.cam_vertical);
        u.lens_radius = aperture * 0.5f;
        u.focus_distance = focus_distance;
    }
};
inline Ray generate_ray(const GpuUniforms& u, uint32_t x, uint32_t y, Vec2 puv, Vec2 luv) {
    // camera.rs:373-405
    float s = ((float)x + puv.x) / (float)u.width;
    float t = ((float)y + puv.y) / (float)u.height;
    Vec3 origin = Vec3::from(u.cam_origin);
    Vec3 target = Vec3::from(u.cam_upper_left) + s * Vec3::from(u.cam_horizontal) +
                  t * Vec3::from(u.cam_vertical);
    if (u.lens_radius <= 0.0f) return Ray{origin, (target - origin).normalize()};
    Vec2 d0 = concentric_sample_disk(luv);
    Vec2 d(d0.x * u.lens_radius, d0.y * u.lens_radius);
    Vec3 right = Vec3::from(u.cam_horizontal).normalize();
    Vec3 down = Vec3::from(u.cam_vertical).normalize();
    Vec3 offset = right * d.x + down * d.y;
    Vec3 o2 = origin + offset;
    return Ray{o2, (target - o2).normalize()};
}

// ---------------------------------------------------------------- bsdf.rs
static const float MIN_ALPHA = 2.0e-3f;
inline float roughness_to_alpha(float r) { return fmax_(r * r, MIN_ALPHA); }
inline float ggx_d(float alpha, float c) {  // bsdf.rs:87-96
    if (c <= 0.0f) return 0.0f;
    float a2 = alpha * alpha;
    float c2 = c * c;
    float sin2 = fmax_(1.0f - c2, 0.0f);
    float denom = a2 * c2 + sin2;
    return a2 / (PI * denom * denom);
}
inline float smith_lambda(float alpha, float cos_theta) {  // :131-140
    float c = std::fabs(cos_theta);
    if (c >= 1.0f) return 0.0f;
    float c2 = c * c;
    float tan2 = (1.0f - c2) / fmax_(c2, 1.0e-12f);
    return 0.5f * (-1.0f + std::sqrt(1.0f + alpha * alpha * tan2));
}
inline float smith_g1(float alpha, float c) { return 1.0f / (1.0f + smith_lambda(alpha, c)); }
inline float smith_g2(float alpha, float co, float ci) {
    return 1.0f / (1.0f + smith_lambda(alpha, co) + smith_lambda(alpha, ci));
}
inline Vec3 sample_ggx_vndf(Vec3 wo, float alpha, Vec2 u) {  // :187-216
    Vec3 v = Vec3(alpha * wo.x, alpha * wo.y, wo.z).normalize();
    float lensq = v.x * v.x + v.y * v.y;
    Vec3 t1 = lensq > 0.0f ? Vec3(-v.y, v.x, 0.0f) / std::sqrt(lensq) : Vec3(1, 0, 0);
    Vec3 t2 = v.cross(t1);
    float r = std::sqrt(u.x);
    float phi = 2.0f * PI * u.y;
    float p1 = r * m_cos(phi);
    float p2 = r * m_sin(phi);
    float s = 0.5f * (1.0f + v.z);
    p2 = (1.0f - s) * std::sqrt(fmax_(1.0f - p1 * p1, 0.0f)) + s * p2;
    Vec3 nh = p1 * t1 + p2 * t2 + std::sqrt(fmax_(1.0f - p1 * p1 - p2 * p2, 0.0f)) * v;
    return Vec3(alpha * nh.x, alpha * nh.y, fmax_(nh.z, 0.0f)).normalize();
}
inline float ggx_vndf_pdf(float alpha, Vec3 wo, Vec3 m) {  // :243-249
    float cos_o = wo.z;
    if (cos_o <= 0.0f) return 0.0f;
    return smith_g1(alpha, cos_o) * ggx_d(alpha, m.z) / (4.0f * cos_o);
}
inline float ggx_vndf_half_pdf(float alpha, Vec3 wo, Vec3 m) {  // :275-282
    float cos_o = wo.z;
    float cos_om = wo.dot(m);
    if (cos_o <= 0.0f || cos_om <= 0.0f) return 0.0f;
    return smith_g1(alpha, cos_o) * ggx_d(alpha, std::fabs(m.z)) * cos_om / cos_o;
}
inline Vec3 fresnel_schlick(Vec3 f0, float c) {  // :301-305
    float m = clampf(1.0f - c, 0.0f, 1.0f);
    float m2 = m * m;
    return f0 + (Vec3::splat(1.0f) - f0) * (m2 * m2 * m);
}
inline float fresnel_dielectric(float cos_theta_i, float eta) {  // :314-329
    float c = std::fabs(clampf(cos_theta_i, -1.0f, 1.0f));
    float sin2_t = (1.0f - c * c) / (eta * eta);
    if (sin2_t >= 1.0f) return 1.0f;
    float cos_t = std::sqrt(fmax_(1.0f - sin2_t, 0.0f));
    float rpa = (eta * c - cos_t) / (eta * c + cos_t);
    float rpe = (c - eta * cos_t) / (c + eta * cos_t);
    return 0.5f * (rpa * rpa + rpe * rpe);
}
inline float f0_from_ior(float ior) {
    float r = (ior - 1.0f) / (ior + 1.0f);
    return r * r;
}
inline Vec3 fresnel_conductor(float cos_theta_i, Vec3 eta, Vec3 k) {  // :358-378
    float c = clampf(cos_theta_i, 0.0f, 1.0f);
    float c2 = c * c;
    float sin2 = 1.0f - c2;
    Vec3 eta2 = eta * eta;
    Vec3 k2 = k * k;
    Vec3 t0 = eta2 - k2 - Vec3::splat(sin2);
    Vec3 a2pb2 = (t0 * t0 + 4.0f * eta2 * k2).max(Vec3()).powf(0.5f);
    Vec3 t1 = a2pb2 + Vec3::splat(c2);
    Vec3 a = (0.5f * (a2pb2 + t0)).max(Vec3()).powf(0.5f);
    Vec3 t2 = 2.0f * c * a;
    Vec3 rs = (t1 - t2) / (t1 + t2);
    Vec3 t3 = c2 * a2pb2 + Vec3::splat(sin2 * sin2);
    Vec3 t4 = t2 * sin2;
    Vec3 rp = rs * (t3 - t4) / (t3 + t4);
    return 0.5f * (rs + rp);
}
inline Vec3 reflect(Vec3 v, Vec3 n) { return -v + 2.0f * v.dot(n) * n; }
inline bool refract(Vec3 wo, Vec3 m, float eta, Vec3& out) {  // :555-567
    float cos_i = wo.dot(m);
    float sin2_i = fmax_(1.0f - cos_i * cos_i, 0.0f);
    float sin2_t = sin2_i / (eta * eta);
    if (sin2_t >= 1.0f) return false;
    float cos_t = std::sqrt(1.0f - sin2_t);
    Vec3 wt = -wo / eta + (cos_i / eta - std::copysign(cos_t, cos_i)) * m;
    out = wt.normalize_or_zero();
    return true;
}

struct BsdfSample {
    Vec3 wi, weight;
    float pdf;
    bool valid() const { return pdf > 0.0f; }
    static BsdfSample invalid() { return BsdfSample{Vec3(0, 0, 1), Vec3(), 0.0f}; }
};

// specular::sample_single (bsdf.rs:488-511)
inline BsdfSample specular_sample_single(float alpha, Vec3 f0, Vec3 wo, Vec2 u) {
    if (wo.z <= 0.0f) return BsdfSample::invalid();
    Vec3 m = sample_ggx_vndf(wo, alpha, u);
    Vec3 wi = reflect(wo, m);
    if (wi.z <= 0.0f) return BsdfSample::invalid();
    float pdf = ggx_vndf_pdf(alpha, wo, m);
    if (pdf <= 0.0f) return BsdfSample::invalid();
    Vec3 f = fresnel_schlick(f0, fmax_(wo.dot(m), 0.0f));
    float g1 = smith_g1(alpha, wo.z);
    float g2 = smith_g2(alpha, wo.z, wi.z);
    return BsdfSample{wi, f * (g2 / g1), pdf};
}
// bsdf.rs:760-777
float specular_directional_albedo_grid(float alpha, float cos_theta_o, uint32_t grid);

// energy module (bsdf.rs:1178-1273)
static const int ENERGY_TABLE_SIZE = 32;
const float* energy_table();  // computed once, bsdf.rs:1210-1225
std::vector<float> compute_energy_table();
inline float energy_lookup(const float* table, float roughness, float cos_theta_o) {
    const int n = ENERGY_TABLE_SIZE;
    float fx = clampf(roughness, 0.0f, 1.0f) * (float)(n - 1);
    float fy = std::sqrt(clampf(cos_theta_o, 0.0f, 1.0f)) * (float)(n - 1);
    uint64_t x0 = std::min<uint64_t>(f2usize(fx), n - 1);
    uint64_t y0 = std::min<uint64_t>(f2usize(fy), n - 1);
    uint64_t x1 = std::min<uint64_t>(x0 + 1, n - 1);
    uint64_t y1 = std::min<uint64_t>(y0 + 1, n - 1);
    float tx = fx - (float)x0;
    float ty = fy - (float)y0;
    float a = table[x0 * n + y0], b = table[x0 * n + y1];
    float c = table[x1 * n + y0], d = table[x1 * n + y1];
    float top = a + (b - a) * ty;
    float bot = c + (d - c) * ty;
    return clampf(top + (bot - top) * tx, 1.0e-3f, 1.0f);
}
inline float directional_albedo(float r, float c) { return energy_lookup(energy_table(), r, c); }
inline Vec3 fresnel_average(Vec3 f0) {
    return f0 + (Vec3::splat(1.0f) - f0) * (1.0f / 21.0f);
}
inline Vec3 compensation(float roughness, float cos_o, Vec3 f0) {
    float e = directional_albedo(roughness, cos_o);
    return Vec3::splat(1.0f) + fresnel_average(f0) * ((1.0f - e) / e);
}

// surface module (bsdf.rs:1301-1661)
struct Surface {
    Vec3 diffuse_albedo;
    float roughness;
    Vec3 f0, eta, k;
    bool conductor;
    float transmission;
    Vec3 transmission_tint;
    float relative_ior;

    static Surface from_material(const GpuMaterial& m, bool front_face) {
        Vec3 base = Vec3::from(m.base_color);
        float metallic = clampf(m.metallic, 0.0f, 1.0f);
        Surface s;
        s.diffuse_albedo = base * (1.0f - metallic);
        Vec3 df0 = Vec3::splat(f0_from_ior(fmax_(m.ior, 1.0f)));
        s.transmission = clampf(m.transmission, 0.0f, 1.0f) * (1.0f - metallic);
        float ior = fmax_(m.ior, 1.0f);
        s.roughness = clampf(m.roughness, 0.0f, 1.0f);
        s.f0 = df0.lerp(base, metallic);
        s.eta = Vec3::from(m.eta);
        s.k = Vec3::from(m.k);
        s.conductor = m.k[0] > 0.0f || m.k[1] > 0.0f || m.k[2] > 0.0f;
        s.transmission_tint = base == Vec3() ? Vec3::splat(1.0f) : base;
        s.relative_ior = front_face ? ior : 1.0f / ior;
        return s;
    }
    Vec3 fresnel(float c) const {
        return conductor ? fresnel_conductor(c, eta, k) : fresnel_schlick(f0, c);
    }
    Vec3 normal_reflectance() const { return conductor ? fresnel_conductor(1.0f, eta, k) : f0; }
    Vec3 specular_albedo(float cos_o) const {
        float e_ss = directional_albedo(roughness, std::fabs(cos_o));
        Vec3 f = fresnel(std::fabs(cos_o));
        Vec3 f_avg = fresnel_average(normal_reflectance());
        return (f * e_ss + f_avg * (1.0f - e_ss)).clamp(Vec3(), Vec3::splat(1.0f));
    }
    float specular_probability(float cos_o) const {
        if (transmission > 0.0f) {
            float f = fresnel_dielectric(std::fabs(cos_o), relative_ior);
            if (f >= 1.0f) return 1.0f;
            return clampf(f, 0.05f, 0.95f);
        }
        float spec = luminance(specular_albedo(cos_o));
        float diff = luminance(diffuse_albedo * (Vec3::splat(1.0f) - specular_albedo(cos_o)));
        if (spec + diff <= 0.0f) return 1.0f;
        return clampf(spec / (spec + diff), 0.1f, 0.9f);
    }
    Vec3 reflection_fresnel(float c) const {
        if (transmission > 0.0f && !conductor) return Vec3::splat(fresnel_dielectric(c, relative_ior));
        return fresnel(c);
    }
};

// dielectric module (bsdf.rs:597-695)
inline bool transmission_half_vector(Vec3 wo, Vec3 wi, float eta, Vec3& h) {
    Vec3 hh = (wo + eta * wi).normalize_or_zero();
    if (hh == Vec3()) return false;
    h = hh.z < 0.0f ? -hh : hh;
    return true;
}
inline float dielectric_eval(float alpha, float eta, Vec3 wo, Vec3 wi) {
    if (wo.z * wi.z >= 0.0f) return 0.0f;
    Vec3 h;
    if (!transmission_half_vector(wo, wi, eta, h)) return 0.0f;
    float wo_h = wo.dot(h), wi_h = wi.dot(h);
    if (wo_h <= 0.0f || wi_h >= 0.0f) return 0.0f;
    float denom = wo_h + eta * wi_h;
    if (std::fabs(denom) < 1.0e-9f) return 0.0f;
    float f = fresnel_dielectric(wo_h, eta);
    float d = ggx_d(alpha, std::fabs(h.z));
    float g2 = smith_g2(alpha, std::fabs(wo.z), std::fabs(wi.z));
    return ((1.0f - f) * d * g2 * std::fabs(wi_h * wo_h)) /
           (std::fabs(wo.z) * std::fabs(wi.z) * denom * denom);
}
inline float dielectric_pdf(float alpha, float eta, Vec3 wo, Vec3 wi) {
    if (wo.z * wi.z >= 0.0f) return 0.0f;
    Vec3 h;
    if (!transmission_half_vector(wo, wi, eta, h)) return 0.0f;
    float wo_h = wo.dot(h), wi_h = wi.dot(h);
    if (wo_h <= 0.0f || wi_h >= 0.0f) return 0.0f;
    float denom = wo_h + eta * wi_h;
    if (std::fabs(denom) < 1.0e-9f) return 0.0f;
    float jac = std::fabs(eta * eta * wi_h) / (denom * denom);
    return ggx_vndf_half_pdf(alpha, wo, h) * jac;
}

Vec3 surface_eval(const Surface& s, Vec3 wo, Vec3 wi);
float surface_pdf(const Surface& s, Vec3 wo, Vec3 wi);
BsdfSample surface_sample(const Surface& s, Vec3 wo, float u_lobe, Vec2 u);

// ---------------------------------------------------------------- light.rs
static const float MIN_COS_LIGHT = 1.0e-6f;
inline float power_heuristic(float a, float b) {  // light.rs:311-317
    if (a <= 0.0f) return 0.0f;
    float r = b / a;
    return 1.0f / (1.0f + r * r);
}
inline float light_pdf_from_geometry(uint32_t n, float area, Vec3 ln, Vec3 sp, Vec3 hp) {
    // light.rs:241-263
    if (n == 0 || area <= 0.0f) return 0.0f;
    Vec3 tl = hp - sp;
    float d2 = tl.length_squared();
    if (d2 <= 0.0f) return 0.0f;
    Vec3 wi = tl / std::sqrt(d2);
    float cl = ln.dot(-wi);
    if (cl <= MIN_COS_LIGHT) return 0.0f;
    float pa = 1.0f / ((float)n * area);
    return pa * d2 / cl;
}
std::vector<GpuLight> build_lights(const std::vector<GpuMaterial>& mats,
                                   const std::vector<GpuPrimitive>& prims,
                                   const std::vector<GpuTriangle>& tris,
                                   const std::vector<float>& positions4);

// ---------------------------------------------------------------- envmap.rs
struct EnvSample {
    Vec3 direction, radiance;
    float pdf;
};
struct EnvMap {
    uint32_t width = 0, height = 0;
    std::vector<float> pixels;       // 4 floats per texel
    std::vector<float> conditional;  // (w+1) * h
    std::vector<float> marginal;     // h+1
    float total_weight = 0.0f;

    bool is_empty() const { return pixels.empty() || total_weight <= 0.0f; }
    static Vec3 direction_from_uv(float u, float v);
    static Vec2 uv_from_direction(Vec3 d);
    static EnvMap build(uint32_t w, uint32_t h, std::vector<float> pixels);
    void texel_of(Vec2 uv, uint64_t& i, uint64_t& j) const;
    Vec3 radiance(Vec3 d) const;
    float pdf(Vec3 d) const;
    EnvSample sample(Vec2 u) const;
};
EnvMap procedural_sky(uint32_t w, uint32_t h, Vec3 sun_dir, float sun_intensity, float sun_radius_deg);

}  // namespace oracle
