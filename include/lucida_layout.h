/*
 * lucida_layout.h — the byte-layout contract shared by every layer.
 *
 * Each struct is a field-for-field, offset-for-offset restatement of the
 * `#[repr(C)]` types in Lucida's crates/core/src/gpu_layout.rs, so a Rust
 * caller can hand its `SceneBlob` arrays (bytemuck slices) across the C ABI
 * without any repacking. The static_asserts below mirror the offset tests in
 * gpu_layout.rs:993-1166.
 *
 * Plain C (C99/C11 and C++ compatible), no CUDA types.
 */
#ifndef LUCIDA_LAYOUT_H
#define LUCIDA_LAYOUT_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LUC_LAYOUT_VERSION 1u

/* gpu_layout.rs:44-74 — 80 bytes. */
typedef struct GpuMaterial {
    float base_color[3]; /* 0  */
    float metallic;      /* 12 */
    float emissive[3];   /* 16 */
    float roughness;     /* 28 */
    float ior;           /* 32 */
    float transmission;  /* 36 */
    float _pad0;         /* 40 */
    float _pad1;         /* 44 */
    float eta[3];        /* 48 */
    float _pad2;         /* 60 */
    float k[3];          /* 64 */
    float _pad3;         /* 76 */
} GpuMaterial;

/* gpu_layout.rs:172-174, 477 */
#define PRIM_KIND_SPHERE 0u
#define PRIM_KIND_QUAD 1u
#define PRIM_KIND_INSTANCE 2u

/* gpu_layout.rs:193-211 — 64 bytes. Spheres and parallelograms. */
typedef struct GpuPrimitive {
    float position[3]; /* 0  */
    float radius;      /* 12 */
    float edge_u[3];   /* 16 */
    uint32_t kind;     /* 28 */
    float edge_v[3];   /* 32 */
    uint32_t material; /* 44 */
    float normal[3];   /* 48 */
    float _pad0;       /* 60 */
} GpuPrimitive;

/* gpu_layout.rs:494-511 — 64 bytes, overlays GpuPrimitive. */
typedef struct GpuInstance {
    float inv_row0[3];        /* 0  */
    uint32_t blas_root;       /* 12 */
    float inv_row1[3];        /* 16 */
    uint32_t kind;            /* 28 */
    float inv_row2[3];        /* 32 */
    uint32_t material;        /* 44 */
    float inv_translation[3]; /* 48 */
    float _pad0;              /* 60 */
} GpuInstance;

/* gpu_layout.rs:254-261 — 32 bytes. */
typedef struct GpuVertexAttr {
    float normal[3]; /* 0  */
    float _pad0;     /* 12 */
    float uv[2];     /* 16 */
    float _pad1[2];  /* 24 */
} GpuVertexAttr;

/* gpu_layout.rs:268-275 — 16 bytes. */
typedef struct GpuTriangle {
    uint32_t i0, i1, i2, material;
} GpuTriangle;

/* gpu_layout.rs:296-305 — 32 bytes. count == 0: internal, right = left + 1. */
typedef struct GpuBvhNode {
    float bounds_min[3];
    uint32_t left_first;
    float bounds_max[3];
    uint32_t count;
} GpuBvhNode;

/* gpu_layout.rs:343-383 — 64 bytes. The HDR accumulator. */
typedef struct GpuAccum {
    float radiance[3];    /* 0  */
    float samples;        /* 12 */
    float albedo[3];      /* 16 */
    float depth;          /* 28 */
    float normal[3];      /* 32 */
    float traversal;      /* 44 */
    float radiance_sq[3]; /* 48 */
    float _pad0;          /* 60 */
} GpuAccum;

/* gpu_layout.rs:393-472 — 160 bytes. */
typedef struct GpuUniforms {
    float cam_origin[3];      /* 0   */
    float lens_radius;        /* 12  */
    float cam_upper_left[3];  /* 16  */
    float focus_distance;     /* 28  */
    float cam_horizontal[3];  /* 32  */
    float _pad1;              /* 44  */
    float cam_vertical[3];    /* 48  */
    float _pad2;              /* 60  */
    uint32_t width;           /* 64  */
    uint32_t height;          /* 68  */
    uint32_t sample_offset;   /* 72  */
    uint32_t samples_per_launch; /* 76 */
    uint32_t max_depth;       /* 80  */
    uint32_t frame_seed;      /* 84  */
    uint32_t num_primitives;  /* 88  */
    uint32_t num_lights;      /* 92  */
    float background[3];      /* 96  */
    uint32_t num_triangles;   /* 108 */
    uint32_t num_bvh_nodes;   /* 112 */
    uint32_t render_mode;     /* 116 */
    uint32_t sampling_mode;   /* 120 */
    uint32_t env_width;       /* 124 */
    uint32_t env_height;      /* 128 */
    float env_total_weight;   /* 132 */
    uint32_t sampler_kind;    /* 136 */
    uint32_t num_instances;   /* 140 */
    uint32_t tlas_root;       /* 144 */
    uint32_t _pad3, _pad4, _pad5; /* 148..160 */
} GpuUniforms;

/* gpu_layout.rs:540-542 */
#define LIGHT_KIND_QUAD 0u
#define LIGHT_KIND_TRIANGLE 1u

/* gpu_layout.rs:554-568 — 64 bytes. */
typedef struct GpuLight {
    float origin[3];   /* 0  */
    float area;        /* 12 */
    float edge_u[3];   /* 16 */
    uint32_t kind;     /* 28 */
    float edge_v[3];   /* 32 */
    uint32_t material; /* 44 */
    float normal[3];   /* 48 */
    float _pad0;       /* 60 */
} GpuLight;

/* integrator.rs:39-57 / SamplingMode::index */
#define LUC_SAMPLING_BSDF 0u
#define LUC_SAMPLING_NEE 1u
#define LUC_SAMPLING_MIS 2u
/* sobol.rs:244-278 / SamplerKind::index */
#define LUC_SAMPLER_INDEPENDENT 0u
#define LUC_SAMPLER_SOBOL 1u

#ifdef __cplusplus
} /* extern "C" */
#endif

#ifdef __cplusplus
#define LUC_STATIC_ASSERT static_assert
#else
#define LUC_STATIC_ASSERT _Static_assert
#endif
LUC_STATIC_ASSERT(sizeof(GpuMaterial) == 80, "GpuMaterial is 80 bytes");
LUC_STATIC_ASSERT(offsetof(GpuMaterial, emissive) == 16, "GpuMaterial.emissive");
LUC_STATIC_ASSERT(offsetof(GpuMaterial, ior) == 32, "GpuMaterial.ior");
LUC_STATIC_ASSERT(offsetof(GpuMaterial, eta) == 48, "GpuMaterial.eta");
LUC_STATIC_ASSERT(offsetof(GpuMaterial, k) == 64, "GpuMaterial.k");
LUC_STATIC_ASSERT(sizeof(GpuPrimitive) == 64, "GpuPrimitive is 64 bytes");
LUC_STATIC_ASSERT(offsetof(GpuPrimitive, kind) == 28, "GpuPrimitive.kind");
LUC_STATIC_ASSERT(offsetof(GpuPrimitive, material) == 44, "GpuPrimitive.material");
LUC_STATIC_ASSERT(offsetof(GpuPrimitive, normal) == 48, "GpuPrimitive.normal");
LUC_STATIC_ASSERT(sizeof(GpuInstance) == 64, "GpuInstance is 64 bytes");
LUC_STATIC_ASSERT(offsetof(GpuInstance, kind) == 28, "GpuInstance.kind overlays GpuPrimitive.kind");
LUC_STATIC_ASSERT(offsetof(GpuInstance, material) == 44, "GpuInstance.material");
LUC_STATIC_ASSERT(sizeof(GpuVertexAttr) == 32, "GpuVertexAttr is 32 bytes");
LUC_STATIC_ASSERT(offsetof(GpuVertexAttr, uv) == 16, "GpuVertexAttr.uv");
LUC_STATIC_ASSERT(sizeof(GpuTriangle) == 16, "GpuTriangle is 16 bytes");
LUC_STATIC_ASSERT(sizeof(GpuBvhNode) == 32, "GpuBvhNode is 32 bytes");
LUC_STATIC_ASSERT(offsetof(GpuBvhNode, left_first) == 12, "GpuBvhNode.left_first");
LUC_STATIC_ASSERT(offsetof(GpuBvhNode, count) == 28, "GpuBvhNode.count");
LUC_STATIC_ASSERT(sizeof(GpuAccum) == 64, "GpuAccum is 64 bytes");
LUC_STATIC_ASSERT(offsetof(GpuAccum, radiance_sq) == 48, "GpuAccum.radiance_sq");
LUC_STATIC_ASSERT(sizeof(GpuUniforms) == 160, "GpuUniforms is 160 bytes");
LUC_STATIC_ASSERT(offsetof(GpuUniforms, width) == 64, "GpuUniforms.width");
LUC_STATIC_ASSERT(offsetof(GpuUniforms, background) == 96, "GpuUniforms.background");
LUC_STATIC_ASSERT(offsetof(GpuUniforms, num_bvh_nodes) == 112, "GpuUniforms.num_bvh_nodes");
LUC_STATIC_ASSERT(offsetof(GpuUniforms, env_total_weight) == 132, "GpuUniforms.env_total_weight");
LUC_STATIC_ASSERT(offsetof(GpuUniforms, tlas_root) == 144, "GpuUniforms.tlas_root");
LUC_STATIC_ASSERT(sizeof(GpuLight) == 64, "GpuLight is 64 bytes");
LUC_STATIC_ASSERT(offsetof(GpuLight, normal) == 48, "GpuLight.normal");

#endif /* LUCIDA_LAYOUT_H */
