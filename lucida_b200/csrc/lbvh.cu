// GPU LBVH builder (placeholder until the device builder lands).
#include "ctx.cuh"
int32_t luc_lbvh_device(luc_ctx* c, uint32_t, uint32_t*) { return luc_fail(c, LUC_ERR_VALIDATION, "LBVH builder not available"); }
int32_t luc_triangle_boxes_device(luc_ctx* c, const GpuTriangle*, const float4*, uint32_t) { return luc_fail(c, LUC_ERR_VALIDATION, "LBVH builder not available"); }
int32_t luc_radix_sort_device(luc_ctx* c, uint32_t) { return luc_fail(c, LUC_ERR_VALIDATION, "sort not available"); }
int32_t luc_gather_triangles(luc_ctx* c, const GpuTriangle*, GpuTriangle*, const uint32_t*, uint32_t) { return luc_fail(c, LUC_ERR_VALIDATION, "LBVH builder not available"); }
extern "C" {
int32_t luc_lbvh_build(luc_ctx* c, const GpuTriangle*, uint32_t, const float*, uint32_t, luc_lbvh_out*) { return luc_fail(c, LUC_ERR_VALIDATION, "LBVH builder not available"); }
int32_t luc_lbvh_build_boxes(luc_ctx* c, const float*, uint32_t, luc_lbvh_out*) { return luc_fail(c, LUC_ERR_VALIDATION, "LBVH builder not available"); }
int32_t luc_sort_u32(luc_ctx* c, const uint32_t*, const uint32_t*, uint32_t, uint32_t*, uint32_t*) { return luc_fail(c, LUC_ERR_VALIDATION, "sort not available"); }
int32_t luc_sort_u32_dev(luc_ctx* c, void*, void*, uint32_t) { return luc_fail(c, LUC_ERR_VALIDATION, "sort not available"); }
}
