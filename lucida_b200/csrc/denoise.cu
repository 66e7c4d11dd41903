// Edge-avoiding a-trous denoiser (placeholder until the device filter lands).
#include "ctx.cuh"
int32_t luc_denoise_device(luc_ctx* c, const GpuAccum*, uint32_t, uint32_t, const luc_denoise_params*, GpuAccum*) { return luc_fail(c, LUC_ERR_VALIDATION, "denoiser not available"); }
extern "C" int32_t luc_denoise(luc_ctx* c, const GpuAccum*, uint32_t, uint32_t, const luc_denoise_params*, GpuAccum*) { return luc_fail(c, LUC_ERR_VALIDATION, "denoiser not available"); }
