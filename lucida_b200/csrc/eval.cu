// Per-function device evaluation: run single device functions over host
// input arrays, the way Lucida's shader eval harness does for WGSL
// (crates/gpu/src/eval.rs, shaders/test/eval_bsdf.wgsl), so the BSDF and
// environment samplers can be diffed against the CPU twins function by
// function and chi-squared tested on the device's own samples.
#include "ctx.cuh"

namespace luc {

__global__ void k_eval_bsdf(GpuMaterial m, int front, const float* __restrict__ wo3, const float* __restrict__ in3,
                            uint32_t n, int mode, const float* __restrict__ energy, float* __restrict__ out_wi,
                            float* __restrict__ out_f, float* __restrict__ out_pdf) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Surface s = make_surface(m, front != 0);
    V3 wo = ld3(wo3 + 3 * i);
    if (mode == 0) {  // surface::sample(wo, u_lobe, u)
        BsdfSample b = bsdf_sample(s, energy, wo, in3[3 * i], in3[3 * i + 1], in3[3 * i + 2]);
        out_wi[3 * i] = b.wi.x; out_wi[3 * i + 1] = b.wi.y; out_wi[3 * i + 2] = b.wi.z;
        out_f[3 * i] = b.weight.x; out_f[3 * i + 1] = b.weight.y; out_f[3 * i + 2] = b.weight.z;
        out_pdf[i] = b.pdf;
    } else {  // surface::eval and surface::pdf at (wo, wi)
        V3 wi = ld3(in3 + 3 * i);
        V3 f = bsdf_eval(s, energy, wo, wi);
        out_f[3 * i] = f.x; out_f[3 * i + 1] = f.y; out_f[3 * i + 2] = f.z;
        out_pdf[i] = bsdf_pdf(s, energy, wo, wi);
    }
}

__global__ void k_eval_env(DevScene sc, const float* __restrict__ in, uint32_t n, int mode, float* __restrict__ dir3,
                           float* __restrict__ rad3, float* __restrict__ pdf) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (mode == 0) {  // EnvMap::sample(u)
        EnvSample e = env_sample(sc, in[2 * i], in[2 * i + 1]);
        dir3[3 * i] = e.dir.x; dir3[3 * i + 1] = e.dir.y; dir3[3 * i + 2] = e.dir.z;
        rad3[3 * i] = e.rad.x; rad3[3 * i + 1] = e.rad.y; rad3[3 * i + 2] = e.rad.z;
        pdf[i] = e.pdf;
    } else {  // EnvMap::radiance and EnvMap::pdf at a direction
        V3 d = ld3(in + 3 * i);
        V3 r = env_radiance(sc, d);
        rad3[3 * i] = r.x; rad3[3 * i + 1] = r.y; rad3[3 * i + 2] = r.z;
        pdf[i] = env_pdf(sc, d);
    }
}

}  // namespace luc

using namespace luc;

namespace {
template <class F>
int32_t with_device_io(luc_ctx* c, std::vector<std::pair<const void*, size_t>> in, std::vector<std::pair<void*, size_t>> out,
                       F launch) {
    size_t total = 0;
    for (auto& a : in) total += (a.second + 255) & ~size_t(255);
    for (auto& a : out) total += (a.second + 255) & ~size_t(255);
    DevBuf buf;
    LUC_CUDA(c, buf.ensure(total + 256), "alloc eval");
    std::vector<void*> din, dout;
    char* p = (char*)buf.p;
    cudaStream_t s = c->stream;
    for (auto& a : in) {
        if (a.second) cudaMemcpyAsync(p, a.first, a.second, cudaMemcpyHostToDevice, s);
        din.push_back(p);
        p += (a.second + 255) & ~size_t(255);
    }
    for (auto& a : out) {
        dout.push_back(p);
        p += (a.second + 255) & ~size_t(255);
    }
    launch(din, dout);
    cudaError_t e = cudaGetLastError();
    for (size_t k = 0; k < out.size() && e == cudaSuccess; ++k)
        if (out[k].second) e = cudaMemcpyAsync(out[k].first, dout[k], out[k].second, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    buf.release();
    if (e != cudaSuccess) return luc_cuda_fail(c, e, "eval");
    return LUC_OK;
}
}  // namespace

extern "C" int32_t luc_eval_bsdf(luc_ctx* c, const GpuMaterial* m, int32_t front, const float* wo3, const float* in3,
                                 uint32_t n, int32_t mode, float* out_wi3, float* out_f3, float* out_pdf) {
    if (!c || !m || (n && (!wo3 || !in3 || !out_f3 || !out_pdf || (mode == 0 && !out_wi3))))
        return LUC_ERR_VALIDATION;
    if (mode != 0 && mode != 1) return luc_fail(c, LUC_ERR_VALIDATION, "mode must be 0 (sample) or 1 (eval)");
    cudaSetDevice(c->device);
    if (n == 0) return LUC_OK;
    size_t v3 = (size_t)n * 12, v1 = (size_t)n * 4;
    GpuMaterial mat = *m;
    const float* energy = c->energy.as<float>();
    return with_device_io(c, {{wo3, v3}, {in3, v3}}, {{out_wi3, mode == 0 ? v3 : 0}, {out_f3, v3}, {out_pdf, v1}},
                          [&](std::vector<void*>& din, std::vector<void*>& dout) {
                              k_eval_bsdf<<<(n + 127) / 128, 128, 0, c->stream>>>(
                                  mat, front, (const float*)din[0], (const float*)din[1], n, mode, energy,
                                  (float*)dout[0], (float*)dout[1], (float*)dout[2]);
                          });
}

extern "C" int32_t luc_eval_env(luc_ctx* c, const float* in, uint32_t n, int32_t mode, float* dir3, float* rad3,
                                float* pdf) {
    if (!c || (n && (!in || !rad3 || !pdf || (mode == 0 && !dir3)))) return LUC_ERR_VALIDATION;
    if (mode != 0 && mode != 1) return luc_fail(c, LUC_ERR_VALIDATION, "mode must be 0 (sample) or 1 (lookup)");
    if (!c->has_scene || !c->scene.has_env) return luc_fail(c, LUC_ERR_VALIDATION, "no environment map resident");
    cudaSetDevice(c->device);
    if (n == 0) return LUC_OK;
    size_t v3 = (size_t)n * 12, v1 = (size_t)n * 4, vin = (size_t)n * (mode == 0 ? 8 : 12);
    DevScene sc = c->scene;
    return with_device_io(c, {{in, vin}}, {{dir3, mode == 0 ? v3 : 0}, {rad3, v3}, {pdf, v1}},
                          [&](std::vector<void*>& din, std::vector<void*>& dout) {
                              k_eval_env<<<(n + 127) / 128, 128, 0, c->stream>>>(
                                  sc, (const float*)din[0], n, mode, (float*)dout[0], (float*)dout[1],
                                  (float*)dout[2]);
                          });
}

// Ray queries against the resident scene: Scene::intersect (scene.rs:452-527)
// for mode 0, Scene::occluded (scene.rs:577-606) for mode 1, through the same
// traversal the integrator uses (wide tree, binary tree or instances).
namespace luc {
__global__ void k_intersect(const __grid_constant__ DevScene sc, const float* __restrict__ rays, uint32_t n,
                           int32_t mode, float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = rays + 8 * (size_t)i;
    const V3 o{r[0], r[1], r[2]}, d{r[4], r[5], r[6]};
    TravCount tc;
    if (mode == 0) {
        float t, u, v;
        uint32_t inst;
        const uint32_t id = sc.num_instances ? closest_hit<true>(sc, o, d, t, u, v, inst, tc)
                                             : closest_hit<false>(sc, o, d, t, u, v, inst, tc);
        reinterpret_cast<float4*>(out)[i] = make_float4(t, u, v, __uint_as_float(id));
    } else {
        const bool occ = sc.num_instances ? occluded<true>(sc, o, d, r[3], tc) : occluded<false>(sc, o, d, r[3], tc);
        reinterpret_cast<uint32_t*>(out)[i] = occ ? 1u : 0u;
    }
}
}  // namespace luc

extern "C" int32_t luc_intersect(luc_ctx* c, const float* rays8, uint32_t n, int32_t mode, void* out) {
    using namespace luc;
    if (!c || (n && (!rays8 || !out))) return LUC_ERR_VALIDATION;
    if (mode != 0 && mode != 1) return luc_fail(c, LUC_ERR_VALIDATION, "mode must be 0 (closest hit) or 1 (occluded)");
    if (!c->has_scene) return luc_fail(c, LUC_ERR_VALIDATION, "no scene uploaded");
    cudaSetDevice(c->device);
    if (n == 0) return LUC_OK;
    DevScene sc = c->scene;
    return with_device_io(c, {{rays8, (size_t)n * 32}}, {{out, (size_t)n * (mode == 0 ? 16 : 4)}},
                          [&](std::vector<void*>& din, std::vector<void*>& dout) {
                              k_intersect<<<(n + 127) / 128, 128, 0, c->stream>>>(sc, (const float*)din[0], n, mode,
                                                                                  (float*)dout[0]);
                          });
}

