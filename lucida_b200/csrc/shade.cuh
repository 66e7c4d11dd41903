// One path vertex (crates/core/src/integrator.rs:227-400): escaped rays,
// emission with MIS, first-hit guides, next event estimation (the light
// sample and its shadow ray) and BSDF sampling (or the learned mixture in
// guided frames). Shared by the wavefront's SHADE, which loads the path from
// the pool and stores the result, and the megakernel, which keeps the path
// in registers, so both architectures run one copy of the shading logic.
#pragma once

#include "render.cuh"

namespace luc {

// GENERATE's camera ray (shaders/wavefront/generate.wgsl:35-88;
// camera.rs:373-405): jittered pixel position, then the thin-lens offset.
// The sampler must be fresh for (pixel, sample); it advances by two pairs.
LUC_D void camera_ray(const FrameParams& fp, uint32_t pixel, Sampler& smp, V3& origin, V3& dir) {
    uint32_t x = pixel % fp.width, y = pixel / fp.width;
    float pu, pv, lu, lv;
    smp.next_vec2(pu, pv);
    smp.next_vec2(lu, lv);
    float s = ((float)x + pu) / (float)fp.width;
    float t = ((float)y + pv) / (float)fp.height;
    origin = fp.cam_origin;
    V3 target = fp.cam_upper_left + s * fp.cam_horizontal + t * fp.cam_vertical;
    if (fp.lens_radius <= 0.0f) {
        dir = normalize(target - origin);
    } else {
        float dx, dy;
        concentric_disk(lu, lv, dx, dy);
        dx = dx * fp.lens_radius;
        dy = dy * fp.lens_radius;
        V3 right = normalize(fp.cam_horizontal), down = normalize(fp.cam_vertical);
        origin = origin + (right * dx + down * dy);
        dir = normalize(target - origin);
    }
}

// What a vertex produces goes to a sink, at the point it is computed (so the
// wavefront's stores happen where the values are live, as in a hand-written
// kernel). A sink provides:
//   V3 prev()                                    the previous vertex (only
//                                                read for the MIS weight of an
//                                                emitter hit)
//   void guides(V3 albedo, float depth, V3 normal)   first-hit guides
//   void shadow(V3 o, V3 d, float t_max, V3 contribution)   NEE shadow ray
//   void next(V3 origin, V3 dir, float pdf, V3 thr, V3 hit_position,
//             V3 hit_normal, bool record, V3 rad)     the path continues
// kSkyMis: MIS sampling in a scene lit only by its environment map (no
// emitter list; the caller checks), with the code of the other cases
// compiled out of the vertex.
// `h4` is the closest-hit record (t, u, v, id bits) and `inst` its instance;
// `rad` is updated in place (the return value says whether it changed);
// `lob` / `lobe_stride` locate the path's guide mixture (guided frames). The
// sampler advances in place.
// An escaped ray (integrator.rs:228-263): the environment through its MIS
// weight (full credit at depth 0 and for BSDF-only sampling, none for
// NEE-only), or the background. `rad` is updated in place; the return value
// says whether it changed. SHADE runs it for a miss; split frames run it in
// k_escape for the escaped queue.
template <bool kSkyMis>
LUC_D bool escape_vertex(const DevScene& sc, const FrameParams& fp, uint32_t depth, V3 dir, V3 thr, V3& rad,
                         float prev_pdf) {
    const uint32_t sampling = kSkyMis ? LUC_SAMPLING_MIS : fp.sampling;
    if (kSkyMis || sc.has_env) {
        float epdf;
        V3 l = env_radiance_pdf(sc, dir, epdf);
        float weight;
        if (depth == 0 || sampling == LUC_SAMPLING_BSDF) weight = 1.0f;
        else if (sampling == LUC_SAMPLING_NEE) weight = 0.0f;
        else {
            uint32_t total = max(sc.light_strategies, 1u);
            weight = power_heuristic(prev_pdf, epdf / (float)total);
        }
        if (weight > 0.0f) {
            rad = rad + thr * l * weight;
            return true;
        }
        return false;
    }
    rad = rad + thr * sc.background;
    return true;
}

template <bool kGuided, bool kInst, bool kSkyMis = false, typename Sink>
LUC_D bool shade_vertex(const DevScene& sc, const FrameParams& fp, uint32_t depth, Sampler& smp, V3 org, V3 dir,
                        V3 thr, V3& rad, float prev_pdf, float4 h4, uint32_t inst, const float4* lob,
                        uint32_t lobe_stride, Sink& sink) {
    const bool last = depth + 1 >= fp.max_depth;
    const uint32_t sampling = kSkyMis ? LUC_SAMPLING_MIS : fp.sampling;
    const uint32_t id = __float_as_uint(h4.w);
    bool rad_changed = false;
    if (id == kMiss) return escape_vertex<kSkyMis>(sc, fp, depth, dir, thr, rad, prev_pdf);
    const SurfaceHit hit = surface_hit_t<kInst>(sc, id, inst, h4.x, h4.y, h4.z, org, dir);
    const GpuMaterial m = sc.materials[hit.material];
    const V3 emissive = ld3(m.emissive);
    // Emission with MIS (integrator.rs:271-309).
    if (hit.front && max_elem(emissive) > 0.0f) {
        float weight;
        if (depth == 0 || sampling == LUC_SAMPLING_BSDF) weight = 1.0f;
        else if (sampling == LUC_SAMPLING_NEE) weight = 0.0f;
        else {
            uint32_t n = kSkyMis ? 0u : sc.num_lights, total = sc.light_strategies;
            float pdf_light = 0.0f;
            if (n != 0 && hit.light_area > 0.0f) {  // light.rs:241-263
                const V3 prev = sink.prev();
                V3 tl = hit.position - prev;
                float d2 = dot(tl, tl);
                if (d2 > 0.0f) {
                    V3 wi = tl / sqrtf(d2);
                    float cl = dot(hit.gnormal, -wi);
                    if (cl > 1.0e-6f) pdf_light = 1.0f / ((float)n * hit.light_area) * d2 / cl;
                }
            }
            pdf_light = pdf_light * ((float)n / (float)max(total, 1u));
            weight = power_heuristic(prev_pdf, pdf_light);
        }
        if (weight > 0.0f) {
            rad = rad + thr * emissive * weight;
            rad_changed = true;
        }
    }
    const Surface surf = make_surface(m, hit.front);
    if (depth == 0 && fp.guides)
        sink.guides(vmax(surf.diffuse_albedo + surf.f0 + emissive, splat(1.0e-3f)), h4.x, hit.normal);
    const V3 wo = to_local(-dir, hit.normal);
    const bool gv = kGuided && fp.guided && !last && surf.transmission <= 0.0f && surf.roughness >= kGuideMinRoughness;
    if (!(wo.z > 0.0f)) return rad_changed;
    // Everything surface::eval / pdf / sample take from wo alone.
    const SurfWo sw = surf_wo(surf, sc.energy, wo.z);
    // Next event estimation (integrator.rs:349-354, 418-532): the light
    // sample and its direction; f and pdf below.
    bool nee = false;
    V3 wiw{0, 0, 0}, lrad{0, 0, 0}, wi_n{0.0f, 0.0f, 1.0f};
    float dist = 0.0f, lpdf = 0.0f;
    if ((sampling == LUC_SAMPLING_NEE || sampling == LUC_SAMPLING_MIS) && !last && sc.light_strategies > 0) {
        float u_sel = smp.next_f32();
        float ua, ub;
        smp.next_vec2(ua, ub);
        uint32_t nl = kSkyMis ? 0u : sc.num_lights, total = sc.light_strategies;
        uint32_t pick = min(f2u(u_sel * (float)total), total - 1u);
        bool ok = true;
        if (pick < nl) {
            float u_light = ((float)pick + 0.5f) / (float)nl;
            uint32_t idx = min(f2u(u_light * (float)nl), nl - 1u);
            const GpuLight L = sc.lights[idx];
            V3 lo = ld3(L.origin), eu = ld3(L.edge_u), ev = ld3(L.edge_v);
            V3 point;
            if (L.kind == LIGHT_KIND_TRIANGLE) {
                float su = sqrtf(ua);
                float b1 = 1.0f - su, b2 = ub * su;
                point = lo + b1 * eu + b2 * ev;
            } else {
                point = lo + ua * eu + ub * ev;
            }
            V3 tl = point - hit.position;
            float d2 = dot(tl, tl);
            if (d2 <= 0.0f) ok = false;
            else {
                dist = sqrtf(d2);
                wiw = tl / dist;
                float cl = dot(ld3(L.normal), -wiw);
                if (cl <= 1.0e-6f) ok = false;
                else {
                    float pa = 1.0f / ((float)nl * L.area);
                    float pw = pa * d2 / cl;
                    if (!isfinite(pw) || pw <= 0.0f) ok = false;
                    else {
                        lrad = ld3(sc.materials[L.material].emissive);
                        lpdf = pw * ((float)nl / (float)total);
                    }
                }
            }
        } else {
            EnvSample es = env_sample(sc, ua, ub);
            if (es.pdf <= 0.0f) ok = false;
            else {
                wiw = es.dir;
                lrad = es.rad;
                dist = __int_as_float(0x7f800000);
                lpdf = es.pdf / (float)total;
            }
        }
        if (ok && lpdf > 0.0f) {
            wi_n = to_local(wiw, hit.normal);
            nee = !(wi_n.z == 0.0f || (wi_n.z < 0.0f && surf.transmission <= 0.0f));
        }
    }
    // BSDF sampling (integrator.rs:360-399): the direction. Skipped on the
    // last bounce, where its result would never be read. Guided frames choose
    // between the BSDF and the learned mixture; the choice dimension is drawn
    // only where the guide applies.
    bool bsd = false;
    V3 wl{0.0f, 0.0f, 1.0f}, wd{0.0f, 0.0f, 1.0f};
    if (!last) {
        const float u_choice = kGuided && gv ? smp.next_f32() : 0.0f;
        const float u_lobe = smp.next_f32();
        float ux, uy;
        smp.next_vec2(ux, uy);
        if (!gv || u_choice < 0.5f) {
            bsd = bsdf_sample_dir_w(surf, sw, wo, u_lobe, ux, uy, wl);
            wd = to_world(wl, hit.normal);
        } else {
            wd = mixture_sample_mem(lob, lobe_stride, u_lobe, ux, uy);
            wl = to_local(wd, hit.normal);
            bsd = !(wl.z == 0.0f || (wl.z < 0.0f && surf.transmission <= 0.0f));
        }
    }
    // f and pdf at both directions through one copy of the BSDF code (the
    // loop is kept rolled on purpose: it halves the instruction footprint).
    V3 f_n{0.0f, 0.0f, 0.0f}, f_b{0.0f, 0.0f, 0.0f};
    float p_n = 0.0f, p_b = 0.0f;
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
        if (!(k == 0 ? nee : bsd)) continue;
        const V3 wi = k == 0 ? wi_n : wl;
        const V3 f = bsdf_eval_w(surf, sw, wo, wi);
        float pdf = 0.0f;
        if (k == 1 || (sampling == LUC_SAMPLING_MIS && max_elem(f) > 0.0f)) pdf = bsdf_pdf_w(surf, sw, wo, wi);
        if (k == 0) {
            f_n = f;
            p_n = pdf;
        } else {
            f_b = f;
            p_b = pdf;
        }
    }
    if (nee && max_elem(f_n) > 0.0f) {
        float mis = 1.0f;
        if (sampling == LUC_SAMPLING_MIS) {
            float pb = p_n;
            if (gv) pb = 0.5f * pb + 0.5f * mixture_pdf_mem(lob, lobe_stride, wiw);
            mis = power_heuristic(lpdf, pb);
        }
        if (mis > 0.0f)
            sink.shadow(offset_ray_origin(hit.position, wi_n.z < 0.0f ? -hit.gnormal : hit.gnormal), wiw,
                        dist * (1.0f - 1.0e-3f), thr * (f_n * fabsf(wi_n.z) * lrad * (mis / lpdf)));
    }
    V3 nthr{0.0f, 0.0f, 0.0f};
    float npdf = 0.0f;
    if (kGuided && !last) {
        const V3 fc = bsd ? f_b * fabsf(wl.z) : splat(0.0f);
        if (max_elem(fc) > 0.0f) {
            npdf = gv ? 0.5f * p_b + 0.5f * mixture_pdf_mem(lob, lobe_stride, wd) : p_b;
            if (npdf > 0.0f) nthr = thr * (fc / npdf);
        }
    } else if (!kGuided && bsd && p_b > 0.0f) {
        npdf = p_b;
        nthr = thr * (f_b * (fabsf(wl.z) / p_b));  // surface::sample's weight f |cos| / pdf
    }
    if (max_elem(nthr) > 0.0f)
        sink.next(offset_ray_origin(hit.position, wl.z < 0.0f ? -hit.gnormal : hit.gnormal), wd, npdf, nthr,
                  hit.position, hit.normal, gv && fp.rec_cap, rad);
    return rad_changed;
}

}  // namespace luc
