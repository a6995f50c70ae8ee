// vpt_trackers.cuh - free-path samplers of the tracer, one device function per VptMode.
//
// Each function follows one reference shader (cited per function) and consumes random numbers in
// exactly the same order, so a path traced here and the same path traced by the CPU oracle take
// the same decisions.  Grid access goes through a sampler object `S` with
//     float operator()(F3 world_pos, Rng& rng)   -> normalised density at world_pos
// so the dense texture and the NanoVDB tree share the trackers.
#pragma once
#include "vpt_device.cuh"
#include "vpt_sparse.cuh"

namespace vpt {

struct FirstEvent {
    bool has;
    F3 x;
    float depth;
    float density;
    F3 w;         // direction after the first scatter (0 when the first event is an absorption)
    float pdf_w;  // phase-function density of that direction (firstEvent.pdf_w)
    bool iso;     // CLOSE_ISOSURFACES: the first event is a surface hit, whose normal is n
    F3 n;
};

struct PathCtx {
    uint32_t steps;      // tentative collisions + supervoxel steps of this path (guard)
    uint32_t max_steps;  // TraceParams::max_steps
    uint32_t lookups;    // density lookups of this path
    bool guard_hit;
};

VPT_DEV bool guard(PathCtx& pc) {
    if (++pc.steps > pc.max_steps) {
        pc.guard_hit = true;
        return true;
    }
    return false;
}

VPT_DEV float free_path(Rng& rng, float inv_majorant) {
    return -m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) * inv_majorant;
}

// A first event without a sampled direction: First W is (w_first, 0), the zero vector for absorptions
// in delta and spectral tracking (DeltaTracking.glsl:118-119, 276-277), the direction of travel for
// absorptions in next event tracking (NextEventTracking.glsl:290-291) and the reflected direction at an
// isosurface hit (CheckIsosurfaceHit.glsl:39-40).
VPT_DEV void record_event(FirstEvent& fe, F3 x, float density, float extinction, float depth,
                          F3 w_first = F3{0.0f, 0.0f, 0.0f}) {
    if (!fe.has) {
        fe.has = true;
        fe.x = x;
        fe.density = density * extinction;
        fe.depth = depth;
        fe.w = w_first;
        fe.pdf_w = 0.0f;
    }
}

// A scatter event: records the first event with the scattered direction w_out and its phase-function
// density (DeltaTracking.glsl:134-141; evaluated for the sampled pair of directions).
VPT_DEV void record_scatter(FirstEvent& fe, F3 x, float density, float extinction, float depth, F3 w_in, F3 w_out,
                            float g) {
    if (!fe.has) {
        record_event(fe, x, density, extinction, depth);
        fe.w = w_out;
        fe.pdf_w = evaluate_phase(g, w_in, w_out);
    }
}

// ---------------------------------------------------------------------------------------------
// Analog delta (Woodcock) tracking: absorb with P_a, scatter with P_s, null collision otherwise;
// escape radiance = sky + sun lobe (deltaTracking, DeltaTracking.glsl:168-344).
template <class S>
VPT_DEV F3 track_delta(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, FirstEvent& fe, PathCtx& pc) {
    float tmin, tmax;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        x = x + w * tmin;
        float d = tmax - tmin;
        int bounces = 0;
        while (true) {
            if (guard(pc)) return f3(0.0f, 0.0f, 0.0f);
            float t = free_path(rng, P.inv_extinction);
            if (t > d) break;
            F3 xn = x + w * t;
            float density = sample(xn, rng);
            pc.lookups++;
            x = xn;
            float xi = rng_next(rng);
            if (xi < P.absorb_albedo * density) {
                record_event(fe, x, density, P.extinction, tmax - d + t);
                // USE_TRANSFER_FUNCTION (DeltaTracking.glsl:293-301): the table's emission
                return P.tf ? sample.tf_emission() : f3(0.0f, 0.0f, 0.0f);
            }
            if (xi < density) {
                if (P.max_bounces > 0 && ++bounces > P.max_bounces) return f3(0.0f, 0.0f, 0.0f);
                const F3 w_in = w;
                w = sample_phase(rng, P.g, w);
                record_scatter(fe, x, density, P.extinction, tmax - d + t, w_in, w, P.g);
                if (ray_box_p(P, x, w, tmin, tmax)) {
                    x = x + w * tmin;
                    d = tmax - tmin;
                }
            } else {
                d -= t;
            }
        }
    }
    return sky_and_sun(P, w);
}

// One free-flight segment [x, x_new] of delta tracking with isosurfaces (CheckIsosurfaceHit.glsl):
// P.iso_subdivisions check points for a sign change of sampleCloudIso - iso_value (the density, or the
// filtered gradient magnitude for gradient isosurfaces) against the first point
// after the last surface event; a crossing is bisected (refineIsoSurfaceHit, VptUtils.glsl:1045-1058,
// 8 steps), the surface reflects (iso_scatter), the path moves 1e-4 off it and restarts from the box
// boundary.  Returns true on a surface event (x, w, d, tmax and weights updated; the first event
// recorded when `fe` is given).  The last check point is x_new itself (a1 = 1: x * 0 + x_new), whose
// density was just looked up: for a repeatable sampler (trilinear, dense, no transfer function: no
// random number drawn) that value is reused; any other sampler looks it up again, as the reference
// does, so that its random stream stays the reference's.
template <class S>
VPT_DEV void iso_surface_nee(const TraceParams& P, S& sample, Rng& rng, F3 x, const IsoFrame& fr,
                             const IsoBrdfSample& bs, F3 thr, F3& color, PathCtx& pc);

// With CLOSE_ISOSURFACES (`outside` given, true until the path's first check point): on that first point
// outside the volume counts as sign(-iso_value), so a path entering the box inside a surface meets the
// closing surface there, whose normal is the face entered from the camera position `cam`
// (rayBoxIntersectionNormal); the surface normal is kept in the first event for the normal map.
template <bool NEE = false, class S>
VPT_DEV bool iso_segment(const TraceParams& P, S& sample, Rng& rng, F3& x, F3 xn, float density, F3& w, float& d,
                         float& tmax, F3& weights, float& last_sign, bool& first_point, uint32_t& lookups,
                         FirstEvent* fe, F3* nee_color = nullptr, PathCtx* pc = nullptr, bool* outside = nullptr,
                         F3 cam = F3{0.0f, 0.0f, 0.0f}) {
    const int nsub = P.iso_subdivisions;
    for (int sub = 0; sub < nsub; ++sub) {
        const float a0 = (float)sub / (float)nsub, a1 = (float)(sub + 1) / (float)nsub;
        F3 x0 = x * (1.0f - a0) + xn * a0;
        F3 x1 = x * (1.0f - a1) + xn * a1;
        float v = density;
        if (P.iso_grad) {
            v = iso_gradient_at(P, x1);
            lookups++;
        } else if (sub != nsub - 1 || !S::kRepeatable) {
            v = sample(x1, rng);
            lookups++;
        }
        const float v_minus = v - P.iso_value;
        const float cur_sign = v_minus > 0.0f ? 1.0f : (v_minus < 0.0f ? -1.0f : 0.0f);
        const bool from_outside = outside && *outside;
        if (from_outside) {
            first_point = false;
            last_sign = -P.iso_value > 0.0f ? 1.0f : (-P.iso_value < 0.0f ? -1.0f : 0.0f);
        } else if (first_point) {
            first_point = false;
            last_sign = cur_sign;
        }
        if (last_sign != cur_sign) {
            for (int r = 0; r < 8; ++r) {
                const F3 mid = f3((x1.x + x0.x) * 0.5f, (x1.y + x0.y) * 0.5f, (x1.z + x0.z) * 0.5f);
                const float vm = P.iso_grad ? iso_gradient_at(P, mid) : sample(mid, rng);
                lookups++;
                if ((vm - P.iso_value) * cur_sign >= 0.0f) x1 = mid;
                else x0 = mid;
            }
            x = x1;
            IsoFrame fr;
            const IsoBrdfSample bs = iso_sample(P, rng, x, w, fr, from_outside ? &cam : nullptr);
            if constexpr (NEE) {  // USE_ISOSURFACE_NEE: the light sample before the throughput takes the BRDF
                iso_surface_nee(P, sample, rng, x, fr, bs, weights, *nee_color, *pc);
            }
            weights = f3(weights.x * bs.value.x, weights.y * bs.value.y, weights.z * bs.value.z);
            w = bs.dir;
            x = x + w * 1e-4f;
            first_point = true;
            if (outside) *outside = false;
            // firstEvent of a surface hit: density = extinction, depth = tMax - d + |x - x1|
            if (fe) {
                if (!fe->has && outside) {
                    fe->iso = true;
                    fe->n = fr.n;
                }
                record_event(*fe, x, 1.0f, P.extinction, tmax - d + length3(x1 - x), w);
            }
            float tmin;
            if (ray_box_p(P, x, w, tmin, tmax)) {
                x = x + w * tmin;
                d = tmax - tmin;
            }
            return true;
        }
        if (outside) *outside = false;
    }
    return false;
}

// Delta tracking with isosurfaces (DeltaTracking.glsl:168-344 with CheckIsosurfaceHit.glsl): every
// free-flight segment goes through iso_segment; escapes carry the surface throughput; weights below
// 1e-3 in every channel end the path after a surface event; the 1000th loop iteration ends the path
// with zero.  Trilinear lookups (the reference forces them with isosurfaces).
template <class S>
VPT_DEV F3 track_delta_iso(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, FirstEvent& fe, PathCtx& pc) {
    const F3 cam = x;  // cameraPosition (Clouds.glsl:99)
    bool outside = P.iso_close != 0;
    F3 weights = f3(1.0f, 1.0f, 1.0f);
    float last_sign = 0.0f;
    bool first_point = true;
    int it = 0;
    float tmin, tmax;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        x = x + w * tmin;
        float d = tmax - tmin;
        int bounces = 0;
        while (true) {
            if (++it == 1000) return f3(0.0f, 0.0f, 0.0f);
            if (guard(pc)) return f3(0.0f, 0.0f, 0.0f);
            float t = free_path(rng, P.inv_extinction);
            if (t > d) break;
            F3 xn = x + w * t;
            float density = sample(xn, rng);
            pc.lookups++;
            if (iso_segment(P, sample, rng, x, xn, density, w, d, tmax, weights, last_sign, first_point, pc.lookups,
                            &fe, nullptr, nullptr, P.iso_close ? &outside : nullptr, cam)) {
                if (weights.x < 1e-3f && weights.y < 1e-3f && weights.z < 1e-3f) return f3(0.0f, 0.0f, 0.0f);
                continue;
            }
            x = xn;
            float xi = rng_next(rng);
            if (xi < P.absorb_albedo * density) {
                record_event(fe, x, density, P.extinction, tmax - d + t);
                return f3(0.0f, 0.0f, 0.0f);
            }
            if (xi < density) {
                if (P.max_bounces > 0 && ++bounces > P.max_bounces) return f3(0.0f, 0.0f, 0.0f);
                const F3 w_in = w;
                w = sample_phase(rng, P.g, w);
                record_scatter(fe, x, density, P.extinction, tmax - d + t, w_in, w, P.g);
                if (ray_box_p(P, x, w, tmin, tmax)) {
                    x = x + w * tmin;
                    d = tmax - tmin;
                }
            } else {
                d -= t;
            }
        }
    }
    return weights * sky_and_sun(P, w);
}

// VptMode::RATIO_TRACKING: delta tracking that never absorbs and weights each real collision by
// the single-scattering albedo (ratioTracking, RatioTracking.glsl:26-95).
template <class S>
VPT_DEV F3 track_ratio(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, FirstEvent& fe, PathCtx& pc) {
    float trans = 1.0f;
    float tmin, tmax;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        x = x + w * tmin;
        float d = tmax - tmin;
        int bounces = 0;
        while (true) {
            if (guard(pc)) return f3(0.0f, 0.0f, 0.0f);
            float t = free_path(rng, P.inv_extinction);
            if (t > d) break;
            x = x + w * t;
            float density = sample(x, rng);
            pc.lookups++;
            float xi = rng_next(rng);
            if (xi < density) {
                if (P.max_bounces > 0 && ++bounces > P.max_bounces) return f3(0.0f, 0.0f, 0.0f);
                float pa = P.absorb_albedo * density;
                float ps = P.albedo * density;
                trans *= 1.0f - pa / (pa + ps);
                const F3 w_in = w;
                w = sample_phase(rng, P.g, w);
                if (!fe.has) {  // RatioTracking.glsl:75-81: no density or depth recorded
                    fe.has = true;
                    fe.x = x;
                    fe.density = 0.0f;
                    fe.depth = 0.0f;
                    fe.w = w;
                    fe.pdf_w = evaluate_phase(P.g, w_in, w);
                }
                if (ray_box_p(P, x, w, tmin, tmax)) {
                    x = x + w * tmin;
                    d = tmax - tmin;
                }
            } else {
                d -= t;
            }
        }
    }
    return sky_and_sun(P, w) * trans;
}

// Ratio-tracking transmittance toward the light (calculateTransmittance without occupancy grid,
// NeeTransmittance.glsl:5-119; T *= P_n = 1 - density per tentative collision).
template <class S>
VPT_DEV float shadow_transmittance(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, PathCtx& pc) {
    float trans = 1.0f;
    float tmin, tmax;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        x = x + w * tmin;
        float d = tmax - tmin;
        while (true) {
            if (guard(pc)) return 0.0f;
            float t = free_path(rng, P.inv_extinction);
            if (t > d) break;
            F3 xn = x + w * t;
            float density = sample(xn, rng);
            pc.lookups++;
            x = xn;
            trans *= 1.0f - density;
            d -= t;
        }
    }
    return trans;
}

// Shadow rays with isosurfaces (calculateTransmittance, NeeTransmittance.glsl:5-119, after the
// `#define USE_TRANSMITTANCE_DELTA_TRACKING` of its isosurface block): a delta-tracked 0/1 estimate,
// 0 at the first tentative collision that is real.  The reference also bisects every isosurface
// crossing on the way; without ISOSURFACE_USE_TF that changes neither the ray nor the random stream
// (trilinear lookups draw no random number), so the crossings are not looked for here.
template <class S>
VPT_DEV float shadow_transmittance_delta(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, PathCtx& pc) {
    float tmin, tmax;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        x = x + w * tmin;
        float d = tmax - tmin;
        while (true) {
            if (guard(pc)) return 0.0f;
            float t = free_path(rng, P.inv_extinction);
            if (t > d) break;
            F3 xn = x + w * t;
            float density = sample(xn, rng);
            pc.lookups++;
            x = xn;
            if (rng_next(rng) > 1.0f - density) return 0.0f;
            d -= t;
        }
    }
    return 1.0f;
}

// Next-event estimation at a surface hit (getIsoSurfaceHit with USE_ISOSURFACE_NEE, VptUtils.glsl:1213-1325,
// no lights): a sky direction l from importanceSampleSkybox; when it lies above the surface, the
// throughput times evaluateBrdfNee / pdf times the shadow ray's transmittance times the sky.  For a
// specular sample of Cook-Torrance or Disney (MIS), the light sample is weighed with
// pdf_l / (pdf_l + pdf_nee) and the BRDF's own direction adds its value weighed with
// pdf_out / (1 / (4 PI) + pdf_out) through a second shadow ray.
template <class S>
VPT_DEV void iso_surface_nee(const TraceParams& P, S& sample, Rng& rng, F3 x, const IsoFrame& fr,
                             const IsoBrdfSample& bs, F3 thr, F3& color, PathCtx& pc) {
    float pdf_light;
    const F3 l = importance_sample_sky(P, rng, pdf_light);
    if (!(dot3(fr.n, l) > 0.0f)) return;
    float pdf_out, pdf_nee;
    const F3 rdf = iso_brdf_nee(P, fr, bs, l, pdf_out, pdf_nee);
    const bool mis = (P.iso_brdf == kBrdfCookTorrance || P.iso_brdf == kBrdfDisney) && bs.specular;
    if (mis) {
        const float pdf_light_out = 1.0f / (4.0f * kPi);  // evaluateSkyboxPDF without an environment image
        const float w_nee = pdf_light / (pdf_light + pdf_nee);
        const float w_out = pdf_out / (pdf_light_out + pdf_out);
        const float tr = shadow_transmittance_delta(P, sample, rng, x + l * 1e-4f, l, pc);
        const F3 sky = sky_and_sun(P, l);
        color = color + f3(((((thr.x * rdf.x) * w_nee) / pdf_light) * tr) * sky.x,
                           ((((thr.y * rdf.y) * w_nee) / pdf_light) * tr) * sky.y,
                           ((((thr.z * rdf.z) * w_nee) / pdf_light) * tr) * sky.z);
        const float tr2 = shadow_transmittance_delta(P, sample, rng, x + bs.dir * 1e-4f, bs.dir, pc);
        const F3 sky2 = sky_and_sun(P, bs.dir);
        color = color + f3((((thr.x * w_out) * bs.value.x) * tr2) * sky2.x,
                           (((thr.y * w_out) * bs.value.y) * tr2) * sky2.y,
                           (((thr.z * w_out) * bs.value.z) * tr2) * sky2.z);
    } else {
        const float tr = shadow_transmittance_delta(P, sample, rng, x + l * 1e-4f, l, pc);
        const F3 sky = sky_and_sun(P, l);
        color = color + f3((((thr.x * rdf.x) / pdf_light) * tr) * sky.x, (((thr.y * rdf.y) / pdf_light) * tr) * sky.y,
                           (((thr.z * rdf.z) / pdf_light) * tr) * sky.z);
    }
}

// Ratio-tracking transmittance toward a light at distance `max_dist`
// (calculateTransmittanceDistance, NeeTransmittance.glsl:264-381, without isosurfaces): the walk
// stops at the box exit or when the accumulated distance passes the light.
template <class S>
VPT_DEV float shadow_transmittance_distance(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, float max_dist,
                                            PathCtx& pc) {
    float trans = 1.0f;
    float tmin, tmax;
    float cur = 0.0f;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        x = x + w * tmin;
        cur += tmin;
        float d = tmax - tmin;
        while (true) {
            if (guard(pc)) return 0.0f;
            float t = free_path(rng, P.inv_extinction);
            cur += t;
            if (t > d || cur > max_dist) break;
            F3 xn = x + w * t;
            float density = sample(xn, rng);
            pc.lookups++;
            x = xn;
            trans *= 1.0f - density;
            d -= t;
        }
    }
    return trans;
}

// Ratio-tracking transmittance with empty-space skipping over the occupancy grid
// (calculateTransmittance with USE_OCCUPANCY_GRID, NeeTransmittance.glsl:121-259).
template <class S>
VPT_DEV float shadow_transmittance_ess(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, PathCtx& pc) {
    float trans = 1.0f;
    const F3 eps = f3(1e-6f, 1e-6f, 1e-6f);
    float tmin_val, tmax_val;
    if (!ray_box(P.box_min + eps, P.box_max - eps, x, w, tmin_val, tmax_val)) return trans;
    F3 delta = P.box_max - P.box_min;
    x = x + w * tmin_val;
    F3 sp = (((x - P.box_min) / delta) * f3((float)P.nx, (float)P.ny, (float)P.nz)) /
            f3((float)P.sv_size, (float)P.sv_size, (float)P.sv_size);
    int ix = (int)floorf(sp.x), iy = (int)floorf(sp.y), iz = (int)floorf(sp.z);
    int cx = ix, cy = iy, cz = iz;
    bool empty = false;
    while (ix >= 0 && iy >= 0 && iz >= 0 && ix < P.svx && iy < P.svy && iz < P.svz) {
        if (guard(pc)) return 0.0f;
        F3 smin = P.box_min + f3((float)ix, (float)iy, (float)iz) * P.sv_world;
        F3 smax = smin + P.sv_world;
        float tmin_sv = 0.0f, tmax_sv = 0.0f;
        ray_box(smin, smax, x, w, tmin_sv, tmax_sv);
        float d_max = tmax_sv - tmin_sv;
        x = x + w * tmin_sv;
        if (cx != ix || cy != iy || cz != iz) {
            empty = __ldg(P.occupancy + ((size_t)iz * P.svy + iy) * P.svx + ix) == 0;
            cx = ix;
            cy = iy;
            cz = iz;
        }
        if (empty) {
            x = x + w * d_max;
        } else {
            // The reference advances x to each sample while t keeps counting from the supervoxel
            // entry, so its samples overshoot (NeeTransmittance.glsl:173-228); ess_ref_compat keeps
            // that behaviour, the default measures t from the entry point.
            const F3 x0 = x;
            float t = 0.0f;
            while (true) {
                if (guard(pc)) return 0.0f;
                t -= m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) * P.inv_extinction;
                if (t >= d_max) {
                    x = (P.ess_ref_compat ? x : x0) + w * d_max;
                    break;
                }
                F3 xn = (P.ess_ref_compat ? x : x0) + w * t;
                float density = sample(xn, rng);
                pc.lookups++;
                x = xn;
                trans *= 1.0f - density;
            }
        }
        F3 center = (smin + smax) * 0.5f;
        F3 mov = (x + w * 0.00001f) - center;
        float sx = signf(mov.x), sy = signf(mov.y), sz = signf(mov.z);
        mov = f3(mov.x * sx, mov.y * sy, mov.z * sz);
        int dx = (mov.x >= mov.y && mov.x >= mov.z) ? 1 : 0;
        int dy = (mov.y >= mov.x && mov.y >= mov.z) ? 1 : 0;
        int dz = (mov.z >= mov.x && mov.z >= mov.y) ? 1 : 0;
        ix += dx * (int)sx;
        iy += dy * (int)sy;
        iz += dz * (int)sz;
    }
    return trans;
}

// Next-event tracking: delta-tracked path; at each scatter one light sample toward the sky / sun
// with ratio-tracked transmittance; escape radiance only if no event happened
// (nextEventTracking, NextEventTracking.glsl:224-393; lights are not supported).
template <bool ESS, class S>
VPT_DEV F3 track_nee(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, FirstEvent& fe, PathCtx& pc) {
    F3 color = f3(0.0f, 0.0f, 0.0f);
    float tmin, tmax;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        x = x + w * tmin;
        float d = tmax - tmin;
        int bounces = 0;
        while (true) {
            if (guard(pc)) return color;
            float t = free_path(rng, P.inv_extinction);
            if (t > d) break;
            F3 xn = x + w * t;
            float density = sample(xn, rng);
            pc.lookups++;
            x = xn;
            float xi = rng_next(rng);
            if (xi < P.absorb_albedo * density) {
                record_event(fe, x, density, P.extinction, tmax - d + t, w);
                // USE_EMISSION (NextEventTracking.glsl:296-301): the absorbed path ends with the
                // emission; else USE_TRANSFER_FUNCTION (:303-310) with the table's
                return P.emission ? color + sample.emission(x, rng) : (P.tf ? color + sample.tf_emission() : color);
            }
            if (xi < density) {
                if (P.max_bounces > 0 && ++bounces > P.max_bounces) return color;
                F3 next_w = sample_phase(rng, P.g, w);
                record_scatter(fe, x, density, P.extinction, tmax - d + t, w, next_w, P.g);
                // with lights: the light list or the sky with probability 1/2 each (all lights when the
                // environment is black), NextEventTracking.glsl:335-364
                bool to_light = false;
                float prob_factor = 1.0f, light_dist = 0.0f, pdf_light = 0.0f;
                int light_idx = 0;
                F3 dir_light;
                if (P.num_lights > 0) {
                    to_light = P.env_is_black ? true : (rng_next(rng) > 0.5f);
                    prob_factor = P.env_is_black ? 1.0f : 2.0f;
                }
                if (to_light) dir_light = light_direction(P, x, rng, light_idx, prob_factor, light_dist);
                else dir_light = importance_sample_sky(P, rng, pdf_light);
                float pdf_phase = evaluate_phase(P.g, w, dir_light);
                w = next_w;
                if (P.num_lights > 0) {
                    const float common = prob_factor * pdf_phase;
                    if (to_light) {
                        float tr = shadow_transmittance_distance(P, sample, rng, x, dir_light, light_dist, pc);
                        float f = common * tr;
                        F3 l = light_radiance(P, x, light_idx);
                        color = color + f3(f * l.x, f * l.y, f * l.z);
                    } else {
                        float tr = ESS ? shadow_transmittance_ess(P, sample, rng, x, dir_light, pc)
                                       : shadow_transmittance(P, sample, rng, x, dir_light, pc);
                        float f = (common / pdf_light) * tr;
                        F3 l = sky_and_sun(P, dir_light);
                        color = color + f3(f * l.x, f * l.y, f * l.z);
                    }
                } else {
                    float tr = ESS ? shadow_transmittance_ess(P, sample, rng, x, dir_light, pc)
                                   : shadow_transmittance(P, sample, rng, x, dir_light, pc);
                    float f = (pdf_phase / pdf_light) * tr;
                    F3 l = sky_and_sun(P, dir_light);
                    color = color + f3(f * l.x, f * l.y, f * l.z);
                }
                if (ray_box_p(P, x, w, tmin, tmax)) {
                    x = x + w * tmin;
                    d = tmax - tmin;
                }
            } else {
                d -= t;
            }
        }
    }
    if (!fe.has) color = color + sky_and_sun(P, w);
    return color;
}

// VptMode::NEXT_EVENT_TRACKING with isosurfaces (NextEventTracking.glsl:224-393 with USE_ISOSURFACES and
// USE_ISOSURFACE_NEE; no lights): the 1000-iteration cap, iso_segment with next-event estimation at every
// surface hit, delta-tracked shadow rays (shadow_transmittance_delta), the volume's light samples scaled
// by the surface throughput, absorption ending the path with color (+ throughput * emission), and the sky
// added at the end only for a path without any event.
template <class S>
VPT_DEV F3 track_nee_iso(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, FirstEvent& fe, PathCtx& pc) {
    const F3 cam = x;  // cameraPosition (Clouds.glsl:99)
    bool outside = P.iso_close != 0;
    F3 color = f3(0.0f, 0.0f, 0.0f);
    F3 weights = f3(1.0f, 1.0f, 1.0f);
    float last_sign = 0.0f;
    bool first_point = true;
    int it = 0;
    float tmin, tmax;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        x = x + w * tmin;
        float d = tmax - tmin;
        int bounces = 0;
        while (true) {
            if (++it == 1000) return f3(0.0f, 0.0f, 0.0f);
            if (guard(pc)) return color;
            float t = free_path(rng, P.inv_extinction);
            if (t > d) break;
            F3 xn = x + w * t;
            float density = sample(xn, rng);
            pc.lookups++;
            if (iso_segment<true>(P, sample, rng, x, xn, density, w, d, tmax, weights, last_sign, first_point,
                                  pc.lookups, &fe, &color, &pc, P.iso_close ? &outside : nullptr, cam)) {
                if (weights.x < 1e-3f && weights.y < 1e-3f && weights.z < 1e-3f) return f3(0.0f, 0.0f, 0.0f);
                continue;
            }
            x = xn;
            float xi = rng_next(rng);
            if (xi < P.absorb_albedo * density) {
                record_event(fe, x, density, P.extinction, tmax - d + t, w);
                if (P.emission) {
                    const F3 e = sample.emission(x, rng);
                    return color + f3(weights.x * e.x, weights.y * e.y, weights.z * e.z);
                }
                return color;
            }
            if (xi < density) {
                if (P.max_bounces > 0 && ++bounces > P.max_bounces) return color;
                F3 next_w = sample_phase(rng, P.g, w);
                record_scatter(fe, x, density, P.extinction, tmax - d + t, w, next_w, P.g);
                float pdf_light;
                const F3 dir_light = importance_sample_sky(P, rng, pdf_light);
                const float pdf_phase = evaluate_phase(P.g, w, dir_light);
                w = next_w;
                const float tr = shadow_transmittance_delta(P, sample, rng, x, dir_light, pc);
                const float f = (pdf_phase / pdf_light) * tr;
                const F3 l = sky_and_sun(P, dir_light);
                color = color + f3((f * l.x) * weights.x, (f * l.y) * weights.y, (f * l.z) * weights.z);
                if (ray_box_p(P, x, w, tmin, tmax)) {
                    x = x + w * tmin;
                    d = tmax - tmin;
                }
            } else {
                d -= t;
            }
        }
    }
    if (!fe.has) color = color + sky_and_sun(P, w);
    return color;
}

// ---------------------------------------------------------------------------------------------
// Spectral tracking (Kutz et al. 2017): chromatic extinction parameters.extinction (rgb) with the
// majorant maxComponent(extinction); per-channel path weights; the collision probabilities of the
// three SpectralDeltaTrackingCollisionProbability modes.  Arithmetic in the shader's order.
struct SdtStep {
    float pa, ps, pn;  // normalised collision probabilities
    F3 sa, ss, sn;     // sigma_a, sigma_s, sigma_n
};

VPT_DEV float max_component(F3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }
VPT_DEV float avg_component(F3 v) { return ((v.x + v.y) + v.z) / 3.0f; }

// The scattering albedo of a spectral step: parameters.scatteringAlbedo, or with
// USE_TRANSFER_FUNCTION_SCATTERING_ALBEDO mix(scatteringAlbedo, the table's rgb at the lookup,
// tfScatteringAlbedoStrength) (DeltaTracking.glsl:76-81, NextEventTracking.glsl:77-82).
template <class S>
VPT_DEV F3 sdt_albedo(const TraceParams& P, const S& sample) {
    const F3 alb = f3(P.albedo_rgb[0], P.albedo_rgb[1], P.albedo_rgb[2]);
    if (!(P.tf && P.tf_albedo_strength > 0.0f)) return alb;
    const float s = P.tf_albedo_strength;
    return f3(alb.x * (1.0f - s) + sample.tf_rgb.x * s, alb.y * (1.0f - s) + sample.tf_rgb.y * s,
              alb.z * (1.0f - s) + sample.tf_rgb.z * s);
}

VPT_DEV SdtStep sdt_probabilities(const TraceParams& P, float density, F3 weights, F3 alb) {
    const F3 ext = f3(P.ext_rgb[0], P.ext_rgb[1], P.ext_rgb[2]);
    const F3 abs_alb = f3(1.0f - alb.x, 1.0f - alb.y, 1.0f - alb.z);
    SdtStep s;
    s.sa = f3((abs_alb.x * ext.x) * density, (abs_alb.y * ext.y) * density, (abs_alb.z * ext.z) * density);
    s.ss = f3((alb.x * ext.x) * density, (alb.y * ext.y) * density, (alb.z * ext.z) * density);
    const float m = P.sdt_majorant;
    s.sn = f3(m - ext.x * density, m - ext.y * density, m - ext.z * density);
    if (P.sdt_prob == kSdtMax) {
        s.pa = max_component(s.sa);
        s.ps = max_component(s.ss);
        s.pn = max_component(s.sn);
    } else if (P.sdt_prob == kSdtAvg) {
        s.pa = avg_component(s.sa);
        s.ps = avg_component(s.ss);
        s.pn = avg_component(s.sn);
    } else {
        s.pa = avg_component(f3(s.sa.x * weights.x, s.sa.y * weights.y, s.sa.z * weights.z));
        s.ps = avg_component(f3(s.ss.x * weights.x, s.ss.y * weights.y, s.ss.z * weights.z));
        s.pn = avg_component(f3(s.sn.x * weights.x, s.sn.y * weights.y, s.sn.z * weights.z));
    }
    const float c = (s.pa + s.ps) + s.pn;
    s.pa /= c;
    s.ps /= c;
    s.pn /= c;
    return s;
}

// weights *= sigma / (majorant * P)
VPT_DEV F3 sdt_reweight(F3 weights, F3 sigma, float majorant, float p) {
    const float den = majorant * p;
    return f3(weights.x * (sigma.x / den), weights.y * (sigma.y / den), weights.z * (sigma.z / den));
}

VPT_DEV F3 sdt_clamp(F3 v, float c) { return f3(fminf(v.x, c), fminf(v.y, c), fminf(v.z, c)); }

// VptMode::SPECTRAL_DELTA_TRACKING (deltaTrackingSpectral, DeltaTracking.glsl:33-163).  ISO: with
// isosurfaces (DeltaTracking.glsl:37-63 and the CheckIsosurfaceHit.glsl include): the 1000-iteration
// cap, iso_segment on every free-flight segment, the surface throughput multiplied into the spectral
// weights, and the path ended when all three fall below 1e-3 after a surface event.
template <bool ISO, class S>
VPT_DEV F3 track_delta_spectral(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, FirstEvent& fe,
                                PathCtx& pc) {
    const F3 cam = x;  // cameraPosition (Clouds.glsl:99)
    bool outside = ISO && P.iso_close != 0;
    F3 weights = f3(1.0f, 1.0f, 1.0f);
    float last_sign = 0.0f;
    bool first_point = true;
    int it = 0;
    float tmin, tmax;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        x = x + w * tmin;
        float d = tmax - tmin;
        int bounces = 0;
        while (true) {
            if (ISO && ++it == 1000) return f3(0.0f, 0.0f, 0.0f);
            if (guard(pc)) return f3(0.0f, 0.0f, 0.0f);
            float t = free_path(rng, P.inv_sdt_majorant);
            if (t > d) break;
            F3 xn = x + w * t;
            float density = sample(xn, rng);
            pc.lookups++;
            if constexpr (ISO) {
                if (iso_segment(P, sample, rng, x, xn, density, w, d, tmax, weights, last_sign, first_point,
                                pc.lookups, &fe, nullptr, nullptr, P.iso_close ? &outside : nullptr, cam)) {
                    if (weights.x < 1e-3f && weights.y < 1e-3f && weights.z < 1e-3f) return f3(0.0f, 0.0f, 0.0f);
                    continue;
                }
            }
            x = xn;
            const SdtStep st = sdt_probabilities(P, density, weights, sdt_albedo(P, sample));
            float xi = rng_next(rng);
            if (xi < st.pa) {
                record_event(fe, x, density, P.sdt_majorant, tmax - d + t);
                if (P.tf) {  // USE_TRANSFER_FUNCTION (DeltaTracking.glsl:125-127): weights sigma_a / (maj Pa) L_e
                    const F3 le = sample.tf_emission();
                    const float den = P.sdt_majorant * st.pa;
                    return f3(weights.x * st.sa.x / den * le.x, weights.y * st.sa.y / den * le.y,
                              weights.z * st.sa.z / den * le.z);
                }
                return f3(0.0f, 0.0f, 0.0f);
            }
            if (xi < st.pa + st.ps) {
                if (P.max_bounces > 0 && ++bounces > P.max_bounces) return f3(0.0f, 0.0f, 0.0f);
                const F3 w_in = w;
                w = sample_phase(rng, P.g, w);
                record_scatter(fe, x, density, P.sdt_majorant, tmax - d + t, w_in, w, P.g);
                if (ray_box_p(P, x, w, tmin, tmax)) {
                    x = x + w * tmin;
                    d = tmax - tmin;
                }
                weights = sdt_reweight(weights, st.ss, P.sdt_majorant, st.ps);
            } else {
                d -= t;
                weights = sdt_reweight(weights, st.sn, P.sdt_majorant, st.pn);
            }
            if (P.sdt_prob == kSdtPathHistory) weights = sdt_clamp(weights, 100.0f);
        }
    }
    const F3 wc = sdt_clamp(weights, 100000.0f);
    const F3 l = sky_and_sun(P, w);
    return f3(wc.x * l.x, wc.y * l.y, wc.z * l.z);
}

// VptMode::NEXT_EVENT_TRACKING_SPECTRAL (nextEventTrackingSpectral, NextEventTracking.glsl:31-220):
// spectral tracking with a next-event estimate at every scatter event (transmittance from the
// achromatic shadow estimators, NeeTransmittance.glsl, like the reference).  ISO: with isosurfaces and
// USE_ISOSURFACE_NEE (no lights): the 1000-iteration cap, iso_segment with surface next-event
// estimation, delta-tracked shadow rays, emission scaled by the surface throughput.
template <bool ESS, bool ISO = false, class S>
VPT_DEV F3 track_nee_spectral(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, FirstEvent& fe, PathCtx& pc) {
    const F3 cam = x;  // cameraPosition (Clouds.glsl:99)
    bool outside = ISO && P.iso_close != 0;
    F3 weights = f3(1.0f, 1.0f, 1.0f);
    F3 color = f3(0.0f, 0.0f, 0.0f);
    float last_sign = 0.0f;
    bool first_point = true;
    int it = 0;
    float tmin, tmax;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        x = x + w * tmin;
        float d = tmax - tmin;
        int bounces = 0;
        while (true) {
            if (ISO && ++it == 1000) return f3(0.0f, 0.0f, 0.0f);
            if (guard(pc)) return color;
            float t = free_path(rng, P.inv_sdt_majorant);
            if (t > d) break;
            F3 xn = x + w * t;
            // with a transfer function the reference looks up the previous point x
            // (NextEventTracking.glsl:74, sampleCloudDensityEmission(x)); reproduced
            float density = sample(P.tf ? x : xn, rng);
            pc.lookups++;
            if constexpr (ISO) {  // CheckIsosurfaceHit.glsl with surface next-event estimation
                if (iso_segment<true>(P, sample, rng, x, xn, density, w, d, tmax, weights, last_sign, first_point,
                                      pc.lookups, &fe, &color, &pc, P.iso_close ? &outside : nullptr, cam)) {
                    if (weights.x < 1e-3f && weights.y < 1e-3f && weights.z < 1e-3f) return f3(0.0f, 0.0f, 0.0f);
                    continue;
                }
            }
            x = xn;
            const SdtStep st = sdt_probabilities(P, density, weights, sdt_albedo(P, sample));
            float xi = rng_next(rng);
            if (xi < st.pa) {
                record_event(fe, x, density, P.sdt_majorant, tmax - d + t);
                // USE_EMISSION (NextEventTracking.glsl:125-131); else USE_TRANSFER_FUNCTION (:133-139),
                // which returns the emission without the NEE colour gathered so far
                if (ISO && P.emission) {  // NextEventTracking.glsl:118-124: the surface throughput applies
                    const F3 e = sample.emission(x, rng);
                    return color + f3(weights.x * e.x, weights.y * e.y, weights.z * e.z);
                }
                return P.emission ? color + sample.emission(x, rng) : (P.tf ? sample.tf_emission() : color);
            }
            if (xi < st.pa + st.ps) {
                if (P.max_bounces > 0 && ++bounces > P.max_bounces) return color;
                F3 next_w = sample_phase(rng, P.g, w);
                record_scatter(fe, x, density, P.sdt_majorant, tmax - d + t, w, next_w, P.g);
                bool to_light = false;
                float prob_factor = 1.0f, light_dist = 0.0f, pdf_light = 0.0f;
                int light_idx = 0;
                F3 dir_light;
                if (P.num_lights > 0) {
                    to_light = P.env_is_black ? true : (rng_next(rng) > 0.5f);
                    prob_factor = P.env_is_black ? 1.0f : 2.0f;
                }
                if (to_light) dir_light = light_direction(P, x, rng, light_idx, prob_factor, light_dist);
                else dir_light = importance_sample_sky(P, rng, pdf_light);
                const float pdf_phase = evaluate_phase(P.g, w, dir_light);
                w = next_w;
                weights = sdt_reweight(weights, st.ss, P.sdt_majorant, st.ps);
                const F3 wc = sdt_clamp(weights, 100000.0f);
                if (P.num_lights > 0) {
                    const float cf = prob_factor * pdf_phase;
                    const F3 common = f3(cf * wc.x, cf * wc.y, cf * wc.z);
                    if (to_light) {
                        const float tr = shadow_transmittance_distance(P, sample, rng, x, dir_light, light_dist, pc);
                        const F3 l = light_radiance(P, x, light_idx);
                        color = color + f3((common.x * tr) * l.x, (common.y * tr) * l.y, (common.z * tr) * l.z);
                    } else {
                        const float tr = ESS ? shadow_transmittance_ess(P, sample, rng, x, dir_light, pc)
                                             : shadow_transmittance(P, sample, rng, x, dir_light, pc);
                        const F3 l = sky_and_sun(P, dir_light);
                        color = color + f3(((common.x / pdf_light) * tr) * l.x, ((common.y / pdf_light) * tr) * l.y,
                                           ((common.z / pdf_light) * tr) * l.z);
                    }
                } else {
                    const float tr = ISO ? shadow_transmittance_delta(P, sample, rng, x, dir_light, pc)
                                         : (ESS ? shadow_transmittance_ess(P, sample, rng, x, dir_light, pc)
                                                : shadow_transmittance(P, sample, rng, x, dir_light, pc));
                    const float f = (pdf_phase / pdf_light) * tr;
                    const F3 l = sky_and_sun(P, dir_light);
                    color = color + f3((f * wc.x) * l.x, (f * wc.y) * l.y, (f * wc.z) * l.z);
                }
                if (ray_box_p(P, x, w, tmin, tmax)) {
                    x = x + w * tmin;
                    d = tmax - tmin;
                }
            } else {
                d -= t;
                weights = sdt_reweight(weights, st.sn, P.sdt_majorant, st.pn);
            }
            if (P.sdt_prob == kSdtPathHistory) weights = sdt_clamp(weights, 100.0f);
        }
    }
    if (!fe.has) {
        const F3 wc = sdt_clamp(weights, 100000.0f);
        const F3 l = sky_and_sun(P, w);
        color = color + f3((1.0f * wc.x) * l.x, (1.0f * wc.y) * l.y, (1.0f * wc.z) * l.z);
    }
    return color;
}

// ---------------------------------------------------------------------------------------------
// Supervoxel stepping shared by decomposition tracking and the occupancy-grid shadow ray: after a
// supervoxel is left, move to the neighbour along the dominant axis of (x + 1e-5 w - centre)
// (DecompositionTracking.glsl:112-118).
VPT_DEV void sv_step(F3 smin, F3 smax, F3 x, F3 w, int& ix, int& iy, int& iz) {
    F3 center = (smin + smax) * 0.5f;
    F3 mov = (x + w * 0.00001f) - center;
    float sx = signf(mov.x), sy = signf(mov.y), sz = signf(mov.z);
    mov = f3(mov.x * sx, mov.y * sy, mov.z * sz);
    int dx = (mov.x >= mov.y && mov.x >= mov.z) ? 1 : 0;
    int dy = (mov.y >= mov.x && mov.y >= mov.z) ? 1 : 0;
    int dz = (mov.z >= mov.x && mov.z >= mov.y) ? 1 : 0;
    ix += dx * (int)sx;
    iy += dy * (int)sy;
    iz += dz * (int)sz;
}

// Analog decomposition tracking over the dense supervoxel grid: per supervoxel a control
// extinction mu_c = majorant * min and a residual majorant majorant * max - mu_c; competing
// exponential samples t_c, t_r; residual collisions accepted with (mu(x) - mu_c) / mu_r
// (analogDecompositionTracking, DecompositionTracking.glsl:35-123).
template <class S>
VPT_DEV F3 track_decomposition(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, FirstEvent& fe,
                               PathCtx& pc) {
    const F3 eps = f3(1e-6f, 1e-6f, 1e-6f);
    float tmin_val, tmax_val;
    if (ray_box(P.box_min + eps, P.box_max - eps, x, w, tmin_val, tmax_val)) {
        const float majorant = P.extinction;
        F3 delta = P.box_max - P.box_min;
        x = x + w * tmin_val;
        F3 sp = (((x - P.box_min) / delta) * f3((float)P.nx, (float)P.ny, (float)P.nz)) /
                f3((float)P.sv_size, (float)P.sv_size, (float)P.sv_size);
        int ix = (int)floorf(sp.x), iy = (int)floorf(sp.y), iz = (int)floorf(sp.z);
        int cx = -1, cy = -1, cz = -1;
        float smin_d = 0.0f, smax_d = 0.0f;
        int bounces = 0;
        while (ix >= 0 && iy >= 0 && iz >= 0 && ix < P.svx && iy < P.svy && iz < P.svz) {
            if (guard(pc)) return f3(0.0f, 0.0f, 0.0f);
            F3 smin = P.box_min + f3((float)ix, (float)iy, (float)iz) * P.sv_world;
            F3 smax = smin + P.sv_world;
            float tmin_sv = 0.0f, tmax_sv = 0.0f;
            ray_box(smin, smax, x, w, tmin_sv, tmax_sv);
            float d_max = tmax_sv - tmin_sv;
            x = x + w * tmin_sv;
            if (cx != ix || cy != iy || cz != iz) {
                const float2 mm = __ldg(reinterpret_cast<const float2*>(P.sv_data) + ((size_t)iz * P.svy + iy) * P.svx + ix);
                smin_d = mm.x;
                smax_d = mm.y;
                cx = ix;
                cy = iy;
                cz = iz;
            }
            if (smax_d < 1e-5f) {
                x = x + w * d_max;
            } else {
                float mu_c = fmaxf(0.0000000001f, majorant * smin_d);
                float mu_r = fmaxf(0.0000000001f, majorant * smax_d - mu_c);
                float t_c = -m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) / mu_c;
                float t_r = 0.0f;
                while (true) {
                    if (guard(pc)) return f3(0.0f, 0.0f, 0.0f);
                    t_r -= m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) / mu_r;
                    if (t_c >= d_max && t_r >= d_max) {
                        x = x + w * d_max;
                        break;
                    }
                    F3 xs = x + w * fminf(t_c, t_r);
                    bool collision;
                    if (t_c <= t_r) {
                        collision = true;
                    } else {
                        float density = sample(xs, rng);
                        pc.lookups++;
                        collision = rng_next(rng) * mu_r < P.extinction * density - mu_c;
                    }
                    if (collision) {
                        x = xs;
                        if (rng_next(rng) < P.absorb_albedo) return f3(0.0f, 0.0f, 0.0f);
                        if (P.max_bounces > 0 && ++bounces > P.max_bounces) return f3(0.0f, 0.0f, 0.0f);
                        w = sample_phase(rng, P.g, w);
                        t_r = 0.0f;
                        t_c = -m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) / mu_c;
                        ray_box(smin, smax, x, w, tmin_sv, tmax_sv);
                        d_max = tmax_sv - tmin_sv;
                    }
                }
            }
            sv_step(smin, smax, x, w, ix, iy, iz);
        }
    }
    return sky_and_sun(P, w);
}

// Analog decomposition tracking over a sparse grid with the hierarchical DDA
// (analogDecompositionTracking, DecompositionTracking.glsl:130-360): the HDDA walks the tree at the
// leaf level (cells of 8^3, coarser in tiles), skips inactive nodes, and inside an active node
// tracks with a control extinction of 1e-10 and a residual majorant equal to the global majorant
// (the node min/max are read but unused by the reference).  After a scattering event the node box
// bounds the next segment and the HDDA restarts behind it.  The node box of a leaf is
// [LeafData::mBBoxMin, +8), of a tile the bounding box of its node, as in the reference.
template <class S>
VPT_DEV F3 track_decomposition_sparse(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, FirstEvent& fe,
                                      PathCtx& pc) {
    const SparseView& V = P.sparse;
    F3 origin = sparse_world_to_index(V, x);
    F3 direction = sparse_world_to_index_dir(V, w);
    const float grid_to_world = 1.0f / length3(direction);
    direction = direction * grid_to_world;
    float t_min = 0.0f, t_max = 1e10f;
    const F3 root_lo = f3((float)V.root_min[0], (float)V.root_min[1], (float)V.root_min[2]);
    const F3 root_hi = f3((float)(V.root_max[0] + 1), (float)(V.root_max[1] + 1), (float)(V.root_max[2] + 1));
    const bool hits_root = hdda_ray_clip(root_lo, root_hi, origin, t_min, direction, t_max);
    if (hits_root && t_max < 1e20f) {
        const float majorant = P.extinction;
        const int lowest = V.lowest_level;
        int bounces = 0;
        Hdda h;
        hdda_init(h, origin, t_min - 1e-4f, direction, t_max + 1e-4f, lowest);
        for (int iteration = 0;; iteration++) {
            if (guard(pc)) return f3(0.0f, 0.0f, 0.0f);
            if (iteration > 0) {
                if (!hdda_step(h)) break;
                const int d = max(sparse_dim(V, h.voxel[0], h.voxel[1], h.voxel[2]), lowest);
                hdda_update(h, origin, direction, d);
            }
            F3 nmin, nmax;
            if (!sparse_cell_node(V, h.voxel, nmin, nmax)) continue;
            float t_min_node = 0.0f, t_max_node = 1e10f;
            const bool hits_node = hdda_ray_clip(nmin, nmax, origin, t_min_node, direction, t_max_node);
            x = sparse_index_to_world(V, origin + direction * t_min_node);
            if (!hits_node) continue;
            float d_max = grid_to_world * (fminf(fminf(h.next[0], h.next[1]), h.next[2]) - h.tmin);
            const float mu_c = 0.0000000001f;
            const float mu_r = fmaxf(0.0000000001f, majorant * 1.0f - mu_c);
            bool direction_changed = false;
            float t_c = -m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) / mu_c;
            float t_r = 0.0f;
            while (true) {
                if (guard(pc)) return f3(0.0f, 0.0f, 0.0f);
                t_r -= m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) / mu_r;
                if (t_c >= d_max && t_r >= d_max) {
                    x = x + d_max * w;
                    break;
                }
                const F3 xs = x + w * fminf(t_c, t_r);
                bool collision;
                if (t_c <= t_r) {
                    collision = true;
                } else {
                    const float density = sample(xs, rng);
                    pc.lookups++;
                    collision = rng_next(rng) * mu_r < P.extinction * density - mu_c;
                }
                if (collision) {
                    x = xs;
                    if (rng_next(rng) < P.absorb_albedo) return f3(0.0f, 0.0f, 0.0f);
                    if (P.max_bounces > 0 && ++bounces > P.max_bounces) return f3(0.0f, 0.0f, 0.0f);
                    w = sample_phase(rng, P.g, w);
                    t_r = 0.0f;
                    t_c = -m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) / mu_c;
                    origin = sparse_world_to_index(V, x);
                    direction = normalize3(sparse_world_to_index_dir(V, w));
                    float t_min_leaf = 0.0f, t_max_leaf = 1e10f;
                    ray_box(nmin, nmax, origin, direction, t_min_leaf, t_max_leaf);
                    hdda_ray_clip(nmin, nmax, origin, t_min_leaf, direction, t_max_leaf);
                    d_max = grid_to_world * (t_max_leaf - t_min_leaf);
                    direction_changed = true;
                }
            }
            if (direction_changed) {
                t_min = 0.0f;
                t_max = 1e10f;
                hdda_ray_clip(root_lo, root_hi, origin, t_min, direction, t_max);
                hdda_init(h, origin, t_min + d_max / grid_to_world + 1e-4f, direction, t_max + 1e-4f, lowest);
            }
        }
    }
    return sky_and_sun(P, w);
}

// Per-supervoxel residual ratio tracking estimator with reservoir selection of the next
// in-scattering distance (residualRatioTrackingEstimator, ResidualRatioTracking.glsl:34-76).
template <class S>
VPT_DEV float rrt_estimator(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, float d_start, float d_end,
                            float T, float& wsum, float& res_t, float& res_dist, float mu_c, float mu_r,
                            PathCtx& pc) {
    float t_c = m_exp(-mu_c * (d_end - d_start));
    float t_r = 1.0f;
    float d_trav = d_start;
    while (true) {
        if (guard(pc)) break;
        float t = -m_log(fmaxf(0.0000000001f, 1.0f - rng_next(rng))) / mu_r;
        x = x + w * t;
        d_trav += t;
        if (d_trav >= d_end) break;
        float density = sample(x, rng);
        pc.lookups++;
        float mu = P.extinction * density;
        t_r *= 1.0f - (mu - mu_c) / mu_r;
        float t_c_local = m_exp(-mu_c * (d_trav - d_start));
        float t_local = (T * t_r) * t_c_local;
        wsum += t_local;
        float xi = rng_next(rng);
        if (xi < t_local / wsum) {
            res_t = t_local;
            res_dist = d_trav;
        }
    }
    return t_c * t_r;
}

VPT_DEV float fractf(float v) { return v - floorf(v); }

// Residual ratio tracking over the supervoxel (mu_c, mu_r_bar) grid with an Amanatides-Woo DDA and
// up to 10 reservoir-sampled in-scattering rays (residualRatioTracking,
// ResidualRatioTracking.glsl:78-223; the reference marks this estimator "work in progress").
template <class S>
VPT_DEV F3 track_residual_ratio(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, FirstEvent& fe,
                                PathCtx& pc) {
    float wsum = 0.0f, res_t = 0.0f, res_dist = 0.0f;
    float T = 1.0f;
    F3 acc = f3(0.0f, 0.0f, 0.0f);
    const F3 eps = f3(1e-6f, 1e-6f, 1e-6f);
    const F3 n = f3((float)P.nx, (float)P.ny, (float)P.nz);
    const F3 sv = f3((float)P.sv_size, (float)P.sv_size, (float)P.sv_size);
    F3 delta = P.box_max - P.box_min;
    F3 old_x = x;
    int iteration = 0;
    while (true) {
        float tmin_val, tmax_val;
        if (!ray_box(P.box_min + eps, P.box_max - eps, x, w, tmin_val, tmax_val)) break;
        x = x + w * tmin_val;
        old_x = x;
        float d_total = tmax_val - tmin_val;
        F3 sp = (((x - P.box_min) / delta) * n) / sv;
        F3 ep = ((((x + w * d_total) - P.box_min) / delta) * n) / sv;
        float spv[3] = {sp.x, sp.y, sp.z};
        float epv[3] = {ep.x, ep.y, ep.z};
        int step[3], idx[3];
        float tdel[3], tmx[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            float diff = epv[a] - spv[a];
            step[a] = (int)signf(diff);
            tdel[a] = step[a] != 0 ? fminf((float)step[a] / diff, 1e7f) : 1e7f;
            tmx[a] = step[a] > 0 ? tdel[a] * (1.0f - fractf(spv[a])) : tdel[a] * fractf(spv[a]);
            idx[a] = (int)floorf(spv[a]);
        }
        if (step[0] == 0 && step[1] == 0 && step[2] == 0) break;
        while (idx[0] >= 0 && idx[1] >= 0 && idx[2] >= 0 && idx[0] < P.svx && idx[1] < P.svy && idx[2] < P.svz) {
            if (guard(pc)) return acc;
            const float2 sv_val =
                __ldg(reinterpret_cast<const float2*>(P.sv_data) + ((size_t)idx[2] * P.svy + idx[1]) * P.svx + idx[0]);
            F3 vmin = f3((float)(idx[0] * P.sv_size), (float)(idx[1] * P.sv_size), (float)(idx[2] * P.sv_size));
            F3 vmax = f3((float)(idx[0] * P.sv_size + P.sv_size), (float)(idx[1] * P.sv_size + P.sv_size),
                         (float)(idx[2] * P.sv_size + P.sv_size));
            vmin = (vmin / n) * delta + P.box_min;
            vmax = (vmax / n) * delta + P.box_min;
            float tmin_v = 0.0f, tmax_v = 0.0f;
            ray_box(vmin, vmax, old_x, w, tmin_v, tmax_v);
            x = old_x + w * tmin_v;
            T *= rrt_estimator(P, sample, rng, x, w, tmin_v, tmax_v, T, wsum, res_t, res_dist, sv_val.x, sv_val.y, pc);
            if (tmx[0] < tmx[1]) {
                if (tmx[0] < tmx[2]) {
                    idx[0] += step[0];
                    tmx[0] += tdel[0];
                } else {
                    idx[2] += step[2];
                    tmx[2] += tdel[2];
                }
            } else {
                if (tmx[1] < tmx[2]) {
                    idx[1] += step[1];
                    tmx[1] += tdel[1];
                } else {
                    idx[2] += step[2];
                    tmx[2] += tdel[2];
                }
            }
        }
        float xi = rng_next(rng);
        if (xi > wsum || iteration >= 10) break;
        acc = acc + sky_and_sun(P, w) * T;
        iteration++;
        T = res_t;
        x = old_x + w * res_dist;
        w = sample_phase(rng, P.g, w);
        wsum = 0.0f;
        res_t = 0.0f;
        res_dist = 0.0f;
    }
    acc = acc + sky_and_sun(P, w) * T;
    return acc;
}


// ---------------------------------------------------------------------------------------------
// Residual ratio tracking, unbiased (no reference counterpart; the reference's residual ratio mode
// is the reservoir estimator above).  Next-event estimation whose shadow transmittance is residual
// ratio tracking (Novak et al. 2014) with the per-supervoxel control and residual extinctions
// (mu_c, mu_r_bar) of SuperVoxelGrid.cpp:218-265, and whose free paths are delta tracking with the
// supervoxel's own majorant: extinction times the largest normalised density of the supervoxel and
// a one-voxel halo, which bounds every lookup inside it (a stochastic or trilinear lookup reads at
// most half a voxel beyond its point).  A supervoxel whose majorant is 0 holds no density that a
// lookup could return, so both walks cross it without drawing a random number.  Supervoxel data:
// 4 floats (mu_c, mu_r_bar, 1 / max density, 1 / majorant; the last two 0 when empty).

// Amanatides-Woo walk over the supervoxel grid in world units: the ray distance to the next cell
// boundary of each axis and between boundaries.
struct SvWalk {
    int idx[3];
    int step[3];
    float next[3];
    float delta[3];
};

VPT_DEV void sv_walk_begin(const TraceParams& P, F3 x, F3 w, SvWalk& s) {
    const float xv[3] = {x.x, x.y, x.z}, wv[3] = {w.x, w.y, w.z};
    const float bmin[3] = {P.box_min.x, P.box_min.y, P.box_min.z};
    const float sw[3] = {P.sv_world.x, P.sv_world.y, P.sv_world.z};
    const float inv[3] = {P.sv_inv_world.x, P.sv_inv_world.y, P.sv_inv_world.z};
    const int n[3] = {P.svx, P.svy, P.svz};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        int i = (int)floorf((xv[a] - bmin[a]) * inv[a]);
        i = min(max(i, 0), n[a] - 1);
        s.idx[a] = i;
        if (wv[a] > 0.0f) {
            s.step[a] = 1;
            s.next[a] = ((bmin[a] + (float)(i + 1) * sw[a]) - xv[a]) / wv[a];
            s.delta[a] = sw[a] / wv[a];
        } else if (wv[a] < 0.0f) {
            s.step[a] = -1;
            s.next[a] = ((bmin[a] + (float)i * sw[a]) - xv[a]) / wv[a];
            s.delta[a] = -sw[a] / wv[a];
        } else {
            s.step[a] = 0;
            s.next[a] = INFINITY;
            s.delta[a] = INFINITY;
        }
    }
}

// the axis whose cell boundary comes first
VPT_DEV int sv_walk_axis(const SvWalk& s) {
    return s.next[0] < s.next[1] ? (s.next[0] < s.next[2] ? 0 : 2) : (s.next[1] < s.next[2] ? 1 : 2);
}

// steps over the boundary of axis a; false when the walk leaves the grid
VPT_DEV bool sv_walk_advance(const TraceParams& P, SvWalk& s, int a) {
    s.idx[a] += s.step[a];
    s.next[a] += s.delta[a];
    const int n = a == 0 ? P.svx : (a == 1 ? P.svy : P.svz);
    return s.idx[a] >= 0 && s.idx[a] < n;
}

VPT_DEV float4 sv_local_cell(const TraceParams& P, const SvWalk& s) {
    return __ldg(reinterpret_cast<const float4*>(P.sv_local) + ((size_t)s.idx[2] * P.svy + s.idx[1]) * P.svx +
                 s.idx[0]);
}

// Residual ratio tracking transmittance from x along w over at most max_dist (the box exit
// otherwise): per supervoxel exp(-mu_c * length) times (1 - (mu(x_i) - mu_c) / mu_r_bar) at the
// points of a Poisson process of rate mu_r_bar.
template <class S>
VPT_DEV float shadow_residual_ratio(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, float max_dist,
                                    PathCtx& pc) {
    float tmin, tmax;
    if (!ray_box_p(P, x, w, tmin, tmax)) return 1.0f;
    const float d = fminf(tmax, max_dist) - tmin;
    if (!(d > 0.0f)) return 1.0f;
    x = x + w * tmin;
    SvWalk s;
    sv_walk_begin(P, x, w, s);
    float T = 1.0f;
    float t0 = 0.0f;
    while (true) {
        if (guard(pc)) return 0.0f;
        const int a = sv_walk_axis(s);
        const float t1 = fminf(s.next[a], d);
        const float4 c = sv_local_cell(P, s);
        if (c.w > 0.0f && t1 > t0) {
            T *= m_exp(-c.x * (t1 - t0));
            const float inv_mu_r = 1.0f / c.y;
            float t = t0;
            while (true) {
                if (guard(pc)) return 0.0f;
                t += free_path(rng, inv_mu_r);
                if (t >= t1) break;
                const float density = sample(x + w * t, rng);
                pc.lookups++;
                T *= 1.0f - (P.extinction * density - c.x) * inv_mu_r;
            }
        }
        if (t1 >= d) break;
        t0 = fmaxf(t0, t1);
        if (!sv_walk_advance(P, s, a)) break;
    }
    return T;
}

template <class S>
VPT_DEV F3 track_residual_ratio_nee(const TraceParams& P, S& sample, Rng& rng, F3 x, F3 w, FirstEvent& fe,
                                    PathCtx& pc) {
    F3 color = f3(0.0f, 0.0f, 0.0f);
    float tmin, tmax;
    if (ray_box_p(P, x, w, tmin, tmax)) {
        x = x + w * tmin;
        float d = tmax - tmin;
        float depth0 = tmin;  // distance of x from the camera while no event has happened
        int bounces = 0;
        while (true) {
            // one free flight from x along w over [0, d)
            SvWalk s;
            sv_walk_begin(P, x, w, s);
            float t0 = 0.0f, t = 0.0f, density = 0.0f;
            bool collided = false;
            while (true) {
                if (guard(pc)) return color;
                const int a = sv_walk_axis(s);
                const float t1 = fminf(s.next[a], d);
                const float4 c = sv_local_cell(P, s);
                if (c.w > 0.0f && t1 > t0) {
                    t = t0;
                    while (true) {
                        if (guard(pc)) return color;
                        t += free_path(rng, c.w);
                        if (t >= t1) break;
                        density = sample(x + w * t, rng);
                        pc.lookups++;
                        const float r = density * c.z;  // density / majorant density
                        const float xi = rng_next(rng);
                        if (xi < P.absorb_albedo * r) {
                            const F3 xa = x + w * t;
                            record_event(fe, xa, density, P.extinction, depth0 + t, w);  // as next event tracking
                            return P.emission ? color + sample.emission(xa, rng) : color;
                        }
                        if (xi < r) {
                            collided = true;
                            break;
                        }
                    }
                    if (collided) break;
                }
                if (t1 >= d) break;
                t0 = fmaxf(t0, t1);
                if (!sv_walk_advance(P, s, a)) break;
            }
            if (!collided) break;
            x = x + w * t;
            if (P.max_bounces > 0 && ++bounces > P.max_bounces) return color;
            const F3 next_w = sample_phase(rng, P.g, w);
            record_scatter(fe, x, density, P.extinction, depth0 + t, w, next_w, P.g);
            // light selection as in next event tracking (NextEventTracking.glsl:335-364)
            bool to_light = false;
            float prob_factor = 1.0f, light_dist = 0.0f, pdf_light = 0.0f;
            int light_idx = 0;
            F3 dir_light;
            if (P.num_lights > 0) {
                to_light = P.env_is_black ? true : (rng_next(rng) > 0.5f);
                prob_factor = P.env_is_black ? 1.0f : 2.0f;
            }
            if (to_light) dir_light = light_direction(P, x, rng, light_idx, prob_factor, light_dist);
            else dir_light = importance_sample_sky(P, rng, pdf_light);
            const float pdf_phase = evaluate_phase(P.g, w, dir_light);
            w = next_w;
            if (to_light) {
                const float tr = shadow_residual_ratio(P, sample, rng, x, dir_light, light_dist, pc);
                const float f = (prob_factor * pdf_phase) * tr;
                const F3 l = light_radiance(P, x, light_idx);
                color = color + f3(f * l.x, f * l.y, f * l.z);
            } else {
                const float tr = shadow_residual_ratio(P, sample, rng, x, dir_light, INFINITY, pc);
                const float f = ((prob_factor * pdf_phase) / pdf_light) * tr;
                const F3 l = sky_and_sun(P, dir_light);
                color = color + f3(f * l.x, f * l.y, f * l.z);
            }
            if (!ray_box_p(P, x, w, tmin, tmax)) break;
            x = x + w * tmin;
            d = tmax - tmin;
        }
    }
    if (!fe.has) color = color + sky_and_sun(P, w);
    return color;
}

}  // namespace vpt
