// Radiance estimators, per camera ray, in FP32 with the reference's draw order.
//
//   PathEstimator::radiance        estimator/path_estimator.cpp:153-185
//   sampleDirectLight              estimator/path_estimator.cpp:73-102
//   weightedEmission / weightedSky estimator/path_estimator.cpp:106-132
//   survivesRoulette               estimator/path_estimator.cpp:140-149
//   ScatterOnlyEstimator           estimator/scatter_only_estimator.cpp:14-48
//   NormalsEstimator               estimator/normals_estimator.cpp:17-38
// Random numbers per bounce: 3 for next-event estimation (drawn even with no
// lights), 3 for the BSDF sample, 1 for roulette once depth >= roulette_start.
#pragma once

#include "launch.hpp"
#include "shade.cuh"

namespace albedo_b200 {

struct TraceContext {
    uint2* stack;
    int stride;
    int capacity;
    unsigned int* error_flag;
    TraversalCounts* counts; // null except in the counting variants
};

ALB_DEV bool closestHit(const DevScene& s, const TraceContext& c, float3 o, float3 d, const SkipRule& skip,
                        TraceHit& hit)
{
    float tmax = INFINITY;
    return traceScene<false>(s, o, d, 0.0f, tmax, skip, hit, c.stack, c.stride, c.capacity, c.error_flag, c.counts);
}

ALB_DEV bool occluded(const DevScene& s, const TraceContext& c, float3 o, float3 d, float tmax, const SkipRule& skip)
{
    TraceHit hit;
    return traceScene<true>(s, o, d, 0.0f, tmax, skip, hit, c.stack, c.stride, c.capacity, c.error_flag, c.counts);
}

// Next-event estimation from one uniformly chosen light, MIS-weighted, scaled
// by nothing (the caller multiplies by the throughput).
ALB_DEV float3 sampleDirectLight(const DevScene& s, const TraceContext& c, const Surface& sf, const Scattering& sc,
                                 float3 wo, Pcg32& g)
{
    const float u_light = g.next1D();
    const float ux = g.next1D();
    const float uy = g.next1D();
    if (s.light_count == 0u) {
        return gray(0.0f);
    }
    const int n = static_cast<int>(s.light_count);
    const int index = min(static_cast<int>(u_light * static_cast<float>(n)), n - 1);
    const DevLight light = s.lights[index];
    LightSample ls;
    if (!sampleLight(light, sf.p, ux, uy, ls) || isBlack(ls.radiance)) {
        return gray(0.0f);
    }
    const float3 f = sc.evaluate(wo, ls.dir);
    if (isBlack(f)) {
        return gray(0.0f);
    }
    const float range_max = shadowRangeMax(ls.distance);
    if (range_max > 0.0f) {
        float3 so;
        SkipRule skip;
        rayLeaving(sf, ls.dir, so, skip);
        if (light.kind == kLightArea) {
            skip.light_object_pos = light.object;
        }
        if (occluded(s, c, so, ls.dir, range_max, skip)) {
            return gray(0.0f);
        }
    }
    const float light_pdf = (1.0f / static_cast<float>(n)) * ls.pdf;
    const float weight = ls.delta ? 1.0f : powerHeuristic(light_pdf, sc.pdf(wo, ls.dir));
    const float cos_theta = fabsf(dot(ls.dir, sf.ns));
    return f * ls.radiance * (cos_theta * weight / light_pdf);
}

ALB_DEV float3 pathRadiance(const DevScene& s, const TraceContext& c, float3 o, float3 d, Pcg32& g, int max_depth,
                           int roulette_start)
{
    float3 throughput = gray(1.0f);
    float3 result = gray(0.0f);
    float3 arrival_origin = o;
    float arrival_pdf = 0.0f;
    bool arrival_specular = true;
    SkipRule skip = SkipRule::none();
    const float choice = s.light_count > 0u ? 1.0f / static_cast<float>(s.light_count) : INFINITY;
    for (int depth = 0;; ++depth) {
        TraceHit hit;
        if (!closestHit(s, c, o, d, skip, hit)) {
            if (s.sky_light >= 0) {
                float3 e = skyRadiance(s.lights[s.sky_light], d);
                if (!isBlack(e) && !arrival_specular) {
                    e = e * powerHeuristic(arrival_pdf, choice * uniformSpherePdf());
                }
                result = result + throughput * e;
            }
            return result;
        }
        Surface sf;
        resolveHit(s, o, d, hit, sf);
        const int light_index = s.object_light[sf.object_id];
        if (light_index >= 0 && sf.front) {
            const DevLight light = s.lights[light_index];
            float3 e = ld3(light.e);
            if (!isBlack(e) && !arrival_specular) {
                e = e * powerHeuristic(arrival_pdf, choice * lightPdf(light, arrival_origin, d));
            }
            result = result + throughput * e;
        }
        if (depth >= max_depth) {
            return result;
        }
        const Scattering sc = scatteringAt(s, sf);
        const float3 wo = -d;
        result = result + throughput * sampleDirectLight(s, c, sf, sc, wo, g);
        const float u_choice = g.next1D();
        const float ux = g.next1D();
        const float uy = g.next1D();
        ScatterSample smp;
        if (!sc.sample(wo, u_choice, ux, uy, smp)) {
            return result;
        }
        throughput = throughput * smp.weight;
        if (isBlack(throughput)) {
            return result;
        }
        if (depth >= roulette_start) {
            const float survival = fminf(0.95f, fmaxf(throughput.x, fmaxf(throughput.y, throughput.z)));
            if (g.next1D() >= survival) {
                return result;
            }
            throughput = throughput / survival;
        }
        arrival_origin = sf.p;
        arrival_pdf = smp.pdf;
        arrival_specular = smp.specular;
        rayLeaving(sf, smp.dir, o, skip);
        d = smp.dir;
    }
}

ALB_DEV float3 scatterOnlyRadiance(const DevScene& s, const TraceContext& c, float3 o, float3 d, Pcg32& g,
                                   int max_scatter)
{
    float3 throughput = gray(1.0f);
    float3 result = gray(0.0f);
    SkipRule skip = SkipRule::none();
    for (int count = 0;; ++count) {
        TraceHit hit;
        if (!closestHit(s, c, o, d, skip, hit)) {
            if (s.sky_light >= 0) {
                result = result + throughput * skyRadiance(s.lights[s.sky_light], d);
            }
            return result;
        }
        Surface sf;
        resolveHit(s, o, d, hit, sf);
        const int light_index = s.object_light[sf.object_id];
        if (light_index >= 0 && sf.front) {
            result = result + throughput * ld3(s.lights[light_index].e);
        }
        if (count >= max_scatter) {
            return result;
        }
        const float u_choice = g.next1D();
        const float ux = g.next1D();
        const float uy = g.next1D();
        ScatterSample smp;
        if (!scatteringAt(s, sf).sample(-d, u_choice, ux, uy, smp)) {
            return result;
        }
        throughput = throughput * smp.weight;
        if (isBlack(throughput)) {
            return result;
        }
        rayLeaving(sf, smp.dir, o, skip);
        d = smp.dir;
    }
}

ALB_DEV float3 normalsRadiance(const DevScene& s, const TraceContext& c, float3 o, float3 d)
{
    TraceHit hit;
    if (closestHit(s, c, o, d, SkipRule::none(), hit)) {
        Surface sf;
        resolveHit(s, o, d, hit, sf);
        return mk(0.5f * (sf.ns.x + 1.0f), 0.5f * (sf.ns.y + 1.0f), 0.5f * (sf.ns.z + 1.0f));
    }
    const float h = 0.5f * (normalized(d).y + 1.0f);
    return gray(1.0f) * (1.0f - h) + mk(0.5f, 0.7f, 1.0f) * h;
}

template <int EST>
ALB_DEV float3 estimateRadiance(const DevScene& s, const TraceContext& c, float3 o, float3 d, Pcg32& g,
                                const RenderArgs& a)
{
    if constexpr (EST == kEstimatorPath) {
        return pathRadiance(s, c, o, d, g, a.max_depth, a.roulette_start);
    } else if constexpr (EST == kEstimatorScatterOnly) {
        return scatterOnlyRadiance(s, c, o, d, g, a.max_depth);
    } else {
        return normalsRadiance(s, c, o, d);
    }
}

} // namespace albedo_b200
