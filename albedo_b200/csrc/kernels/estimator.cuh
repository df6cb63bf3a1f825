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

// Where a thread's queries keep their stack, and how they are traced: INLINE
// places the closest-hit traversal in the calling kernel, INLINE_SHADOW the
// shadow queries' traversal (by default as INLINE), COUNT counts the work into
// `counts` (traceScene). Stack entries are uint2 (child reference and entry
// distance) or unsigned (the reference alone).
template <bool INLINE, bool COUNT = false, bool INLINE_SHADOW = INLINE, typename Stack = uint2>
struct TraceContext {
    static constexpr bool kInline = INLINE;
    static constexpr bool kInlineShadow = INLINE_SHADOW;
    static constexpr bool kCount = COUNT;
    Stack* stack;
    int stride;
    int capacity;
    unsigned int* error_flag;
    TraversalCounts* counts; // null except in the counting variants
};

template <typename Ctx>
ALB_DEV bool closestHit(const DevScene& s, const Ctx& c, float3 o, float3 d, const SkipRule& skip, TraceHit& hit)
{
    float tmax = INFINITY;
    return traceScene<false, Ctx::kInline, Ctx::kCount>(s, o, d, 0.0f, tmax, skip, hit, c.stack, c.stride,
                                                        c.capacity, c.error_flag, c.counts);
}

template <typename Ctx>
ALB_DEV bool occluded(const DevScene& s, const Ctx& c, float3 o, float3 d, float tmax, const SkipRule& skip)
{
    TraceHit hit;
    return traceScene<true, Ctx::kInlineShadow, Ctx::kCount>(s, o, d, 0.0f, tmax, skip, hit, c.stack, c.stride,
                                                             c.capacity, c.error_flag, c.counts);
}

// Next-event estimation from one uniformly chosen light, MIS-weighted, before
// the shadow test: what sampleDirectLight computes up to Scene::occluded. The
// contribution is not yet scaled by the path throughput.
struct NeeCandidate {
    bool valid;         // a non-zero contribution exists
    bool needs_test;    // a shadow ray must confirm it (the range is not empty)
    float3 contribution;
    float3 origin;
    float3 dir;
    float range_max;
    SkipRule skip;
};

ALB_DEV NeeCandidate directLightCandidate(const DevScene& s, const Surface& sf, const Scattering& sc, float3 wo,
                                          Pcg32& g)
{
    NeeCandidate nc;
    nc.valid = false;
    nc.needs_test = false;
    const float u_light = g.next1D();
    const float ux = g.next1D();
    const float uy = g.next1D();
    if (s.light_count == 0u) {
        return nc;
    }
    const int n = static_cast<int>(s.light_count);
    const int index = min(static_cast<int>(u_light * static_cast<float>(n)), n - 1);
    const DevLight light = s.lights[index];
    LightSample ls;
    if (!sampleLight(light, sf.p, ux, uy, ls) || isBlack(ls.radiance)) {
        return nc;
    }
    const float3 f = sc.evaluate(wo, ls.dir);
    if (isBlack(f)) {
        return nc;
    }
    const float range_max = shadowRangeMax(ls.distance);
    if (range_max > 0.0f) {
        nc.needs_test = true;
        rayLeaving(sf, ls.dir, nc.origin, nc.skip);
        if (light.kind == kLightArea) {
            nc.skip.light_object_pos = light.object;
        }
        nc.dir = ls.dir;
        nc.range_max = range_max;
    }
    const float light_pdf = (1.0f / static_cast<float>(n)) * ls.pdf;
    const float weight = ls.delta ? 1.0f : powerHeuristic(light_pdf, sc.pdf(wo, ls.dir));
    const float cos_theta = fabsf(dot(ls.dir, sf.ns));
    nc.contribution = f * ls.radiance * (cos_theta * weight / light_pdf);
    nc.valid = true;
    return nc;
}

// The state of one path between bounces: PathEstimator::radiance's loop
// variables (estimator/path_estimator.cpp:155-160) plus the skip rule of the ray.
struct PathState {
    float3 o;
    float3 d;
    float3 throughput;
    float3 result;
    float3 arrival_origin;
    float arrival_pdf;
    int depth;
    bool arrival_specular;
    SkipRule skip;
};

ALB_DEV void beginPath(PathState& p, float3 o, float3 d)
{
    p.o = o;
    p.d = d;
    p.throughput = gray(1.0f);
    p.result = gray(0.0f);
    p.arrival_origin = o;
    p.arrival_pdf = 0.0f;
    p.depth = 0;
    p.arrival_specular = true;
    p.skip = SkipRule::none();
}

// Emission seen at a surface along the path's ray, MIS-weighted against light
// sampling at the previous vertex (weightedEmission).
ALB_DEV float3 weightedEmission(const DevScene& s, const PathState& p, const Surface& sf)
{
    const int light_index = s.object_light[sf.object_id];
    if (light_index < 0 || !sf.front) {
        return gray(0.0f);
    }
    const DevLight light = s.lights[light_index];
    float3 e = ld3(light.e);
    if (!isBlack(e) && !p.arrival_specular) {
        e = e * powerHeuristic(p.arrival_pdf, (1.0f / static_cast<float>(s.light_count)) *
                                                  lightPdf(light, p.arrival_origin, p.d));
    }
    return e;
}

// The sky seen by an escaping path, MIS-weighted likewise (weightedSky).
ALB_DEV float3 weightedSky(const DevScene& s, const PathState& p)
{
    if (s.sky_light < 0) {
        return gray(0.0f);
    }
    float3 e = skyRadiance(s.lights[s.sky_light], p.d);
    if (!isBlack(e) && !p.arrival_specular) {
        e = e * powerHeuristic(p.arrival_pdf, (1.0f / static_cast<float>(s.light_count)) * uniformSpherePdf());
    }
    return e;
}

// The part of a bounce after the surface is known: next-event estimation, BSDF
// sampling and roulette. Returns false when the path ends.
//
// The light sample's shadow query runs last, once the path's next ray is
// known: it draws no random numbers and its contribution is added to the
// result exactly as before the BSDF sample (the sample never touches the
// result), but the surface and its scattering are then dead, so the traversal
// call does not carry them.
template <typename Ctx>
ALB_DEV bool scatterAtSurface(const DevScene& s, const Ctx& c, PathState& p, const Surface& sf, Pcg32& g,
                              int roulette_start)
{
    const float3 throughput_here = p.throughput;
    NeeCandidate nc;
    bool alive = true;
    {
        const Scattering sc = scatteringAt(s, sf);
        const float3 wo = -p.d;
        nc = directLightCandidate(s, sf, sc, wo, g);
        const float u_choice = g.next1D();
        const float ux = g.next1D();
        const float uy = g.next1D();
        ScatterSample smp;
        if (!sc.sample(wo, u_choice, ux, uy, smp)) {
            alive = false;
        } else {
            p.throughput = p.throughput * smp.weight;
            if (isBlack(p.throughput)) {
                alive = false;
            } else {
                if (p.depth >= roulette_start) {
                    const float survival =
                        fminf(0.95f, fmaxf(p.throughput.x, fmaxf(p.throughput.y, p.throughput.z)));
                    if (g.next1D() >= survival) {
                        alive = false;
                    } else {
                        p.throughput = p.throughput / survival;
                    }
                }
                if (alive) {
                    p.arrival_origin = sf.p;
                    p.arrival_pdf = smp.pdf;
                    p.arrival_specular = smp.specular;
                    rayLeaving(sf, smp.dir, p.o, p.skip);
                    p.d = smp.dir;
                    ++p.depth;
                }
            }
        }
    }
    const bool lit = nc.valid && !(nc.needs_test && occluded(s, c, nc.origin, nc.dir, nc.range_max, nc.skip));
    p.result = p.result + throughput_here * (lit ? nc.contribution : gray(0.0f));
    return alive;
}

// One iteration of PathEstimator::radiance's loop. Returns false when the path
// has ended; p.result then holds its radiance.
template <typename Ctx>
ALB_DEV bool pathBounce(const DevScene& s, const Ctx& c, PathState& p, Pcg32& g, int max_depth,
                        int roulette_start)
{
    TraceHit hit;
    if (!closestHit(s, c, p.o, p.d, p.skip, hit)) {
        p.result = p.result + p.throughput * weightedSky(s, p);
        return false;
    }
    Surface sf;
    resolveHit(s, p.o, p.d, hit, sf);
    p.result = p.result + p.throughput * weightedEmission(s, p, sf);
    if (p.depth >= max_depth) {
        return false;
    }
    return scatterAtSurface(s, c, p, sf, g, roulette_start);
}

// One iteration of ScatterOnlyEstimator::radiance's loop
// (estimator/scatter_only_estimator.cpp:14-48).
template <typename Ctx>
ALB_DEV bool scatterOnlyBounce(const DevScene& s, const Ctx& c, PathState& p, Pcg32& g, int max_scatter)
{
    TraceHit hit;
    if (!closestHit(s, c, p.o, p.d, p.skip, hit)) {
        if (s.sky_light >= 0) {
            p.result = p.result + p.throughput * skyRadiance(s.lights[s.sky_light], p.d);
        }
        return false;
    }
    Surface sf;
    resolveHit(s, p.o, p.d, hit, sf);
    const int light_index = s.object_light[sf.object_id];
    if (light_index >= 0 && sf.front) {
        p.result = p.result + p.throughput * ld3(s.lights[light_index].e);
    }
    if (p.depth >= max_scatter) {
        return false;
    }
    const float u_choice = g.next1D();
    const float ux = g.next1D();
    const float uy = g.next1D();
    ScatterSample smp;
    if (!scatteringAt(s, sf).sample(-p.d, u_choice, ux, uy, smp)) {
        return false;
    }
    p.throughput = p.throughput * smp.weight;
    if (isBlack(p.throughput)) {
        return false;
    }
    rayLeaving(sf, smp.dir, p.o, p.skip);
    p.d = smp.dir;
    ++p.depth;
    return true;
}

// NormalsEstimator::radiance (estimator/normals_estimator.cpp:32-38): one query.
template <typename Ctx>
ALB_DEV bool normalsBounce(const DevScene& s, const Ctx& c, PathState& p)
{
    TraceHit hit;
    if (closestHit(s, c, p.o, p.d, SkipRule::none(), hit)) {
        Surface sf;
        resolveHit(s, p.o, p.d, hit, sf);
        p.result = mk(0.5f * (sf.ns.x + 1.0f), 0.5f * (sf.ns.y + 1.0f), 0.5f * (sf.ns.z + 1.0f));
    } else {
        const float h = 0.5f * (normalized(p.d).y + 1.0f);
        p.result = gray(1.0f) * (1.0f - h) + mk(0.5f, 0.7f, 1.0f) * h;
    }
    return false;
}

template <int EST, typename Ctx>
ALB_DEV bool estimatorBounce(const DevScene& s, const Ctx& c, PathState& p, Pcg32& g, const RenderArgs& a)
{
    if constexpr (EST == kEstimatorPath) {
        return pathBounce(s, c, p, g, a.max_depth, a.roulette_start);
    } else if constexpr (EST == kEstimatorScatterOnly) {
        return scatterOnlyBounce(s, c, p, g, a.max_depth);
    } else {
        return normalsBounce(s, c, p);
    }
}

// Draws sample `index` of a pixel's n x n grid (row-major cells, x jitter then y,
// render/render_image.cpp:32-40) and starts its camera path.
ALB_DEV void startSample(const DevCamera& cam, PathState& p, Pcg32& g, int x, int y, int index, int n, float inv_n,
                         float width, float height)
{
    const int sy = index / n;
    const int sx = index - sy * n;
    const float jx = g.next1D();
    const float jy = g.next1D();
    const float fx = (static_cast<float>(x) + (static_cast<float>(sx) + jx) * inv_n) / width;
    const float fy = (static_cast<float>(y) + (static_cast<float>(sy) + jy) * inv_n) / height;
    float3 o, d;
    cameraRay(cam, fx, fy, o, d);
    beginPath(p, o, d);
}

} // namespace albedo_b200
