// C-ABI driver over the reference renderer's public C++ API (test infrastructure).
//
// This file is compiled by oracle/Makefile together with the reference sources,
// unmodified, into oracle/_ref/libalbedo_ref.so. It is the checker that the
// parity tests and the CPU baseline call; nothing in the product links it.
// Every entry point only calls public reference API:
//   readScene                         scene/scene_file.hpp:133-146
//   Scene::add (shapes, TriangleMesh)  scene/scene.hpp:31-62
//   renderImage / RenderJob           render/render_image.hpp:17-49
//   SampleGenerator::forPixel         sampling/sample_generator.hpp:35-45
//   PerspectiveCamera::generateRay    camera/perspective_camera.cpp:74-87
//   PathEstimator::radiance           estimator/path_estimator.cpp:153-185
//   Scene::intersect / occluded       scene/scene.cpp:107-133, 157-165
//   lobes, Fresnel, warps, noise      scattering/*.cpp, sampling/warps.cpp, texture/*.cpp
// The per-pixel loop in ref_render_pixels restates render/render_image.cpp:27-44
// so that sums of squares (for two-sample tests) and pixel subsets are available.

#include "albedo/camera/perspective_camera.hpp"
#include "albedo/estimator/normals_estimator.hpp"
#include "albedo/estimator/path_estimator.hpp"
#include "albedo/estimator/radiance_estimator.hpp"
#include "albedo/estimator/scatter_only_estimator.hpp"
#include "albedo/geometry/mesh_geometry.hpp"
#include "albedo/geometry/mesh_instance.hpp"
#include "albedo/geometry/sphere.hpp"
#include "albedo/geometry/triangle.hpp"
#include "albedo/geometry/triangle_mesh.hpp"
#include "albedo/color/srgb.hpp"
#include "albedo/image/pixel_buffer.hpp"
#include "albedo/image/ppm.hpp"
#include "albedo/light/area_light.hpp"
#include "albedo/render/render_image.hpp"
#include "albedo/sampling/pcg32.hpp"
#include "albedo/sampling/sample_generator.hpp"
#include "albedo/sampling/warps.hpp"
#include "albedo/scattering/conductor_lobe.hpp"
#include "albedo/scattering/dielectric_lobe.hpp"
#include "albedo/scattering/fresnel.hpp"
#include "albedo/scattering/ggx_distribution.hpp"
#include "albedo/scattering/lambert_lobe.hpp"
#include "albedo/scene/scene.hpp"
#include "albedo/scene/scene_file.hpp"
#include "albedo/texture/perlin_noise.hpp"

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <exception>
#include <filesystem>
#include <memory>
#include <string>
#include <thread>
#include <vector>

using namespace albedo;

namespace {

thread_local std::string last_error;

struct RefScene {
    SceneDescription description;
};

template <typename F>
int guarded(F&& body)
{
    try {
        body();
        return 0;
    } catch (const std::exception& error) {
        last_error = error.what();
        return 1;
    } catch (...) {
        last_error = "unknown exception";
        return 1;
    }
}

PerspectiveCamera cameraFor(const RefScene& scene, int width, int height)
{
    CameraSettings settings{scene.description.camera};
    settings.aspect_ratio = static_cast<Real>(width) / static_cast<Real>(height);
    return PerspectiveCamera{settings};
}

RadianceEstimator estimatorFor(int kind, int max_depth, int roulette_start)
{
    switch (kind) {
    case 1:
        return ScatterOnlyEstimator{.max_scatter_count = max_depth};
    case 2:
        return NormalsEstimator{};
    default:
        return PathEstimator{.max_depth = max_depth, .roulette_start = roulette_start};
    }
}

// Runs `work(i)` for i in [0, count) on `threads` threads with an atomic counter.
template <typename F>
void parallelFor(std::int64_t count, int threads, F&& work)
{
    std::atomic<std::int64_t> next{0};
    auto drain = [&] {
        for (;;) {
            const std::int64_t i{next.fetch_add(1)};
            if (i >= count) {
                return;
            }
            work(i);
        }
    };
    std::vector<std::thread> pool;
    for (int t{1}; t < threads; ++t) {
        pool.emplace_back(drain);
    }
    drain();
    for (auto& thread : pool) {
        thread.join();
    }
}

Ray rayAt(const double* rays, std::int64_t i)
{
    const double* r{rays + 6 * i};
    return Ray{.origin = {r[0], r[1], r[2]}, .direction = {r[3], r[4], r[5]}};
}

} // namespace

extern "C" {

const char* ref_last_error() { return last_error.c_str(); }

int ref_available_threads() { return availableThreadCount(); }

void* ref_scene_load(const char* path)
{
    RefScene* scene{nullptr};
    if (guarded([&] { scene = new RefScene{readScene(std::filesystem::path{path})}; }) != 0) {
        return nullptr;
    }
    return scene;
}

// A scene built through Scene's own add calls (scene/scene.hpp:31-62) instead
// of a file: ref_scene_create, then ref_scene_add_triangles (Scene::add of a
// TriangleMesh: every triangle its own object, scene/scene.cpp:33-61) and
// ref_scene_add_sphere in any order. Materials are black diffuse: these scenes
// serve ray queries.
void* ref_scene_create()
{
    RefScene* scene{nullptr};
    if (guarded([&] { scene = new RefScene{}; }) != 0) {
        return nullptr;
    }
    return scene;
}

int ref_scene_add_triangles(void* handle, const double* positions, std::int64_t position_count,
                            const std::int64_t* faces, std::int64_t face_count)
{
    return guarded([&] {
        std::vector<Point3r> points;
        points.reserve(static_cast<std::size_t>(position_count));
        for (std::int64_t i{0}; i < position_count; ++i) {
            points.push_back({positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]});
        }
        std::vector<TriangleMesh::Face> corners;
        corners.reserve(static_cast<std::size_t>(face_count));
        for (std::int64_t f{0}; f < face_count; ++f) {
            corners.push_back({static_cast<std::size_t>(faces[3 * f]), static_cast<std::size_t>(faces[3 * f + 1]),
                               static_cast<std::size_t>(faces[3 * f + 2])});
        }
        static_cast<RefScene*>(handle)->description.scene.add(TriangleMesh{std::move(points), std::move(corners)},
                                                              Material{DiffuseMaterial{}});
    });
}

int ref_scene_add_sphere(void* handle, const double* center, double radius)
{
    return guarded([&] {
        static_cast<RefScene*>(handle)->description.scene.add(Sphere{{center[0], center[1], center[2]}, radius},
                                                              Material{DiffuseMaterial{}});
    });
}

void ref_scene_free(void* handle) { delete static_cast<RefScene*>(handle); }

std::int64_t ref_scene_object_count(void* handle)
{
    return static_cast<std::int64_t>(static_cast<RefScene*>(handle)->description.scene.shapeCount());
}

// The reference's own entry point: renderImage into a PixelBuffer, returning the
// per-pixel averages (W*H*3 doubles, row-major from the top-left pixel).
int ref_render_image(void* handle, int width, int height, int samples_per_axis,
                     std::uint64_t seed, int max_depth, int roulette_start, int threads,
                     double* out_average)
{
    return guarded([&] {
        const RefScene& scene{*static_cast<RefScene*>(handle)};
        const PerspectiveCamera camera{cameraFor(scene, width, height)};
        PixelBuffer image{width, height};
        renderImage(RenderJob{.camera = camera,
                              .scene = scene.description.scene,
                              .samples_per_axis = samples_per_axis,
                              .seed = seed,
                              .estimator = PathEstimator{.max_depth = max_depth,
                                                         .roulette_start = roulette_start},
                              .thread_count = threads},
                    image);
        if (out_average != nullptr) {
            for (int y{0}; y < height; ++y) {
                for (int x{0}; x < width; ++x) {
                    const Rgb average{image.average({.x = x, .y = y})};
                    double* out{out_average + 3 * (static_cast<std::int64_t>(y) * width + x)};
                    out[0] = average.r;
                    out[1] = average.g;
                    out[2] = average.b;
                }
            }
        }
    });
}

// The per-pixel sample loop of render/render_image.cpp:27-44 over a list of
// pixels (x, y pairs), accumulating sums and sums of squares per pixel.
// estimator: 0 = PathEstimator, 1 = ScatterOnlyEstimator, 2 = NormalsEstimator.
int ref_render_pixels(void* handle, int width, int height, int samples_per_axis,
                      std::uint64_t seed, int estimator, int max_depth, int roulette_start,
                      int threads, const std::int32_t* pixels, std::int64_t pixel_count,
                      double* out_sum, double* out_sum_squares)
{
    return guarded([&] {
        const RefScene& scene{*static_cast<RefScene*>(handle)};
        const PerspectiveCamera camera{cameraFor(scene, width, height)};
        const RadianceEstimator chosen{estimatorFor(estimator, max_depth, roulette_start)};
        const Real w{static_cast<Real>(width)};
        const Real h{static_cast<Real>(height)};
        const int n{samples_per_axis};
        parallelFor(pixel_count, threads, [&](std::int64_t i) {
            const Point2i pixel{.x = pixels[2 * i], .y = pixels[2 * i + 1]};
            SampleGenerator generator{SampleGenerator::forPixel(seed, pixel, width)};
            Rgb sum{};
            Rgb squares{};
            for (int sy{0}; sy < n; ++sy) {
                for (int sx{0}; sx < n; ++sx) {
                    const Point2r jitter{generator.next2D()};
                    const Real offset_x{(sx + jitter.x) / n};
                    const Real offset_y{(sy + jitter.y) / n};
                    const PixelSample sample{
                        .film = {(pixel.x + offset_x) / w, (pixel.y + offset_y) / h}};
                    const Rgb value{radiance(chosen, camera.generateRay(sample),
                                             scene.description.scene, generator)};
                    sum += value;
                    squares += value * value;
                }
            }
            out_sum[3 * i] = sum.r;
            out_sum[3 * i + 1] = sum.g;
            out_sum[3 * i + 2] = sum.b;
            if (out_sum_squares != nullptr) {
                out_sum_squares[3 * i] = squares.r;
                out_sum_squares[3 * i + 1] = squares.g;
                out_sum_squares[3 * i + 2] = squares.b;
            }
        });
    });
}

// Scene::intersect for N rays (6 doubles each) over (t_min, t_max).
int ref_intersect(void* handle, const double* rays, std::int64_t count, double t_min,
                  double t_max, int threads, std::int32_t* out_hit, double* out_t,
                  std::int64_t* out_object, double* out_point, double* out_normal,
                  double* out_shading_normal, std::int32_t* out_front, double* out_uv)
{
    return guarded([&] {
        const Scene& scene{static_cast<RefScene*>(handle)->description.scene};
        parallelFor(count, threads, [&](std::int64_t i) {
            const auto hit{scene.intersect(rayAt(rays, i), Interval{.min = t_min, .max = t_max})};
            out_hit[i] = hit ? 1 : 0;
            if (!hit) {
                return;
            }
            out_t[i] = hit->t;
            out_object[i] = static_cast<std::int64_t>(hit->object);
            if (out_point != nullptr) {
                out_point[3 * i] = hit->point.x;
                out_point[3 * i + 1] = hit->point.y;
                out_point[3 * i + 2] = hit->point.z;
            }
            if (out_normal != nullptr) {
                out_normal[3 * i] = hit->normal.x;
                out_normal[3 * i + 1] = hit->normal.y;
                out_normal[3 * i + 2] = hit->normal.z;
            }
            if (out_shading_normal != nullptr) {
                out_shading_normal[3 * i] = hit->shading_normal.x;
                out_shading_normal[3 * i + 1] = hit->shading_normal.y;
                out_shading_normal[3 * i + 2] = hit->shading_normal.z;
            }
            if (out_front != nullptr) {
                out_front[i] = hit->front_face ? 1 : 0;
            }
            if (out_uv != nullptr) {
                out_uv[2 * i] = hit->uv.x;
                out_uv[2 * i + 1] = hit->uv.y;
            }
        });
    });
}

// Scene::occluded for N rays over (0, t_max[i]).
int ref_occluded(void* handle, const double* rays, const double* t_max, std::int64_t count,
                 int threads, std::int32_t* out_occluded)
{
    return guarded([&] {
        const Scene& scene{static_cast<RefScene*>(handle)->description.scene};
        parallelFor(count, threads, [&](std::int64_t i) {
            out_occluded[i] =
                scene.occluded(rayAt(rays, i), Interval{.min = 0, .max = t_max[i]}) ? 1 : 0;
        });
    });
}

// Camera rays through film positions (N pairs) for an image of width x height.
int ref_camera_rays(void* handle, int width, int height, const double* film, std::int64_t count,
                    double* out_rays)
{
    return guarded([&] {
        const PerspectiveCamera camera{cameraFor(*static_cast<RefScene*>(handle), width, height)};
        for (std::int64_t i{0}; i < count; ++i) {
            const Ray ray{camera.generateRay({.film = {film[2 * i], film[2 * i + 1]}})};
            double* out{out_rays + 6 * i};
            out[0] = ray.origin.x;
            out[1] = ray.origin.y;
            out[2] = ray.origin.z;
            out[3] = ray.direction.x;
            out[4] = ray.direction.y;
            out[5] = ray.direction.z;
        }
    });
}

// The first `count` outputs of Pcg32{seed, stream}.
void ref_pcg32(std::uint64_t seed, std::uint64_t stream, std::int64_t count, std::uint32_t* out)
{
    Pcg32 generator{{.seed = seed, .stream = stream}};
    for (std::int64_t i{0}; i < count; ++i) {
        out[i] = generator.nextUint32();
    }
}

// The first `count` next1D values of SampleGenerator::forPixel(seed, (x, y), width).
void ref_pixel_stream(std::uint64_t seed, int x, int y, int width, std::int64_t count,
                      double* out)
{
    SampleGenerator generator{SampleGenerator::forPixel(seed, {.x = x, .y = y}, width)};
    for (std::int64_t i{0}; i < count; ++i) {
        out[i] = generator.next1D();
    }
}

void ref_perlin_noise(const double* points, std::int64_t count, double* out_noise,
                      double* out_turbulence)
{
    for (std::int64_t i{0}; i < count; ++i) {
        const Point3r p{points[3 * i], points[3 * i + 1], points[3 * i + 2]};
        out_noise[i] = perlinNoise(p);
        out_turbulence[i] = turbulence(p);
    }
}

// Lobe evaluation in local space. kind: 0 Lambert (params: albedo rgb),
// 1 conductor (eta rgb, k rgb, alpha), 2 dielectric (eta, alpha).
// For each of N (wo, wi) pairs: f (3), pdf (1).
int ref_lobe_eval(int kind, const double* params, const double* wo_wi, std::int64_t count,
                  double* out_f, double* out_pdf)
{
    return guarded([&] {
        for (std::int64_t i{0}; i < count; ++i) {
            const double* v{wo_wi + 6 * i};
            const Vector3r wo{v[0], v[1], v[2]};
            const Vector3r wi{v[3], v[4], v[5]};
            Rgb f{};
            Real pdf{};
            if (kind == 0) {
                const LambertLobe lobe{.albedo = {params[0], params[1], params[2]}};
                f = lobe.evaluate(wo, wi);
                pdf = LambertLobe::pdf(wo, wi);
            } else if (kind == 1) {
                const ConductorLobe lobe{.eta = {params[0], params[1], params[2]},
                                         .k = {params[3], params[4], params[5]},
                                         .alpha = params[6]};
                f = lobe.evaluate(wo, wi);
                pdf = lobe.pdf(wo, wi);
            } else {
                const DielectricLobe lobe{.eta = params[0], .alpha = params[1]};
                f = lobe.evaluate(wo, wi);
                pdf = lobe.pdf(wo, wi);
            }
            out_f[3 * i] = f.r;
            out_f[3 * i + 1] = f.g;
            out_f[3 * i + 2] = f.b;
            out_pdf[i] = pdf;
        }
    });
}

// Lobe sampling in local space: inputs per sample are wo (3), u_choice, u (2).
// Outputs: valid flag, direction (3), weight (3), pdf, specular flag.
int ref_lobe_sample(int kind, const double* params, const double* inputs, std::int64_t count,
                    std::int32_t* out_valid, double* out_direction, double* out_weight,
                    double* out_pdf, std::int32_t* out_specular)
{
    return guarded([&] {
        for (std::int64_t i{0}; i < count; ++i) {
            const double* v{inputs + 6 * i};
            const Vector3r wo{v[0], v[1], v[2]};
            const Point2r u{v[4], v[5]};
            std::optional<ScatterSample> s;
            if (kind == 0) {
                s = LambertLobe{.albedo = {params[0], params[1], params[2]}}.sample(wo, v[3], u);
            } else if (kind == 1) {
                s = ConductorLobe{.eta = {params[0], params[1], params[2]},
                                  .k = {params[3], params[4], params[5]},
                                  .alpha = params[6]}
                        .sample(wo, v[3], u);
            } else {
                s = DielectricLobe{.eta = params[0], .alpha = params[1]}.sample(wo, v[3], u);
            }
            out_valid[i] = s ? 1 : 0;
            if (!s) {
                continue;
            }
            out_direction[3 * i] = s->direction.x;
            out_direction[3 * i + 1] = s->direction.y;
            out_direction[3 * i + 2] = s->direction.z;
            out_weight[3 * i] = s->weight.r;
            out_weight[3 * i + 1] = s->weight.g;
            out_weight[3 * i + 2] = s->weight.b;
            out_pdf[i] = s->pdf;
            out_specular[i] = s->specular ? 1 : 0;
        }
    });
}

void ref_fresnel_dielectric(const double* cos_theta, const double* eta, std::int64_t count,
                            double* out)
{
    for (std::int64_t i{0}; i < count; ++i) {
        out[i] = fresnelDielectric(cos_theta[i], eta[i]);
    }
}

void ref_fresnel_conductor(const double* cos_theta, std::int64_t count, const double* eta_k,
                           double* out)
{
    const Rgb eta{eta_k[0], eta_k[1], eta_k[2]};
    const Rgb k{eta_k[3], eta_k[4], eta_k[5]};
    for (std::int64_t i{0}; i < count; ++i) {
        const Rgb f{fresnelConductor(cos_theta[i], eta, k)};
        out[3 * i] = f.r;
        out[3 * i + 1] = f.g;
        out[3 * i + 2] = f.b;
    }
}

// Sphere::intersect on one sphere for N rays over (t_min, t_max).
void ref_sphere_intersect(const double* center_radius, const double* rays, std::int64_t count,
                          double t_min, double t_max, std::int32_t* out_hit, double* out_t)
{
    const Sphere sphere{{center_radius[0], center_radius[1], center_radius[2]}, center_radius[3]};
    for (std::int64_t i{0}; i < count; ++i) {
        const auto hit{sphere.intersect(rayAt(rays, i), Interval{.min = t_min, .max = t_max})};
        out_hit[i] = hit ? 1 : 0;
        out_t[i] = hit ? hit->t : 0.0;
    }
}

// Triangle::intersect on one triangle (9 doubles) for N rays.
void ref_triangle_intersect(const double* vertices, const double* rays, std::int64_t count,
                            double t_min, double t_max, std::int32_t* out_hit, double* out_t)
{
    const Triangle triangle{{vertices[0], vertices[1], vertices[2]},
                            {vertices[3], vertices[4], vertices[5]},
                            {vertices[6], vertices[7], vertices[8]}};
    for (std::int64_t i{0}; i < count; ++i) {
        const auto hit{triangle.intersect(rayAt(rays, i), Interval{.min = t_min, .max = t_max})};
        out_hit[i] = hit ? 1 : 0;
        out_t[i] = hit ? hit->t : 0.0;
    }
}

void ref_warps(const double* u, std::int64_t count, double* out_cosine, double* out_sphere)
{
    for (std::int64_t i{0}; i < count; ++i) {
        const Point2r p{u[2 * i], u[2 * i + 1]};
        const Vector3r c{sampleCosineHemisphere(p)};
        const Vector3r s{sampleUniformSphere(p)};
        out_cosine[3 * i] = c.x;
        out_cosine[3 * i + 1] = c.y;
        out_cosine[3 * i + 2] = c.z;
        out_sphere[3 * i] = s.x;
        out_sphere[3 * i + 1] = s.y;
        out_sphere[3 * i + 2] = s.z;
    }
}

// toByte(encodeSrgb(x)) for each value (color/srgb.cpp:18-36).
void ref_srgb_bytes(const double* linear, std::int64_t count, std::uint8_t* out)
{
    for (std::int64_t i{0}; i < count; ++i) {
        out[i] = toByte(encodeSrgb(linear[i]));
    }
}

// writePpm(path, image) (image/ppm.cpp:61-85) of a PixelBuffer whose pixels hold
// the given averages (W*H*3 doubles, rows from the top): one sample each, so
// each pixel's average is the value itself.
int ref_write_ppm(const char* path, int width, int height, const double* averages)
{
    return guarded([&] {
        PixelBuffer image{width, height};
        for (int y{0}; y < height; ++y) {
            for (int x{0}; x < width; ++x) {
                const double* v{averages + 3 * (static_cast<std::int64_t>(y) * width + x)};
                image.addSample({.x = x, .y = y}, Rgb{v[0], v[1], v[2]});
            }
        }
        writePpm(std::filesystem::path{path}, image);
    });
}

} // extern "C"
