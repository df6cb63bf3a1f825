// albedo_b200_adapter.hpp: the reference's render call, on the GPU.
//
// A header-only C++20 adapter over the C ABI in albedo_b200.h for a program
// built against the reference's own headers (src/albedo/...). It gives
//
//     void albedo_b200::renderImage(const albedo::RenderJob& job, albedo::PixelBuffer& image);
//
// the meaning of albedo::renderImage (src/albedo/render/render_image.hpp:36-49):
// the job's camera, scene, samples_per_axis, seed and estimator; n^2 samples
// ADDED to every pixel of the caller's PixelBuffer; std::invalid_argument with
// the reference's messages for a non-positive samples_per_axis or thread_count
// (render/render_image.cpp:60-67). thread_count is checked and otherwise
// ignored: the image does not depend on it in either renderer.
//
// The reference's Scene keeps its objects private (scene/scene.hpp:94-97), so
// the GPU cannot be handed one. Instead a program binds each Scene it read from
// a file to a GPU copy of the same file:
//
//     const albedo::SceneDescription description{albedo::readScene(path)};
//     albedo_b200::bindScene(description.scene, path);   // one added line
//     ...
//     albedo_b200::renderImage(job, image);               // was albedo::renderImage
//
// The GPU copy is read by this library's reader, which accepts, refuses and
// orders a file exactly as readScene does, so object ids, lights and BVHs are
// the reference's.
//
// The camera. PerspectiveCamera keeps its frame private too
// (camera/perspective_camera.hpp:42-53), so the adapter recovers the camera's
// settings from rays it generates: the ray through the film centre gives the
// position and view direction, the rays through the middles of the right and
// top edges give the half extents of the film, hence the field of view, the up
// direction and the aspect ratio. The device builds its frame from those
// settings with the image's width / height as aspect ratio; a camera built for
// another aspect ratio is refused with std::invalid_argument.
//
// The pixels. PixelBuffer keeps its {Rgb sum; int64 count} accumulators
// private (image/pixel_buffer.hpp:53-57) and adds samples one at a time through
// addSample. The adapter renders into a host array of the same layout and then
// adds each pixel's GPU sum with one addSample and its remaining n^2 - 1
// samples as zeros, which leaves the pixel's sum exactly `sum + gpu_sum` and
// its count `count + n^2`, as a direct update would. That host loop costs about
// a nanosecond per sample; a PixelBuffer member adding a sum and a count at once
// (one added line in the reference: `void addSamples(Point2i, Rgb sum,
// std::int64_t count) noexcept;`) would remove it. Define
// ALBEDO_B200_PIXEL_BUFFER_ADD_SAMPLES when the reference has that member.
//
// Errors become the reference's exception types (albedo_b200::check).
#ifndef ALBEDO_B200_ADAPTER_HPP
#define ALBEDO_B200_ADAPTER_HPP

#include "albedo/camera/perspective_camera.hpp"
#include "albedo/estimator/normals_estimator.hpp"
#include "albedo/estimator/path_estimator.hpp"
#include "albedo/estimator/scatter_only_estimator.hpp"
#include "albedo/image/pixel_buffer.hpp"
#include "albedo/render/render_image.hpp"
#include "albedo/scene/scene.hpp"
#include "albedo_b200.h"

#include <cmath>
#include <cstddef>
#include <filesystem>
#include <format>
#include <map>
#include <memory>
#include <mutex>
#include <numbers>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <variant>
#include <vector>

namespace albedo_b200 {

// Throws the exception the reference throws for the failure a status reports.
inline void check(int status)
{
    if (status == ALBEDO_OK) {
        return;
    }
    const std::string message{albedo_last_error()};
    switch (status) {
    case ALBEDO_INVALID_ARGUMENT:
        throw std::invalid_argument{message};
    case ALBEDO_OUT_OF_RANGE:
        throw std::out_of_range{message};
    default:
        // Parse and I/O failures, device failures and unsupported scenes.
        throw std::runtime_error{message};
    }
}

// A scene file read and made resident on the current CUDA device.
class GpuScene {
public:
    explicit GpuScene(const std::filesystem::path& path) { check(albedo_scene_load(path.string().c_str(), &handle)); }
    GpuScene(const GpuScene&) = delete;
    GpuScene& operator=(const GpuScene&) = delete;
    ~GpuScene() { albedo_scene_destroy(handle); }
    const albedo_scene* get() const noexcept { return handle; }

private:
    albedo_scene* handle{nullptr};
};

namespace detail {

struct Bindings {
    std::mutex mutex;
    std::map<const albedo::Scene*, std::shared_ptr<GpuScene>> scenes;
};

inline Bindings& bindings()
{
    static Bindings table;
    return table;
}

inline std::shared_ptr<GpuScene> boundTo(const albedo::Scene& scene)
{
    Bindings& table{bindings()};
    const std::lock_guard lock{table.mutex};
    const auto found{table.scenes.find(&scene)};
    if (found == table.scenes.end()) {
        throw std::invalid_argument{"renderImage: the scene has no GPU copy; call albedo_b200::bindScene first"};
    }
    return found->second;
}

inline double dot(const albedo::Vector3r& a, const albedo::Vector3r& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

} // namespace detail

// Binds `scene`, which albedo::readScene read from `path`, to a GPU copy of
// that file; renderImage renders jobs on `scene` from the copy. Rebinding
// replaces the copy. The binding is by address: unbind before the Scene dies.
inline void bindScene(const albedo::Scene& scene, const std::filesystem::path& path)
{
    auto copy{std::make_shared<GpuScene>(path)};
    detail::Bindings& table{detail::bindings()};
    const std::lock_guard lock{table.mutex};
    table.scenes[&scene] = std::move(copy);
}

inline void unbindScene(const albedo::Scene& scene)
{
    detail::Bindings& table{detail::bindings()};
    const std::lock_guard lock{table.mutex};
    table.scenes.erase(&scene);
}

// CameraSettings that build `camera`'s frame, recovered from its rays, for an
// image of width / height `aspect_ratio`.
inline albedo_camera settingsOf(const albedo::PerspectiveCamera& camera, double aspect_ratio)
{
    const albedo::Ray centre{camera.generateRay({.film = {0.5, 0.5}})};
    const albedo::Ray right{camera.generateRay({.film = {1.0, 0.5}})};
    const albedo::Ray top{camera.generateRay({.film = {0.5, 0.0}})};
    const albedo::Vector3r forward{centre.direction};
    // With a unit forward vector, the ray through the right edge's middle is
    // along forward + half_width, and the top edge's along forward + half_height.
    const albedo::Vector3r half_width{right.direction / detail::dot(right.direction, forward) - forward};
    const albedo::Vector3r half_height{top.direction / detail::dot(top.direction, forward) - forward};
    const double width_extent{std::sqrt(detail::dot(half_width, half_width))};
    const double height_extent{std::sqrt(detail::dot(half_height, half_height))};
    const double camera_aspect{width_extent / height_extent};
    if (!(std::abs(camera_aspect - aspect_ratio) <= 1e-9 * aspect_ratio)) {
        throw std::invalid_argument{std::format(
            "renderImage: the camera's aspect ratio {} is not the image's {}; the GPU renderer builds the camera "
            "for the image",
            camera_aspect, aspect_ratio)};
    }
    albedo_camera settings{};
    const albedo::Point3r target{centre.origin + forward};
    for (int k{0}; k < 3; ++k) {
        const double component[3][3]{{centre.origin.x, centre.origin.y, centre.origin.z},
                                     {target.x, target.y, target.z},
                                     {half_height.x, half_height.y, half_height.z}};
        settings.look_from[k] = component[0][k];
        settings.look_at[k] = component[1][k];
        settings.up[k] = component[2][k];
    }
    settings.vertical_fov_degrees = 2 * std::atan(height_extent) * 180 / std::numbers::pi;
    return settings;
}

// The estimator fields of a C-ABI job for the job's RadianceEstimator.
inline void setEstimator(const albedo::RadianceEstimator& estimator, albedo_render_job& out)
{
    std::visit(
        [&](const auto& chosen) {
            using Chosen = std::decay_t<decltype(chosen)>;
            if constexpr (std::is_same_v<Chosen, albedo::PathEstimator>) {
                out.estimator = ALBEDO_PATH;
                out.max_depth = chosen.max_depth;
                out.roulette_start = chosen.roulette_start;
            } else if constexpr (std::is_same_v<Chosen, albedo::ScatterOnlyEstimator>) {
                out.estimator = ALBEDO_SCATTER_ONLY;
                out.max_depth = chosen.max_scatter_count;
            } else {
                static_assert(std::is_same_v<Chosen, albedo::NormalsEstimator>, "an estimator the GPU lacks");
                out.estimator = ALBEDO_NORMALS;
            }
        },
        estimator);
}

// albedo::renderImage on the GPU (see the top of this file).
inline void renderImage(const albedo::RenderJob& job, albedo::PixelBuffer& image)
{
    if (job.samples_per_axis <= 0) {
        throw std::invalid_argument{std::format("samples per axis must be positive, got {}", job.samples_per_axis)};
    }
    if (job.thread_count <= 0) {
        throw std::invalid_argument{std::format("thread count must be positive, got {}", job.thread_count)};
    }
    const std::shared_ptr<GpuScene> scene{detail::boundTo(job.scene.get())};
    const int width{image.width()};
    const int height{image.height()};
    albedo_render_job gpu_job{};
    gpu_job.width = width;
    gpu_job.height = height;
    gpu_job.samples_per_axis = job.samples_per_axis;
    gpu_job.seed = job.seed;
    gpu_job.max_depth = 64;
    gpu_job.roulette_start = 3;
    gpu_job.method = ALBEDO_MEGAKERNEL;
    gpu_job.accumulation = ALBEDO_ACCUMULATE_FP64;
    setEstimator(job.estimator, gpu_job);
    const albedo_camera camera{settingsOf(job.camera.get(), static_cast<double>(width) / height)};
    std::vector<albedo_accumulator> sums(static_cast<std::size_t>(width) * static_cast<std::size_t>(height));
    check(albedo_render_view_host(scene->get(), &gpu_job, &camera, sums.data()));
    for (int y{0}; y < height; ++y) {
        for (int x{0}; x < width; ++x) {
            const albedo_accumulator& a{sums[static_cast<std::size_t>(y) * width + x]};
            if (a.count == 0) {
                continue;
            }
            const albedo::Point2i pixel{.x = x, .y = y};
#ifdef ALBEDO_B200_PIXEL_BUFFER_ADD_SAMPLES
            image.addSamples(pixel, {.r = a.r, .g = a.g, .b = a.b}, a.count);
#else
            image.addSample(pixel, {.r = a.r, .g = a.g, .b = a.b});
            for (std::int64_t k{1}; k < a.count; ++k) {
                image.addSample(pixel, {});
            }
#endif
        }
    }
}

} // namespace albedo_b200

#endif // ALBEDO_B200_ADAPTER_HPP
