// Test harness for include/albedo_b200_adapter.hpp: built against the
// reference's own headers and library (oracle/Makefile, target `adapter`) and
// called from tests/test_adapter.py and tests/test_gpu_adapter.py through ctypes.
#include "albedo/camera/perspective_camera.hpp"
#include "albedo/estimator/normals_estimator.hpp"
#include "albedo/estimator/path_estimator.hpp"
#include "albedo/estimator/scatter_only_estimator.hpp"
#include "albedo/image/pixel_buffer.hpp"
#include "albedo/render/render_image.hpp"
#include "albedo/scene/scene_file.hpp"
#include "albedo_b200_adapter.hpp"

#include <cstdint>
#include <cstring>
#include <exception>
#include <filesystem>
#include <string>

namespace {

thread_local std::string message;

albedo::PerspectiveCamera cameraFor(const albedo::SceneDescription& description, int width, int height)
{
    albedo::CameraSettings settings{description.camera};
    settings.aspect_ratio = static_cast<double>(width) / height;
    return albedo::PerspectiveCamera{settings};
}

albedo::RadianceEstimator estimatorFor(int kind, int max_depth)
{
    switch (kind) {
    case 1:
        return albedo::ScatterOnlyEstimator{.max_scatter_count = max_depth};
    case 2:
        return albedo::NormalsEstimator{};
    default:
        return albedo::PathEstimator{.max_depth = max_depth, .roulette_start = 3};
    }
}

} // namespace

extern "C" {

const char* adapter_message() { return message.c_str(); }

// The settings the adapter recovers from the scene file's camera at width x
// height, next to the file's own: out[0..9] recovered look_from, look_at, up,
// fov; out[10..19] the file's.
int adapter_camera(const char* path, int width, int height, double* out)
{
    try {
        const albedo::SceneDescription description{albedo::readScene(std::filesystem::path{path})};
        const albedo::PerspectiveCamera camera{cameraFor(description, width, height)};
        const albedo_camera got{albedo_b200::settingsOf(camera, static_cast<double>(width) / height)};
        const albedo::CameraSettings& file{description.camera};
        const double mine[10]{got.look_from[0], got.look_from[1], got.look_from[2], got.look_at[0], got.look_at[1],
                              got.look_at[2], got.up[0], got.up[1], got.up[2], got.vertical_fov_degrees};
        const double theirs[10]{file.look_from.x, file.look_from.y, file.look_from.z, file.look_at.x, file.look_at.y,
                                file.look_at.z, file.up.x, file.up.y, file.up.z, file.vertical_fov_degrees};
        std::memcpy(out, mine, sizeof mine);
        std::memcpy(out + 10, theirs, sizeof theirs);
        return 0;
    } catch (const std::exception& error) {
        message = error.what();
        return 1;
    }
}

// One render job through the adapter (`gpu` != 0) or the reference's own
// renderImage (`gpu` == 0), with the given samples_per_axis and thread_count
// (which may be invalid), the scene bound (`bind` != 0) or not, and the camera
// built for `camera_width` x height (another width tests the aspect check).
// Returns 0 and the per-pixel averages (width * height * 3), or 1 with the
// exception's type (1 invalid_argument, 2 runtime_error, 3 other) in *kind and
// its message in adapter_message().
int adapter_render(const char* path, int gpu, int bind, int width, int height, int camera_width, int samples_per_axis,
                   std::uint64_t seed, int estimator, int max_depth, int thread_count, int prior_samples,
                   double* out_average, std::int64_t* out_count, int* kind)
{
    try {
        const albedo::SceneDescription description{albedo::readScene(std::filesystem::path{path})};
        if (gpu != 0 && bind != 0) {
            albedo_b200::bindScene(description.scene, path);
        }
        const albedo::PerspectiveCamera camera{cameraFor(description, camera_width, height)};
        albedo::PixelBuffer image{width, height};
        // Samples already in the buffer: renders add to them.
        for (int k{0}; k < prior_samples; ++k) {
            image.addSample({.x = 0, .y = 0}, {.r = 1, .g = 2, .b = 3});
        }
        const albedo::RenderJob job{.camera = camera,
                                    .scene = description.scene,
                                    .samples_per_axis = samples_per_axis,
                                    .seed = seed,
                                    .estimator = estimatorFor(estimator, max_depth),
                                    .thread_count = thread_count};
        try {
            if (gpu != 0) {
                albedo_b200::renderImage(job, image);
            } else {
                albedo::renderImage(job, image);
            }
        } catch (...) {
            albedo_b200::unbindScene(description.scene);
            throw;
        }
        albedo_b200::unbindScene(description.scene);
        for (int y{0}; y < height; ++y) {
            for (int x{0}; x < width; ++x) {
                const albedo::Rgb a{image.average({.x = x, .y = y})};
                double* o{out_average + 3 * (static_cast<std::int64_t>(y) * width + x)};
                o[0] = a.r;
                o[1] = a.g;
                o[2] = a.b;
            }
        }
        // PixelBuffer shows no counts; the average of pixel (0, 0) with prior
        // samples tells whether the render added to them.
        *out_count = 0;
        *kind = 0;
        return 0;
    } catch (const std::invalid_argument& error) {
        message = error.what();
        *kind = 1;
    } catch (const std::runtime_error& error) {
        message = error.what();
        *kind = 2;
    } catch (const std::exception& error) {
        message = error.what();
        *kind = 3;
    }
    return 1;
}

} // extern "C"
