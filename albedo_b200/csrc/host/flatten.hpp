// HostScene -> device tables (host copies), ready for one upload.
#pragma once

#include "../device_layout.hpp"
#include "host_scene.hpp"

#include <stdexcept>
#include <string>
#include <vector>

namespace albedo_b200 {

// A scene the device tables cannot hold as given (FP32 range), though the
// reference, which works in FP64, accepts it.
class LayoutLimitError : public std::runtime_error {
public:
    explicit LayoutLimitError(const std::string& what) : std::runtime_error{what} {}
};

struct DeviceImage {
    std::vector<DevNode> nodes;
    std::vector<DevObject> objects;
    std::vector<DevSphere> spheres;
    std::vector<DevTriangle> triangles;
    std::vector<DevTriangleAttr> attrs;
    std::vector<DevInstance> instances;
    std::vector<DevMaterial> materials;
    std::vector<DevLight> lights;
    std::vector<std::int32_t> object_light;
    std::vector<double> instance_to_object64;
    // Leaf position of each object id, and the triangle-table base of each mesh.
    std::vector<std::uint32_t> object_position;
    std::vector<std::uint32_t> mesh_triangle_base;
    std::uint32_t tlas_root{kEmptyChild};
    std::int32_t sky_light{-1};
    // Traversal stack entries a query can need: TLAS depth + deepest BLAS + 2.
    std::uint32_t stack_need{0};
};

// Throws std::invalid_argument if the scene exceeds the device layout's limits
// (leaf positions must fit 28 bits), and LayoutLimitError if a coordinate of
// its geometry, instance maps or lights is beyond FP32's range.
DeviceImage flattenScene(const HostScene& scene);

// The camera frame for an image of the given size, rounded to FP32 (throws
// LayoutLimitError if it leaves FP32's range).
DevCamera deviceCamera(const HostScene& scene, int width, int height);
DevCamera deviceCamera(const CameraSettings& settings, int width, int height);

} // namespace albedo_b200
