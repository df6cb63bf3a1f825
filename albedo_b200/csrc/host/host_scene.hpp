// The host-side scene: what the reference's Scene holds (scene/scene.hpp:94-97),
// flattened into tables that the device layout is built from.
//
// Objects keep the reference's add order, which is the `object` id a hit reports
// (scene/hit_record.hpp:29-32). Materials are shared by index instead of being
// copied into each object; lights keep the reference's light order, including
// where the sky sits (scene/scene.cpp:87-94), because next-event estimation picks
// a light by index.
#pragma once

#include "bvh_build.hpp"
#include "host_math.hpp"

#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace albedo_b200 {

struct Rgb {
    double r{};
    double g{};
    double b{};
};

enum class TextureKind : std::uint32_t { Constant = 0, Checker = 1, Perlin = 2 };
enum class BasicKind : std::uint32_t { Diffuse = 0, Conductor = 1, Dielectric = 2 };
enum class ObjectKind : std::uint32_t { Sphere = 0, Triangle = 1, Instance = 2 };
enum class LightKind : std::uint32_t { Point = 0, Area = 1, Sky = 2 };

// texture/texture.hpp:26-37: constant (a), checker (even a, odd b, frequency),
// Perlin (low a, high b, scale, veins).
struct TextureDesc {
    TextureKind kind{TextureKind::Constant};
    Rgb a{};
    Rgb b{};
    double frequency_or_scale{1};
    double veins{0};
};

// material/basic_material.hpp: diffuse (texture), conductor (eta, k, roughness),
// dielectric (ior, roughness).
struct BasicMaterialDesc {
    BasicKind kind{BasicKind::Diffuse};
    TextureDesc texture{};
    Rgb eta{1, 1, 1};
    Rgb k{};
    double ior{1.5};
    double roughness{0};
};

// material/material.hpp: a basic material, or a mix of two
// (material/mix_material.hpp:23-35).
struct MaterialDesc {
    bool mix{false};
    BasicMaterialDesc first{};
    BasicMaterialDesc second{};
    double scale{1};
    double veins{0};
    double threshold{0.5};
};

struct SphereDesc {
    Vec3 center{};
    double radius{};
};

// One triangle as geometry/triangle.hpp keeps it: vertices, unit front normal
// and texture coordinates per corner.
struct TriangleDesc {
    std::array<Vec3, 3> v{};
    Vec3 normal{};
    std::array<std::array<double, 2>, 3> uv{};
};

// A shared mesh (geometry/mesh_geometry.hpp:62-66): its triangles, optional
// smooth corner normals, bounds and BLAS.
struct MeshDesc {
    std::vector<TriangleDesc> triangles;
    std::vector<std::array<Vec3, 3>> corner_normals; // empty when flat
    Box3 bounds{};
    BuiltBvh bvh;
};

struct InstanceDesc {
    std::uint32_t mesh{};
    Transform to_world{};
    Transform to_object{};
    Box3 world_bounds{};
};

struct LightDesc {
    LightKind kind{LightKind::Point};
    Vec3 position{};     // point: position; area: sphere center
    double radius{};     // area
    Rgb emission{};      // point: intensity; area: radiance
    Rgb nadir{};         // sky
    Rgb zenith{};        // sky
    std::uint32_t object{}; // area: the object that is its surface
};

struct ObjectDesc {
    ObjectKind kind{ObjectKind::Sphere};
    std::uint32_t index{};    // into spheres, triangles or instances
    std::uint32_t material{}; // into materials
    std::int32_t light{-1};   // area light index, or -1
};

struct CameraSettings {
    Vec3 look_from{};
    Vec3 look_at{};
    Vec3 up{0, 1, 0};
    double vertical_fov_degrees{60};
};

// The camera frame of camera/perspective_camera.cpp:89-110 for a given aspect ratio.
struct CameraFrame {
    Vec3 origin{};
    Vec3 forward{};
    Vec3 half_width{};
    Vec3 half_height{};
};

class HostScene {
public:
    // Scene building, mirroring the reference Scene API (scene/scene.hpp:31-90).
    // Each throws std::invalid_argument with the reference's message for the
    // inputs the reference rejects.
    std::uint32_t addMaterial(const MaterialDesc& material);
    std::uint32_t addSphere(Vec3 center, double radius, std::uint32_t material);
    std::uint32_t addAreaLight(Vec3 center, double radius, Rgb radiance, std::uint32_t material);
    std::uint32_t addPointLight(Vec3 position, Rgb intensity);
    void setSky(Rgb nadir, Rgb zenith);
    // A mesh from positions and faces (geometry/triangle_mesh.hpp): faces
    // without a computable area are dropped. `texture_faces` is empty or one per face.
    std::uint32_t addMesh(const std::vector<Vec3>& positions,
                          const std::vector<std::array<std::uint32_t, 3>>& faces,
                          const std::vector<std::array<double, 2>>& texture_coordinates,
                          const std::vector<std::array<std::uint32_t, 3>>& texture_faces, bool smooth);
    std::uint32_t addInstance(std::uint32_t mesh, const Transform& to_world, std::uint32_t material);
    // Scene::add(const TriangleMesh&, ...): every triangle of the mesh as its own object.
    void addTriangles(const std::vector<Vec3>& positions, const std::vector<std::array<std::uint32_t, 3>>& faces,
                      const std::vector<std::array<double, 2>>& texture_coordinates,
                      const std::vector<std::array<std::uint32_t, 3>>& texture_faces, std::uint32_t material);

    // Builds the TLAS over every object's box, as the last Scene::add did.
    void finalize();

    CameraFrame cameraFrame(double aspect_ratio) const;
    // The world box of one object.
    Box3 objectBounds(const ObjectDesc& object) const;

    std::vector<MaterialDesc> materials;
    std::vector<SphereDesc> spheres;
    std::vector<TriangleDesc> triangles;
    std::vector<MeshDesc> meshes;
    std::vector<InstanceDesc> instances;
    std::vector<LightDesc> lights;
    std::vector<ObjectDesc> objects;
    std::int32_t sky_light{-1};
    BuiltBvh tlas;
    CameraSettings camera{};
    bool has_camera{false};
};

// A grid of 8 x 8 x 8 cells over the scene's compact core, for binning rays by
// where they start: {x0, y0, z0, cells per unit length}. The core is the box
// of the objects whose box diagonal is at most 16 times the median one (room
// walls and ground spheres of radius 1e4 are left out); cells per unit length
// is 0 when the core has no finite extent (every ray then falls in one cell).
std::array<float, 4> coherenceGrid(const HostScene& scene);

// True when the three points form a triangle with a computable area
// (geometry/triangle.cpp:197-205).
bool formsTriangle(Vec3 p0, Vec3 p1, Vec3 p2);
// Triangle built as geometry/triangle.cpp:116-121 builds one.
TriangleDesc makeTriangle(Vec3 p0, Vec3 p1, Vec3 p2, const std::array<std::array<double, 2>, 3>& uv);
Box3 triangleBounds(const TriangleDesc& triangle);
Box3 sphereBounds(const SphereDesc& sphere);
// Sphere validation of geometry/sphere.cpp:22-43; throws std::invalid_argument.
void validateSphere(Vec3 center, double radius);

// Validates camera settings as camera/perspective_camera.cpp:24-80 does and
// returns the frame; throws std::invalid_argument with the reference's message.
CameraFrame buildCameraFrame(const CameraSettings& settings, double aspect_ratio);

} // namespace albedo_b200
