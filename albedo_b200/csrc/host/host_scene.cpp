// Scene building on the host: restates the reference's constructors and
// Scene::add* (scene/scene.cpp:23-105) over flat tables, and the camera frame
// (camera/perspective_camera.cpp:24-110).
#include "host_scene.hpp"

#include <algorithm>
#include <cmath>
#include <format>
#include <numbers>
#include <stdexcept>
#include <thread>
#include <vector>

namespace albedo_b200 {

namespace {

constexpr double kPi{std::numbers::pi_v<double>};

// Default texture coordinates of a triangle (geometry/triangle.hpp:17-18).
constexpr std::array<std::array<double, 2>, 3> kDefaultUv{{{0.0, 0.0}, {1.0, 0.0}, {1.0, 1.0}}};

} // namespace

void validateSphere(Vec3 center, double radius)
{
    if (!isFinite(center)) {
        throw std::invalid_argument{
            std::format("sphere center ({}, {}, {}) must be finite", center.x, center.y, center.z)};
    }
    if (!(radius > 0) || !std::isfinite(radius) || !std::isnormal(radius * radius)) {
        throw std::invalid_argument{
            std::format("sphere radius must be positive and its square a normal number, got {}", radius)};
    }
}

bool formsTriangle(Vec3 p0, Vec3 p1, Vec3 p2)
{
    if (!isFinite(p0) || !isFinite(p1) || !isFinite(p2)) {
        return false;
    }
    return std::isnormal(lengthSquared(cross(p1 - p0, p2 - p0)));
}

TriangleDesc makeTriangle(Vec3 p0, Vec3 p1, Vec3 p2, const std::array<std::array<double, 2>, 3>& uv)
{
    if (!isFinite(p0) || !isFinite(p1) || !isFinite(p2)) {
        throw std::invalid_argument{"triangle vertices must have finite coordinates"};
    }
    if (!formsTriangle(p0, p1, p2)) {
        throw std::invalid_argument{std::format("triangle ({}, {}, {}), ({}, {}, {}), ({}, {}, {}) has no computable area",
                                                p0.x, p0.y, p0.z, p1.x, p1.y, p1.z, p2.x, p2.y, p2.z)};
    }
    for (const auto& corner : uv) {
        if (!std::isfinite(corner[0]) || !std::isfinite(corner[1])) {
            throw std::invalid_argument{
                std::format("triangle texture coordinates ({}, {}) must be finite", corner[0], corner[1])};
        }
    }
    TriangleDesc triangle;
    triangle.v = {p0, p1, p2};
    triangle.normal = normalized(cross(p1 - p0, p2 - p0));
    triangle.uv = uv;
    return triangle;
}

Box3 triangleBounds(const TriangleDesc& triangle)
{
    return merged(merged(merged(Box3{}, triangle.v[0]), triangle.v[1]), triangle.v[2]);
}

Box3 sphereBounds(const SphereDesc& sphere)
{
    const Vec3 half{sphere.radius, sphere.radius, sphere.radius};
    return {sphere.center - half, sphere.center + half};
}

std::uint32_t HostScene::addMaterial(const MaterialDesc& material)
{
    materials.push_back(material);
    return static_cast<std::uint32_t>(materials.size() - 1);
}

std::uint32_t HostScene::addSphere(Vec3 center, double radius, std::uint32_t material)
{
    validateSphere(center, radius);
    spheres.push_back({center, radius});
    objects.push_back({ObjectKind::Sphere, static_cast<std::uint32_t>(spheres.size() - 1), material, -1});
    return static_cast<std::uint32_t>(objects.size() - 1);
}

std::uint32_t HostScene::addAreaLight(Vec3 center, double radius, Rgb radiance, std::uint32_t material)
{
    validateSphere(center, radius);
    spheres.push_back({center, radius});
    const auto object{static_cast<std::uint32_t>(objects.size())};
    lights.push_back({.kind = LightKind::Area, .position = center, .radius = radius, .emission = radiance,
                      .object = object});
    objects.push_back({ObjectKind::Sphere, static_cast<std::uint32_t>(spheres.size() - 1), material,
                       static_cast<std::int32_t>(lights.size() - 1)});
    return object;
}

std::uint32_t HostScene::addPointLight(Vec3 position, Rgb intensity)
{
    lights.push_back({.kind = LightKind::Point, .position = position, .emission = intensity});
    return static_cast<std::uint32_t>(lights.size() - 1);
}

void HostScene::setSky(Rgb nadir, Rgb zenith)
{
    const LightDesc sky{.kind = LightKind::Sky, .nadir = nadir, .zenith = zenith};
    if (sky_light >= 0) {
        lights[static_cast<std::size_t>(sky_light)] = sky;
    } else {
        lights.push_back(sky);
        sky_light = static_cast<std::int32_t>(lights.size() - 1);
    }
}

namespace {

// Meshes of at least this many faces are processed on several threads.
constexpr std::size_t kParallelFaces{8192};

std::size_t chunkCount(std::size_t faces)
{
    if (faces < kParallelFaces) {
        return 1;
    }
    return std::max<std::size_t>(1, std::min<std::size_t>(std::thread::hardware_concurrency(), faces / 4096));
}

// Runs body(chunk, begin, end) over `chunks` contiguous ranges of [0, n), each
// on its own thread (the first on the calling one).
template <typename F>
void forEachChunk(std::size_t n, std::size_t chunks, F&& body)
{
    const auto range = [&](std::size_t chunk) { return n * chunk / chunks; };
    // A jthread joins when destroyed, so an exception that leaves early (a
    // thread that fails to start, or the calling thread's own share) still
    // waits for the workers already running.
    std::vector<std::jthread> workers;
    for (std::size_t chunk{1}; chunk < chunks; ++chunk) {
        workers.emplace_back([&, chunk] { body(chunk, range(chunk), range(chunk + 1)); });
    }
    body(0, range(0), range(1));
    for (std::jthread& worker : workers) {
        worker.join();
    }
}

// Area-weighted vertex normals (geometry/triangle_mesh.cpp:92-107): the
// unnormalized edge cross product of every face that forms a triangle, summed
// per position in face order. Each thread owns a range of positions and scans
// all faces in order, adding only to the positions it owns, so every sum adds
// the same terms in the same order as one thread would.
std::vector<Vec3> smoothNormalSums(const std::vector<Vec3>& positions,
                                   const std::vector<std::array<std::uint32_t, 3>>& faces,
                                   const std::vector<std::uint8_t>& forms, std::size_t chunks)
{
    std::vector<Vec3> sums(positions.size());
    forEachChunk(positions.size(), chunks, [&](std::size_t, std::size_t begin, std::size_t end) {
        const auto owned = [&](std::uint32_t index) { return index >= begin && index < end; };
        for (std::size_t face{0}; face < faces.size(); ++face) {
            const auto& f{faces[face]};
            if (!forms[face] || !(owned(f[0]) || owned(f[1]) || owned(f[2]))) {
                continue;
            }
            const Vec3 p0{positions[f[0]]};
            const Vec3 p1{positions[f[1]]};
            const Vec3 p2{positions[f[2]]};
            const Vec3 area_normal{cross(p1 - p0, p2 - p0)};
            for (const std::uint32_t index : f) {
                if (owned(index)) {
                    sums[index] = sums[index] + area_normal;
                }
            }
        }
    });
    return sums;
}

// TriangleMesh validation (geometry/triangle_mesh.cpp:57-74) and its triangles()
// and smoothNormals() (geometry/triangle_mesh.cpp:76-125).
struct MeshTriangles {
    std::vector<TriangleDesc> triangles;
    std::vector<std::array<Vec3, 3>> corner_normals;
};

MeshTriangles meshTriangles(const std::vector<Vec3>& positions, const std::vector<std::array<std::uint32_t, 3>>& faces,
                            const std::vector<std::array<double, 2>>& uvs,
                            const std::vector<std::array<std::uint32_t, 3>>& texture_faces, bool smooth)
{
    for (std::size_t i{0}; i < positions.size(); ++i) {
        if (!isFinite(positions[i])) {
            throw std::invalid_argument{std::format("mesh position {} has a non-finite coordinate", i)};
        }
    }
    for (std::size_t face{0}; face < faces.size(); ++face) {
        for (const std::uint32_t index : faces[face]) {
            if (index >= positions.size()) {
                throw std::out_of_range{std::format("mesh face {} uses position {}, but the mesh has {} positions",
                                                    face, index, positions.size())};
            }
        }
    }
    for (std::size_t i{0}; i < uvs.size(); ++i) {
        if (!std::isfinite(uvs[i][0]) || !std::isfinite(uvs[i][1])) {
            throw std::invalid_argument{std::format("mesh texture coordinate {} is not finite", i)};
        }
    }
    if (!texture_faces.empty() && texture_faces.size() != faces.size()) {
        throw std::invalid_argument{
            std::format("mesh has {} texture faces for {} faces", texture_faces.size(), faces.size())};
    }
    for (std::size_t face{0}; face < texture_faces.size(); ++face) {
        for (const std::uint32_t index : texture_faces[face]) {
            if (index >= uvs.size()) {
                throw std::out_of_range{std::format(
                    "mesh face {} uses texture coordinate {}, but the mesh has {} texture coordinates", face, index,
                    uvs.size())};
            }
        }
    }
    // Faces are independent except for the vertex-normal sums, so large meshes
    // are processed in chunks on several threads; the results are the
    // one-thread results (see smoothNormalSums for the sums).
    const std::size_t chunks{chunkCount(faces.size())};
    std::vector<std::uint8_t> forms(faces.size());
    std::vector<std::size_t> kept_before(chunks + 1, 0);
    forEachChunk(faces.size(), chunks, [&](std::size_t chunk, std::size_t begin, std::size_t end) {
        std::size_t kept{0};
        for (std::size_t face{begin}; face < end; ++face) {
            forms[face] = formsTriangle(positions[faces[face][0]], positions[faces[face][1]],
                                        positions[faces[face][2]]);
            kept += forms[face];
        }
        kept_before[chunk + 1] = kept;
    });
    for (std::size_t chunk{0}; chunk < chunks; ++chunk) {
        kept_before[chunk + 1] += kept_before[chunk];
    }
    MeshTriangles result;
    result.triangles.resize(kept_before[chunks]);
    forEachChunk(faces.size(), chunks, [&](std::size_t chunk, std::size_t begin, std::size_t end) {
        std::size_t out{kept_before[chunk]};
        for (std::size_t face{begin}; face < end; ++face) {
            if (!forms[face]) {
                continue;
            }
            std::array<std::array<double, 2>, 3> uv{kDefaultUv};
            if (!texture_faces.empty()) {
                uv = {uvs[texture_faces[face][0]], uvs[texture_faces[face][1]], uvs[texture_faces[face][2]]};
            }
            result.triangles[out++] =
                makeTriangle(positions[faces[face][0]], positions[faces[face][1]], positions[faces[face][2]], uv);
        }
    });
    if (!smooth) {
        return result;
    }
    const std::vector<Vec3> sums{smoothNormalSums(positions, faces, forms, chunks)};
    result.corner_normals.resize(result.triangles.size());
    forEachChunk(faces.size(), chunks, [&](std::size_t chunk, std::size_t begin, std::size_t end) {
        std::size_t out{kept_before[chunk]};
        for (std::size_t face{begin}; face < end; ++face) {
            if (!forms[face]) {
                continue;
            }
            const auto& f{faces[face]};
            const Vec3 p0{positions[f[0]]};
            const Vec3 p1{positions[f[1]]};
            const Vec3 p2{positions[f[2]]};
            const Vec3 face_normal{normalized(cross(p1 - p0, p2 - p0))};
            const auto corner = [&](std::uint32_t index) {
                const Vec3 sum{sums[index]};
                return std::isnormal(lengthSquared(sum)) ? normalized(sum) : face_normal;
            };
            result.corner_normals[out++] = {corner(f[0]), corner(f[1]), corner(f[2])};
        }
    });
    return result;
}

} // namespace

std::uint32_t HostScene::addMesh(const std::vector<Vec3>& positions,
                                 const std::vector<std::array<std::uint32_t, 3>>& faces,
                                 const std::vector<std::array<double, 2>>& texture_coordinates,
                                 const std::vector<std::array<std::uint32_t, 3>>& texture_faces, bool smooth)
{
    MeshTriangles built{meshTriangles(positions, faces, texture_coordinates, texture_faces, smooth)};
    if (built.triangles.empty()) {
        throw std::invalid_argument{"mesh geometry needs at least one triangle with area"};
    }
    MeshDesc mesh;
    mesh.triangles = std::move(built.triangles);
    mesh.corner_normals = std::move(built.corner_normals);
    std::vector<Box3> boxes;
    boxes.reserve(mesh.triangles.size());
    for (const TriangleDesc& triangle : mesh.triangles) {
        boxes.push_back(triangleBounds(triangle));
        mesh.bounds = merged(mesh.bounds, boxes.back());
    }
    mesh.bvh = buildBvh(boxes);
    meshes.push_back(std::move(mesh));
    return static_cast<std::uint32_t>(meshes.size() - 1);
}

std::uint32_t HostScene::addInstance(std::uint32_t mesh, const Transform& to_world, std::uint32_t material)
{
    if (mesh >= meshes.size()) {
        throw std::invalid_argument{"mesh instance needs a mesh"};
    }
    const Box3 world_bounds{to_world.applyBox(meshes[mesh].bounds)};
    if (!isFinite(world_bounds.min) || !isFinite(world_bounds.max)) {
        throw std::invalid_argument{"mesh instance transform takes the mesh out of range"};
    }
    instances.push_back({mesh, to_world, to_world.inverse(), world_bounds});
    objects.push_back({ObjectKind::Instance, static_cast<std::uint32_t>(instances.size() - 1), material, -1});
    return static_cast<std::uint32_t>(objects.size() - 1);
}

void HostScene::addTriangles(const std::vector<Vec3>& positions,
                             const std::vector<std::array<std::uint32_t, 3>>& faces,
                             const std::vector<std::array<double, 2>>& texture_coordinates,
                             const std::vector<std::array<std::uint32_t, 3>>& texture_faces, std::uint32_t material)
{
    MeshTriangles built{meshTriangles(positions, faces, texture_coordinates, texture_faces, false)};
    for (TriangleDesc& triangle : built.triangles) {
        triangles.push_back(triangle);
        objects.push_back({ObjectKind::Triangle, static_cast<std::uint32_t>(triangles.size() - 1), material, -1});
    }
}

Box3 HostScene::objectBounds(const ObjectDesc& object) const
{
    switch (object.kind) {
    case ObjectKind::Sphere:
        return sphereBounds(spheres[object.index]);
    case ObjectKind::Triangle:
        return triangleBounds(triangles[object.index]);
    default:
        return instances[object.index].world_bounds;
    }
}

void HostScene::finalize()
{
    std::vector<Box3> boxes;
    boxes.reserve(objects.size());
    for (const ObjectDesc& object : objects) {
        boxes.push_back(objectBounds(object));
    }
    tlas = buildBvh(boxes);
}

CameraFrame HostScene::cameraFrame(double aspect_ratio) const { return buildCameraFrame(camera, aspect_ratio); }

CameraFrame buildCameraFrame(const CameraSettings& settings, double aspect_ratio)
{
    const double fov{settings.vertical_fov_degrees};
    if (std::isnan(fov) || fov <= 0 || fov >= 180) {
        throw std::invalid_argument{std::format("vertical field of view must be in (0, 180) degrees, got {}", fov)};
    }
    if (!(aspect_ratio > 0) || !std::isnormal(aspect_ratio)) {
        throw std::invalid_argument{std::format("aspect ratio must be a positive normal number, got {}", aspect_ratio)};
    }
    if (!isFinite(settings.look_from) || !isFinite(settings.look_at)) {
        throw std::invalid_argument{"camera position and target must be finite"};
    }
    const Vec3 backward{settings.look_from - settings.look_at};
    if (!std::isnormal(lengthSquared(backward))) {
        throw std::invalid_argument{"distance from camera position to target must be "
                                    "non-zero, finite and within roughly [1e-154, 1e154]"};
    }
    if (!std::isnormal(lengthSquared(settings.up))) {
        throw std::invalid_argument{"length of the camera up direction must be non-zero, "
                                    "finite and within roughly [1e-154, 1e154]"};
    }
    const Vec3 w{normalized(backward)};
    const Vec3 right{cross(normalized(settings.up), w)};
    if (lengthSquared(right) < 1e-12) {
        throw std::invalid_argument{"camera up direction must not be parallel to the view"};
    }
    const Vec3 u{normalized(right)};
    const Vec3 v{cross(w, u)};
    const double half_fov{settings.vertical_fov_degrees * kPi / 360};
    const double half_height{std::tan(half_fov)};
    const double half_width{aspect_ratio * half_height};
    const CameraFrame frame{settings.look_from, -w, u * half_width, v * half_height};
    if (!std::isnormal(lengthSquared(frame.forward + frame.half_width + frame.half_height))) {
        throw std::invalid_argument{"field of view and aspect ratio make the film too large"};
    }
    return frame;
}

} // namespace albedo_b200

namespace albedo_b200 {

std::array<float, 4> coherenceGrid(const HostScene& scene)
{
    std::vector<Box3> boxes;
    std::vector<double> diagonals;
    for (const ObjectDesc& object : scene.objects) {
        const Box3 box{scene.objectBounds(object)};
        const double diagonal{std::sqrt(lengthSquared(box.extent()))};
        if (!box.isEmpty() && std::isfinite(diagonal)) {
            boxes.push_back(box);
            diagonals.push_back(diagonal);
        }
    }
    if (boxes.empty()) {
        return {0.0f, 0.0f, 0.0f, 0.0f};
    }
    std::vector<double> sorted{diagonals};
    std::nth_element(sorted.begin(), sorted.begin() + static_cast<std::ptrdiff_t>(sorted.size() / 2), sorted.end());
    const double limit{16 * sorted[sorted.size() / 2]};
    Box3 core;
    for (std::size_t i{0}; i < boxes.size(); ++i) {
        if (diagonals[i] <= limit) {
            core = merged(core, boxes[i]);
        }
    }
    const Vec3 extent{core.extent()};
    const double largest{std::max({extent.x, extent.y, extent.z})};
    if (core.isEmpty() || !(largest > 0) || !std::isfinite(largest)) {
        return {0.0f, 0.0f, 0.0f, 0.0f};
    }
    return {static_cast<float>(core.min.x), static_cast<float>(core.min.y), static_cast<float>(core.min.z),
            static_cast<float>(8.0 / largest)};
}

} // namespace albedo_b200
