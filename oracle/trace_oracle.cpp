// Test infrastructure: an FP64 restatement of the reference's ray-query path,
// run over the host scene tables this repository builds (HostScene), with
// per-query work counts. It is the checker for
//   * the host build: hits must equal the reference's Scene::intersect bit for
//     bit (object id, t, point, normal), which holds only if the BVH topology,
//     transforms and triangles are the reference's;
//   * the device: triangle ids inside instanced meshes (which the reference's
//     API does not expose) and the node / primitive visit counts that the
//     roofline's algorithmic bytes are built from.
// Each function restates the reference function named beside it; the file is
// built with -ffp-contract=off like the reference's geometry and transform code.
//
// Entry points take the pointer albedo_scene_host_view() returns, so this
// library must be built against the same headers as libalbedo_b200.so.

#include "../albedo_b200/csrc/host/host_scene.hpp"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <limits>
#include <thread>
#include <vector>

using namespace albedo_b200;

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();
// 1 + 2 gamma(3) in FP64 (accel/bvh.hpp:80-84).
constexpr double kWiden = 1 + 2 * (3 * std::numeric_limits<double>::epsilon() / 2) /
                                  (1 - 3 * std::numeric_limits<double>::epsilon() / 2);

struct Ray {
    Vec3 o;
    Vec3 d;
};

struct Counts {
    std::int64_t boxes{0};
    std::int64_t triangles{0};
    std::int64_t spheres{0};
    std::int64_t instances{0};
};

struct ShapeHit {
    double t{};
    Vec3 point{};
    Vec3 normal{};
    Vec3 shading{};
    std::int64_t triangle{-1};
};

// clipToSlab / entersBox (accel/bvh.hpp:93-114).
bool entersBox(const Box3& box, const Ray& ray, const Vec3& inv, double lo, double hi)
{
    const double o[3]{ray.o.x, ray.o.y, ray.o.z};
    const double iv[3]{inv.x, inv.y, inv.z};
    const double mn[3]{box.min.x, box.min.y, box.min.z};
    const double mx[3]{box.max.x, box.max.y, box.max.z};
    for (int a{0}; a < 3; ++a) {
        double n{(mn[a] - o[a]) * iv[a]};
        double f{(mx[a] - o[a]) * iv[a]};
        if (n > f) {
            std::swap(n, f);
        }
        f *= f < 0 ? 2 - kWiden : kWiden;
        lo = n > lo ? n : lo;
        hi = f < hi ? f : hi;
    }
    return lo <= hi;
}

// Bvh::traverse (accel/bvh.hpp:239-278): visit(primitive) returns true to stop;
// `range_max` is re-read at every node so nearest-hit searches shrink it.
template <typename Visit>
void traverse(const BuiltBvh& bvh, const Ray& ray, double range_min, const double& range_max, Counts& counts,
              Visit&& visit)
{
    if (bvh.nodes.empty()) {
        return;
    }
    const Vec3 inv{1 / ray.d.x, 1 / ray.d.y, 1 / ray.d.z};
    const unsigned second_first{(ray.d.x < 0 ? 1U : 0U) | (ray.d.y < 0 ? 2U : 0U) | (ray.d.z < 0 ? 4U : 0U)};
    std::array<std::size_t, 128> stack{};
    std::size_t size{0};
    std::size_t current{0};
    for (;;) {
        const BuildNode& node{bvh.nodes[current]};
        ++counts.boxes;
        if (entersBox(node.bounds, ray, inv, range_min, range_max)) {
            if (node.count == 0) {
                const std::size_t first{current + 1};
                const std::size_t second{static_cast<std::size_t>(node.offset)};
                const bool swap{((second_first >> node.axis) & 1U) != 0};
                stack.at(size++) = swap ? first : second;
                current = swap ? second : first;
                continue;
            }
            bool stop{false};
            for (std::uint64_t e{node.offset}; e < node.offset + node.count; ++e) {
                if (visit(bvh.order[e])) {
                    stop = true;
                    break;
                }
            }
            if (stop) {
                return;
            }
        }
        if (size == 0) {
            return;
        }
        current = stack.at(--size);
    }
}

// Sphere::intersect (geometry/sphere.cpp:92-135).
bool sphereHit(const SphereDesc& s, const Ray& ray, double lo, double hi, ShapeHit& out)
{
    const Vec3 oc{ray.o - s.center};
    const double a{lengthSquared(ray.d)};
    if (!std::isnormal(a)) {
        return false;
    }
    const double h{dot(ray.d, oc)};
    const double c{lengthSquared(oc) - s.radius * s.radius};
    const Vec3 l{oc - ray.d * (h / a)};
    const double disc{a * (s.radius * s.radius - lengthSquared(l))};
    if (disc < 0) {
        return false;
    }
    const double q{-(h + std::copysign(std::sqrt(disc), h))};
    double n{0};
    double f{0};
    if (q != 0) {
        n = q / a;
        f = c / q;
        if (n > f) {
            std::swap(n, f);
        }
    }
    double t{n};
    if (!(lo < t && t < hi)) {
        t = f;
        if (!(lo < t && t < hi)) {
            return false;
        }
    }
    const Vec3 p{ray.o + ray.d * t};
    const Vec3 outward{p - s.center};
    if (!(lengthSquared(outward) > 0)) {
        return false;
    }
    out.t = t;
    out.point = p;
    out.normal = normalized(outward);
    out.shading = out.normal;
    return true;
}

double comp(Vec3 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

// Triangle::intersect (geometry/triangle.cpp:132-176), watertight, FP64.
bool triangleHit(const TriangleDesc& tri, const Ray& ray, double lo, double hi, ShapeHit& out, double* bary)
{
    if (!std::isnormal(lengthSquared(ray.d))) {
        return false;
    }
    const Vec3 m{std::abs(ray.d.x), std::abs(ray.d.y), std::abs(ray.d.z)};
    const int kz{m.x > m.y ? (m.x > m.z ? 0 : 2) : (m.y > m.z ? 1 : 2)};
    const double dz{comp(ray.d, kz)};
    int kx{(kz + 1) % 3};
    int ky{(kx + 1) % 3};
    if (dz < 0) {
        std::swap(kx, ky);
    }
    const double sx{comp(ray.d, kx) / dz};
    const double sy{comp(ray.d, ky) / dz};
    const double sz{1 / dz};
    const auto transformed = [&](Vec3 off) {
        const double z{comp(off, kz)};
        return Vec3{comp(off, kx) - sx * z, comp(off, ky) - sy * z, sz * z};
    };
    const Vec3 a{transformed(tri.v[0] - ray.o)};
    const Vec3 b{transformed(tri.v[1] - ray.o)};
    const Vec3 c{transformed(tri.v[2] - ray.o)};
    const auto edge = [](Vec3 p, Vec3 q) { return q.x * p.y - q.y * p.x; };
    const double u{edge(b, c)};
    const double v{edge(c, a)};
    const double w{edge(a, b)};
    if (!((u >= 0 && v >= 0 && w >= 0) || (u <= 0 && v <= 0 && w <= 0))) {
        return false;
    }
    const double det{u + v + w};
    if (det == 0) {
        return false;
    }
    const double t{(u * a.z + v * b.z + w * c.z) / det};
    if (!(lo < t && t < hi)) {
        return false;
    }
    const double b0{u / det};
    const double b1{v / det};
    const double b2{w / det};
    out.t = t;
    out.point = tri.v[0] + (tri.v[1] - tri.v[0]) * b1 + (tri.v[2] - tri.v[0]) * b2;
    out.normal = tri.normal;
    out.shading = tri.normal;
    if (bary != nullptr) {
        bary[0] = b0;
        bary[1] = b1;
        bary[2] = b2;
    }
    return true;
}

// blendedNormal (geometry/mesh_geometry.cpp:53-64) with barycentricCoordinatesOf
// (geometry/triangle.cpp:182-195).
Vec3 blendedNormal(const TriangleDesc& tri, const std::array<Vec3, 3>& n, Vec3 p)
{
    const Vec3 e1{tri.v[1] - tri.v[0]};
    const Vec3 e2{tri.v[2] - tri.v[0]};
    const Vec3 off{p - tri.v[0]};
    const Vec3 an{cross(e1, e2)};
    const double area2{lengthSquared(an)};
    const double b1{dot(cross(off, e2), an) / area2};
    const double b2{dot(cross(e1, off), an) / area2};
    const double b0{1 - b1 - b2};
    const Vec3 blended{n[0] * b0 + n[1] * b1 + n[2] * b2};
    if (!(lengthSquared(blended) >= 1e-12)) {
        return tri.normal;
    }
    return normalized(blended);
}

// MeshGeometry::intersect + MeshInstance::intersect (geometry/mesh_geometry.cpp:77-98,
// geometry/mesh_instance.cpp:32-60).
bool instanceHit(const HostScene& scene, const InstanceDesc& inst, const Ray& world, double lo, double hi,
                 ShapeHit& out, Counts& counts)
{
    const MeshDesc& mesh{scene.meshes[inst.mesh]};
    const Ray ray{inst.to_object.applyPoint(world.o), inst.to_object.applyVector(world.d)};
    std::int64_t nearest{-1};
    ShapeHit best;
    double range_max{hi};
    traverse(mesh.bvh, ray, lo, range_max, counts, [&](std::uint32_t index) {
        ++counts.triangles;
        ShapeHit h;
        if (triangleHit(mesh.triangles[index], ray, lo, range_max, h, nullptr)) {
            best = h;
            nearest = index;
            range_max = h.t;
        }
        return false;
    });
    if (nearest < 0) {
        return false;
    }
    if (!mesh.corner_normals.empty()) {
        best.shading = blendedNormal(mesh.triangles[nearest], mesh.corner_normals[nearest], best.point);
    }
    const Vec3 wn{inst.to_world.applyNormal(best.normal)};
    if (!std::isnormal(lengthSquared(wn))) {
        return false;
    }
    out.t = best.t;
    out.point = inst.to_world.applyPoint(best.point);
    out.normal = normalized(wn);
    if (best.shading == best.normal) {
        out.shading = out.normal;
    } else {
        const Vec3 ws{inst.to_world.applyNormal(best.shading)};
        out.shading = std::isnormal(lengthSquared(ws)) ? normalized(ws) : out.normal;
    }
    out.triangle = nearest;
    return true;
}

bool objectHit(const HostScene& scene, std::uint32_t id, const Ray& ray, double lo, double hi, ShapeHit& out,
               Counts& counts)
{
    const ObjectDesc& obj{scene.objects[id]};
    switch (obj.kind) {
    case ObjectKind::Sphere:
        ++counts.spheres;
        return sphereHit(scene.spheres[obj.index], ray, lo, hi, out);
    case ObjectKind::Triangle:
        ++counts.triangles;
        return triangleHit(scene.triangles[obj.index], ray, lo, hi, out, nullptr);
    default:
        ++counts.instances;
        return instanceHit(scene, scene.instances[obj.index], ray, lo, hi, out, counts);
    }
}

template <typename F>
void parallelFor(std::int64_t count, int threads, F&& work)
{
    std::atomic<std::int64_t> next{0};
    auto drain = [&] {
        for (;;) {
            const std::int64_t chunk{next.fetch_add(64)};
            if (chunk >= count) {
                return;
            }
            for (std::int64_t i{chunk}; i < std::min(count, chunk + 64); ++i) {
                work(i);
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t{1}; t < threads; ++t) {
        pool.emplace_back(drain);
    }
    drain();
    for (auto& th : pool) {
        th.join();
    }
}

} // namespace

extern "C" {

// Scene::intersect (scene/scene.cpp:107-133) per ray, plus the triangle id within
// an instanced mesh and the work each query did (boxes as the reference tests
// them: one per node visited).
void oracle_intersect(const void* view, const double* rays, std::int64_t count, double t_min, double t_max,
                      int threads, std::int32_t* out_hit, double* out_t, std::int64_t* out_object,
                      std::int64_t* out_triangle, double* out_point, double* out_normal, double* out_shading,
                      std::int32_t* out_front, std::int64_t* out_counts)
{
    const HostScene& scene{*static_cast<const HostScene*>(view)};
    parallelFor(count, threads, [&](std::int64_t i) {
        const Ray ray{{rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]}, {rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]}};
        Counts counts;
        std::int64_t nearest_object{-1};
        ShapeHit nearest;
        double range_max{t_max};
        traverse(scene.tlas, ray, t_min, range_max, counts, [&](std::uint32_t id) {
            ShapeHit h;
            if (objectHit(scene, id, ray, t_min, range_max, h, counts)) {
                nearest = h;
                nearest_object = id;
                range_max = h.t;
            }
            return false;
        });
        out_hit[i] = nearest_object >= 0 ? 1 : 0;
        if (out_counts != nullptr) {
            out_counts[4 * i] = counts.boxes;
            out_counts[4 * i + 1] = counts.triangles;
            out_counts[4 * i + 2] = counts.spheres;
            out_counts[4 * i + 3] = counts.instances;
        }
        if (nearest_object < 0) {
            return;
        }
        const bool front{dot(ray.d, nearest.normal) < 0};
        const Vec3 n{front ? nearest.normal : -nearest.normal};
        const Vec3 s{front ? nearest.shading : -nearest.shading};
        out_t[i] = nearest.t;
        out_object[i] = nearest_object;
        out_triangle[i] = nearest.triangle;
        out_front[i] = front ? 1 : 0;
        for (int k{0}; k < 3; ++k) {
            out_point[3 * i + k] = comp(nearest.point, k);
            out_normal[3 * i + k] = comp(n, k);
            out_shading[3 * i + k] = comp(s, k);
        }
    });
}

} // extern "C"
