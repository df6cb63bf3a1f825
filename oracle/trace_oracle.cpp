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

// ---------------------------------------------------------------- near-tie classification
//
// A device answer that differs from the FP64 one is a near-tie only when FP32
// rounding can explain it. Rounding moves the primitives relative to the ray by
// at most delta = ulps * 2^-24 * M, where M is the largest coordinate magnitude
// among the ray origin, the crossing point and the primitive (its vertices, or
// its centre and radius), in the primitive's own space (object space inside an
// instance). So, for every primitive, its margin is measured in the plane
// perpendicular to the ray: the distance from the ray to the primitive's
// outline, positive when the ray passes through it, negative when it passes
// beside it. A primitive may be hit by a rounded ray if margin >= -delta and is
// surely hit if margin > delta (both with the crossing distance inside the query
// range by more than delta). A device hit on a primitive is explained if that
// primitive may be hit and lies no farther than the nearest sure hit plus both
// deltas; a device miss is explained if no primitive is surely hit.

struct Candidate {
    double t{kInf};      // distance parameter of the crossing (closest approach for a miss)
    double margin{-kInf};
    double delta{0};
    double scale{1};     // |d| in the primitive's space: t * scale is a distance there
};

double maxAbs(Vec3 v) { return std::max({std::abs(v.x), std::abs(v.y), std::abs(v.z)}); }

// The signed distance in 2D from the origin to triangle (a, b, c): positive
// inside (the ray passes through), minus the distance to the outline outside.
double signedDistance2(const double a[2], const double b[2], const double c[2])
{
    const double* p[3]{a, b, c};
    double area{(b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])};
    if (area == 0) {
        return -kInf;
    }
    const double orient{area > 0 ? 1.0 : -1.0};
    bool inside{true};
    double nearest_edge{kInf};
    double outside{kInf};
    for (int e{0}; e < 3; ++e) {
        const double* u{p[e]};
        const double* v{p[(e + 1) % 3]};
        const double ex{v[0] - u[0]};
        const double ey{v[1] - u[1]};
        const double length{std::sqrt(ex * ex + ey * ey)};
        // Signed distance of the origin from the edge's line, positive on the inner side.
        const double side{orient * (ex * (0 - u[1]) - ey * (0 - u[0])) / length};
        nearest_edge = std::min(nearest_edge, std::abs(side));
        if (side < 0) {
            inside = false;
        }
        // Distance from the origin to the segment.
        double s{-(u[0] * ex + u[1] * ey) / (length * length)};
        s = std::clamp(s, 0.0, 1.0);
        const double qx{u[0] + s * ex};
        const double qy{u[1] + s * ey};
        outside = std::min(outside, std::sqrt(qx * qx + qy * qy));
    }
    return inside ? nearest_edge : -outside;
}

// An orthonormal pair perpendicular to unit `w`.
void perpendicularPair(Vec3 w, Vec3& u, Vec3& v)
{
    const Vec3 helper{std::abs(w.x) < 0.6 ? Vec3{1, 0, 0} : Vec3{0, 1, 0}};
    u = normalized(cross(helper, w));
    v = cross(w, u);
}

Candidate triangleCandidate(const TriangleDesc& tri, const Ray& ray, double ulps)
{
    Candidate c;
    const double length{std::sqrt(lengthSquared(ray.d))};
    const Vec3 w{ray.d / length};
    Vec3 u;
    Vec3 v;
    perpendicularPair(w, u, v);
    double p2[3][2];
    for (int k{0}; k < 3; ++k) {
        const Vec3 off{tri.v[k] - ray.o};
        p2[k][0] = dot(off, u);
        p2[k][1] = dot(off, v);
    }
    c.margin = signedDistance2(p2[0], p2[1], p2[2]);
    const Vec3 n{cross(tri.v[1] - tri.v[0], tri.v[2] - tri.v[0])};
    const double denom{dot(n, ray.d)};
    c.t = denom != 0 ? dot(n, tri.v[0] - ray.o) / denom : kInf;
    double m{maxAbs(ray.o)};
    for (const Vec3& p : tri.v) {
        m = std::max(m, maxAbs(p));
    }
    if (std::isfinite(c.t)) {
        m = std::max(m, maxAbs(ray.o + ray.d * c.t));
    }
    c.delta = ulps * 0x1p-24 * m;
    c.scale = length;
    return c;
}

// Both roots of a sphere (the closest approach twice for a miss).
std::array<Candidate, 2> sphereCandidates(const SphereDesc& s, const Ray& ray, double ulps, bool wide)
{
    const double a{lengthSquared(ray.d)};
    const double length{std::sqrt(a)};
    const Vec3 oc{ray.o - s.center};
    const double closest{-dot(ray.d, oc) / a};
    const Vec3 l{oc + ray.d * closest};
    const double miss_distance{std::sqrt(lengthSquared(l))};
    Candidate c;
    c.margin = s.radius - miss_distance;
    c.scale = length;
    // FP64-handled spheres (the device's wide spheres) round only the ray.
    const double m{wide ? std::max(maxAbs(ray.o), maxAbs(ray.o + ray.d * closest))
                        : std::max({maxAbs(ray.o), maxAbs(s.center) + s.radius})};
    c.delta = ulps * 0x1p-24 * m;
    std::array<Candidate, 2> roots{c, c};
    if (c.margin >= 0) {
        const double half{std::sqrt(std::max(s.radius * s.radius - miss_distance * miss_distance, 0.0)) / length};
        roots[0].t = closest - half;
        roots[1].t = closest + half;
    } else {
        roots[0].t = closest;
        roots[1].t = closest;
    }
    return roots;
}

struct Reach {
    bool possible{false};
    bool sure{false};
};

Reach reachOf(const Candidate& c, double t_min, double t_max)
{
    const double along_min{(c.t - t_min) * c.scale};
    const double along_max{(t_max - c.t) * c.scale};
    Reach v;
    v.possible = c.margin >= -c.delta && along_min >= -c.delta && along_max >= -c.delta;
    v.sure = c.margin > c.delta && along_min > c.delta && along_max > c.delta;
    return v;
}

// Visits every primitive of the scene (no hierarchy: the classification must
// not depend on the traversal it checks) with its world-space candidates.
// visit(object, triangle (-1 for spheres and flattened triangles), candidate,
// world distance per unit t).
template <typename Visit>
void forEachCandidate(const HostScene& scene, const Ray& world, double ulps, Visit&& visit)
{
    const double world_length{std::sqrt(lengthSquared(world.d))};
    for (std::size_t id{0}; id < scene.objects.size(); ++id) {
        const ObjectDesc& obj{scene.objects[id]};
        switch (obj.kind) {
        case ObjectKind::Sphere: {
            const SphereDesc& s{scene.spheres[obj.index]};
            const double extent{maxAbs(s.center) + s.radius};
            for (const Candidate& c : sphereCandidates(s, world, ulps, extent >= 256.0)) {
                visit(static_cast<std::int64_t>(id), std::int64_t{-1}, c, world_length);
            }
            break;
        }
        case ObjectKind::Triangle:
            visit(static_cast<std::int64_t>(id), std::int64_t{-1},
                  triangleCandidate(scene.triangles[obj.index], world, ulps), world_length);
            break;
        default: {
            const InstanceDesc& inst{scene.instances[obj.index]};
            const MeshDesc& mesh{scene.meshes[inst.mesh]};
            const Ray local{inst.to_object.applyPoint(world.o), inst.to_object.applyVector(world.d)};
            for (std::size_t k{0}; k < mesh.triangles.size(); ++k) {
                visit(static_cast<std::int64_t>(id), static_cast<std::int64_t>(k),
                      triangleCandidate(mesh.triangles[k], local, ulps), world_length);
            }
            break;
        }
        }
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

// Scene::intersect (scene/scene.cpp:107-133): the nearest object and its hit.
std::int64_t nearestHit(const HostScene& scene, const Ray& ray, double t_min, double t_max, ShapeHit& nearest,
                        Counts& counts)
{
    std::int64_t nearest_object{-1};
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
    return nearest_object;
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
        ShapeHit nearest;
        const std::int64_t nearest_object{nearestHit(scene, ray, t_min, t_max, nearest, counts)};
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

// Classifies device closest-hit answers (hit flag, object id, triangle id within
// an instanced mesh or -1) against the FP64 restatement: out_class[i] = 0 when
// the device's answer is the FP64 one, 1 when it differs only by a near-tie
// that FP32 rounding of `ulps` units explains (see Candidate above), 2 when
// nothing explains it. For classes 1 and 2, out_detail (4 doubles per ray, may
// be NULL) holds the device primitive's margin / delta, the nearest sure hit's
// margin / delta, (t_device - t_sure) over the tie bound, and the number of
// primitives that may be hit nearer than the sure one.
void oracle_classify(const void* view, const double* rays, std::int64_t count, double t_min, double t_max,
                     double ulps, int threads, const std::int32_t* device_hit, const std::int64_t* device_object,
                     const std::int64_t* device_triangle, std::int32_t* out_class, double* out_detail)
{
    const HostScene& scene{*static_cast<const HostScene*>(view)};
    parallelFor(count, threads, [&](std::int64_t i) {
        const Ray ray{{rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]}, {rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]}};
        Counts counts;
        ShapeHit nearest;
        const std::int64_t object{nearestHit(scene, ray, t_min, t_max, nearest, counts)};
        const bool device_found{device_hit[i] != 0};
        if ((object < 0 && !device_found) ||
            (object >= 0 && device_found && device_object[i] == object && device_triangle[i] == nearest.triangle)) {
            out_class[i] = 0;
            return;
        }
        // The nearest sure hit, and the device's primitive among the candidates.
        double sure_t{kInf};
        Candidate sure;
        Candidate mine;
        bool mine_possible{false};
        std::int64_t possible_nearer{0};
        forEachCandidate(scene, ray, ulps, [&](std::int64_t id, std::int64_t tri, const Candidate& c, double) {
            const Reach v{reachOf(c, t_min, t_max)};
            if (v.sure && c.t < sure_t) {
                sure_t = c.t;
                sure = c;
            }
            if (device_found && id == device_object[i] && tri == device_triangle[i] && v.possible) {
                if (!mine_possible || std::abs(c.t) < std::abs(mine.t)) {
                    mine = c;
                }
                mine_possible = true;
            }
        });
        forEachCandidate(scene, ray, ulps, [&](std::int64_t, std::int64_t, const Candidate& c, double) {
            if (reachOf(c, t_min, t_max).possible && c.t < sure_t) {
                ++possible_nearer;
            }
        });
        bool explained{false};
        double tie{0};
        if (!device_found) {
            explained = !std::isfinite(sure_t);
        } else if (mine_possible) {
            const double bound{mine.delta / mine.scale + (std::isfinite(sure_t) ? sure.delta / sure.scale : 0)};
            tie = std::isfinite(sure_t) ? (mine.t - sure_t) / bound : -kInf;
            explained = !std::isfinite(sure_t) || mine.t - sure_t <= bound;
        }
        out_class[i] = explained ? 1 : 2;
        if (out_detail != nullptr) {
            out_detail[4 * i] = mine_possible ? mine.margin / mine.delta : -kInf;
            out_detail[4 * i + 1] = std::isfinite(sure_t) ? sure.margin / sure.delta : kInf;
            out_detail[4 * i + 2] = tie;
            out_detail[4 * i + 3] = static_cast<double>(possible_nearer);
        }
    });
}

} // extern "C"
