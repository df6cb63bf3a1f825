// Double-precision host math for scene building: vectors, boxes and affine maps.
//
// Everything here runs once per scene on the host and must round exactly as the
// reference does, because the BVH topology, instance transforms and bounds it
// produces decide which primitives a ray tests. So each operation keeps the
// reference's evaluation order:
//   vectors, dot, cross, normalized    core/vector3.hpp:113-181
//   componentMin/Max, merged            core/point3.hpp:66-77, core/bounds3.hpp:62-73
//   surfaceArea                         core/bounds3.hpp:49-56
//   affine maps and their inverses      core/transform.cpp:23-225
// All host sources build with -ffp-contract=off (no FMA), as the reference's
// x86-64 build has none.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <limits>

namespace albedo_b200 {

struct Vec3 {
    double x{};
    double y{};
    double z{};
};

inline Vec3 operator+(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator-(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator-(Vec3 v) { return {-v.x, -v.y, -v.z}; }
inline Vec3 operator*(Vec3 v, double s) { return {v.x * s, v.y * s, v.z * s}; }
inline Vec3 operator/(Vec3 v, double s) { return {v.x / s, v.y / s, v.z / s}; }
inline bool operator==(Vec3 a, Vec3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline double dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Vec3 cross(Vec3 a, Vec3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double lengthSquared(Vec3 v) { return dot(v, v); }
inline Vec3 normalized(Vec3 v) { return v / std::sqrt(lengthSquared(v)); }
inline bool isFinite(Vec3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }
inline double axisOf(Vec3 v, std::size_t axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

inline Vec3 componentMin(Vec3 a, Vec3 b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
inline Vec3 componentMax(Vec3 a, Vec3 b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }

struct Box3 {
    Vec3 min{std::numeric_limits<double>::max(), std::numeric_limits<double>::max(),
             std::numeric_limits<double>::max()};
    Vec3 max{std::numeric_limits<double>::lowest(), std::numeric_limits<double>::lowest(),
             std::numeric_limits<double>::lowest()};

    bool isEmpty() const { return min.x > max.x || min.y > max.y || min.z > max.z; }
    Vec3 extent() const { return max - min; }
    double surfaceArea() const
    {
        if (isEmpty()) {
            return 0.0;
        }
        const Vec3 d{extent()};
        return 2 * (d.x * d.y + d.y * d.z + d.z * d.x);
    }
};

inline Box3 merged(const Box3& box, Vec3 p) { return {componentMin(box.min, p), componentMax(box.max, p)}; }
inline Box3 merged(const Box3& a, const Box3& b) { return {componentMin(a.min, b.min), componentMax(a.max, b.max)}; }

using Matrix3 = std::array<std::array<double, 3>, 3>;

// p -> linear p + offset; `linear` multiplies column vectors.
struct Affine {
    Matrix3 linear{{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};
    Vec3 offset{};
};

inline Vec3 multiplied(const Matrix3& m, Vec3 v)
{
    return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z, m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
            m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
}

inline Vec3 multipliedByTranspose(const Matrix3& m, Vec3 v)
{
    return {m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z, m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
            m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z};
}

// An affine map kept with its closed-form inverse (no numerical inversion).
class Transform {
public:
    Transform() = default;

    // Each factory throws std::invalid_argument on the inputs the reference rejects.
    static Transform translation(Vec3 offset);
    static Transform scaling(Vec3 factors);
    static Transform rotation(Vec3 axis, double degrees);

    // A transform from a map and its inverse given by the caller (the C ABI's
    // instances); the caller guarantees `backward` undoes `forward`.
    static Transform fromMaps(const Affine& forward, const Affine& backward) { return Transform{forward, backward}; }

    // The transform applying `first`, then `*this` (core/transform.cpp:183-191).
    Transform operator*(const Transform& first) const;
    Transform inverse() const { return Transform{inverse_map, forward_map}; }

    Vec3 applyPoint(Vec3 p) const { return Vec3{} + (multiplied(forward_map.linear, p - Vec3{}) + forward_map.offset); }
    Vec3 applyVector(Vec3 v) const { return multiplied(forward_map.linear, v); }
    Vec3 applyNormal(Vec3 n) const { return multipliedByTranspose(inverse_map.linear, n); }
    Box3 applyBox(const Box3& box) const;

    const Affine& forward() const { return forward_map; }
    const Affine& backward() const { return inverse_map; }

private:
    Transform(const Affine& forward, const Affine& backward) : forward_map{forward}, inverse_map{backward} {}

    Affine forward_map{};
    Affine inverse_map{};
};

} // namespace albedo_b200
