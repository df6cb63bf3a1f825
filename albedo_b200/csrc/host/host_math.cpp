// Affine transforms with closed-form inverses: restates core/transform.cpp:23-225
// operation for operation, so instance placements (and the world boxes the TLAS
// is built over) round exactly as in the reference.
#include "host_math.hpp"

#include <format>
#include <numbers>
#include <stdexcept>

namespace albedo_b200 {

namespace {

// `outer` applied after `inner` (core/transform.cpp:62-77).
Affine composed(const Affine& outer, const Affine& inner)
{
    Affine result{};
    for (std::size_t row{0}; row < 3; ++row) {
        for (std::size_t column{0}; column < 3; ++column) {
            double sum{0};
            for (std::size_t k{0}; k < 3; ++k) {
                sum += outer.linear[row][k] * inner.linear[k][column];
            }
            result.linear[row][column] = sum;
        }
    }
    result.offset = multiplied(outer.linear, inner.offset) + outer.offset;
    return result;
}

bool isFiniteMap(const Affine& map)
{
    for (const auto& row : map.linear) {
        for (const double value : row) {
            if (!std::isfinite(value)) {
                return false;
            }
        }
    }
    return isFinite(map.offset);
}

void checkFinite(double value, const char* what)
{
    if (!std::isfinite(value)) {
        throw std::invalid_argument{std::format("transform {} {} is not finite", what, value)};
    }
}

// Rodrigues' rotation matrix about a unit axis (core/transform.cpp:98-107).
Matrix3 rotationMatrix(Vec3 axis, double radians)
{
    const double c{std::cos(radians)};
    const double s{std::sin(radians)};
    const double t{1 - c};
    const double x{axis.x};
    const double y{axis.y};
    const double z{axis.z};
    return {{{t * x * x + c, t * x * y - s * z, t * x * z + s * y},
             {t * x * y + s * z, t * y * y + c, t * y * z - s * x},
             {t * x * z - s * y, t * y * z + s * x, t * z * z + c}}};
}

Matrix3 transposed(const Matrix3& m)
{
    Matrix3 result{};
    for (std::size_t row{0}; row < 3; ++row) {
        for (std::size_t column{0}; column < 3; ++column) {
            result[row][column] = m[column][row];
        }
    }
    return result;
}

struct AxisRange {
    double min{};
    double max{};
};

// Arvo's transformed box along one output axis, summed in the order that
// applyPoint sums a transformed corner (core/transform.cpp:124-137).
AxisRange transformedRange(const std::array<double, 3>& row, double offset, const Box3& box)
{
    const std::array<double, 3> low{box.min.x, box.min.y, box.min.z};
    const std::array<double, 3> high{box.max.x, box.max.y, box.max.z};
    AxisRange range{};
    for (std::size_t axis{0}; axis < 3; ++axis) {
        const double a{row[axis] * low[axis]};
        const double b{row[axis] * high[axis]};
        range.min = axis == 0 ? std::min(a, b) : range.min + std::min(a, b);
        range.max = axis == 0 ? std::max(a, b) : range.max + std::max(a, b);
    }
    range.min += offset;
    range.max += offset;
    return range;
}

} // namespace

Transform Transform::translation(Vec3 offset)
{
    checkFinite(offset.x, "translation component");
    checkFinite(offset.y, "translation component");
    checkFinite(offset.z, "translation component");
    Affine forward{};
    Affine backward{};
    forward.offset = offset;
    backward.offset = -offset;
    return Transform{forward, backward};
}

Transform Transform::scaling(Vec3 factors)
{
    Affine forward{};
    Affine backward{};
    const std::array<double, 3> scale{factors.x, factors.y, factors.z};
    for (std::size_t axis{0}; axis < 3; ++axis) {
        const double factor{scale[axis]};
        if (!std::isfinite(factor) || factor == 0 || !std::isfinite(1 / factor)) {
            throw std::invalid_argument{std::format(
                "transform scale factor {} must be finite and non-zero with a finite reciprocal", factor)};
        }
        forward.linear[axis][axis] = factor;
        backward.linear[axis][axis] = 1 / factor;
    }
    return Transform{forward, backward};
}

Transform Transform::rotation(Vec3 axis, double degrees)
{
    checkFinite(degrees, "rotation angle");
    if (!std::isnormal(lengthSquared(axis))) {
        throw std::invalid_argument{std::format(
            "transform rotation axis ({}, {}, {}) has no usable direction", axis.x, axis.y, axis.z)};
    }
    constexpr double degrees_to_radians{std::numbers::pi_v<double> / 180};
    Affine forward{};
    Affine backward{};
    forward.linear = rotationMatrix(normalized(axis), degrees * degrees_to_radians);
    backward.linear = transposed(forward.linear);
    return Transform{forward, backward};
}

Transform Transform::operator*(const Transform& first) const
{
    const Affine forward{composed(forward_map, first.forward_map)};
    const Affine backward{composed(first.inverse_map, inverse_map)};
    if (!isFiniteMap(forward) || !isFiniteMap(backward)) {
        throw std::invalid_argument{"composed transform has a non-finite entry"};
    }
    return Transform{forward, backward};
}

Box3 Transform::applyBox(const Box3& box) const
{
    if (box.isEmpty()) {
        return {};
    }
    const std::array<double, 3> offset{forward_map.offset.x, forward_map.offset.y, forward_map.offset.z};
    std::array<AxisRange, 3> ranges{};
    for (std::size_t axis{0}; axis < 3; ++axis) {
        ranges[axis] = transformedRange(forward_map.linear[axis], offset[axis], box);
    }
    return {{ranges[0].min, ranges[1].min, ranges[2].min}, {ranges[0].max, ranges[1].max, ranges[2].max}};
}

} // namespace albedo_b200
