#include "srgb.hpp"

#include <algorithm>
#include <bit>
#include <cmath>
#include <format>
#include <fstream>
#include <limits>
#include <stdexcept>
#include <string>
#include <system_error>

namespace albedo_b200 {

namespace {

// IEC 61966-2-1:1999 constants, as the reference spells them (color/srgb.cpp:11-15).
constexpr double linear_segment_end{0.0031308};
constexpr double linear_slope{12.92};
constexpr double power_scale{1.055};
constexpr double power_offset{0.055};
constexpr double inverse_gamma{1 / 2.4};

SrgbTable buildTable()
{
    SrgbTable table{};
    table.lower[0] = -std::numeric_limits<double>::infinity();
    // Positive doubles order like their bit patterns; +0 has byte 0 and 1.0 has
    // byte 255, so for every b the boundary lies in (bits(0), bits(1)].
    const std::uint64_t zero_bits{std::bit_cast<std::uint64_t>(0.0)};
    const std::uint64_t one_bits{std::bit_cast<std::uint64_t>(1.0)};
    for (int b{1}; b <= 255; ++b) {
        std::uint64_t lo{zero_bits};
        std::uint64_t hi{one_bits};
        while (hi - lo > 1) {
            const std::uint64_t mid{lo + (hi - lo) / 2};
            if (srgbByte(std::bit_cast<double>(mid)) >= b) {
                hi = mid;
            } else {
                lo = mid;
            }
        }
        table.lower[static_cast<std::size_t>(b)] = std::bit_cast<double>(hi);
    }
    if (!(table.lower[1] > 0x1p-13) || !(table.lower[255] <= 1.0)) {
        throw std::logic_error{"sRGB thresholds outside the bucketed range"};
    }
    // The byte at a value: the number of thresholds at or below it.
    const auto byteAt = [&](double v) {
        return static_cast<int>(std::upper_bound(table.lower.begin() + 1, table.lower.end(), v) -
                                (table.lower.begin() + 1));
    };
    for (int k{0}; k < kSrgbBuckets; ++k) {
        const std::int64_t first_bits{(kSrgbBucketBase + k) << (52 - kSrgbBucketBits)};
        const double first{std::bit_cast<double>(first_bits)};
        const double last{std::bit_cast<double>(first_bits + (std::int64_t{1} << (52 - kSrgbBucketBits)) - 1)};
        const int low{byteAt(first)};
        if (byteAt(last) > low + 1) {
            throw std::logic_error{"an sRGB bucket holds more than one threshold"};
        }
        table.start[static_cast<std::size_t>(k)] = static_cast<std::uint8_t>(low);
    }
    return table;
}

// Removes a half-written output (image/ppm.cpp:38-45): only a regular file at
// `path` itself, never a device such as /dev/full or a symlink's target.
void discardPartialFile(std::ofstream& file, const std::filesystem::path& path) noexcept
{
    file.close();
    std::error_code ignored;
    if (std::filesystem::is_regular_file(std::filesystem::symlink_status(path, ignored))) {
        std::filesystem::remove(path, ignored);
    }
}

} // namespace

double encodeSrgb(double linear) noexcept
{
    if (linear <= linear_segment_end) {
        return linear_slope * linear;
    }
    return power_scale * std::pow(linear, inverse_gamma) - power_offset;
}

std::uint8_t srgbByte(double linear) noexcept
{
    const double encoded{encodeSrgb(linear)};
    if (!(encoded > 0)) {
        return 0;
    }
    if (encoded >= 1) {
        return 255;
    }
    return static_cast<std::uint8_t>(std::lround(encoded * 255));
}

const SrgbTable& srgbTable()
{
    static const SrgbTable table{buildTable()};
    return table;
}

void writePpm(const std::filesystem::path& path, const std::uint8_t* rgb, int width, int height)
{
    if (width <= 0 || height <= 0 ||
        static_cast<std::uint64_t>(width) > (std::uint64_t{1} << 28) / static_cast<std::uint64_t>(height)) {
        throw std::invalid_argument{
            std::format("invalid image size {}x{}: dimensions must be positive and the image at most {} pixels",
                        width, height, std::uint64_t{1} << 28)};
    }
    const std::string text{path.string()};
    std::ofstream file{path, std::ios::binary | std::ios::trunc};
    if (!file) {
        throw std::runtime_error{std::format("cannot open '{}' for writing", text)};
    }
    file << std::format("P6\n{} {}\n255\n", width, height);
    const std::streamsize row_bytes{static_cast<std::streamsize>(width) * 3};
    for (int y{0}; y < height; ++y) {
        file.write(reinterpret_cast<const char*>(rgb) + static_cast<std::ptrdiff_t>(y) * row_bytes, row_bytes);
    }
    if (!file) {
        discardPartialFile(file, path);
        throw std::runtime_error{std::format("failed to write '{}': failed to write PPM image", text)};
    }
    file.close();
    if (!file) {
        discardPartialFile(file, path);
        throw std::runtime_error{std::format("failed to write '{}'", text)};
    }
}

} // namespace albedo_b200
