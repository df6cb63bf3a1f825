// The film's output encoding: linear FP64 radiance to 8-bit sRGB, as the
// reference's encodeSrgb and toByte compute it (color/srgb.cpp:18-36), and the
// binary PPM writer around it (image/ppm.cpp:47-85).
#pragma once

#include <array>
#include <cstdint>
#include <filesystem>

namespace albedo_b200 {

// The IEC 61966-2-1 transfer function, with the reference's constants and
// order of operations (color/srgb.cpp:11-27).
double encodeSrgb(double linear) noexcept;

// toByte(encodeSrgb(linear)) (color/srgb.cpp:29-36): 0 for NaN and values at
// or below 0, 255 from 1 up, else the nearest byte (halves away from zero).
std::uint8_t srgbByte(double linear) noexcept;

// The byte of a linear value as a table of thresholds: lower[b] (b = 1..255) is
// the smallest positive double whose srgbByte is at least b, found by bisection
// over the ordered bit patterns of positive doubles; lower[0] is -infinity. A
// value's byte is the largest b with value >= lower[b], and 0 when no b >= 1
// qualifies (NaN included), which equals srgbByte because srgbByte never
// decreases as its argument grows. The device resolve compares against this
// table, so it needs no transcendental function of its own.
//
// start[k] speeds the search up: it is the byte of the smallest double in bucket
// k, where the buckets split [2^-13, 1) by the double's exponent and the top 7
// bits of its mantissa (bucket k holds the doubles whose bits shifted right by
// 45 equal kSrgbBucketBase + k). No bucket holds more than one threshold (the
// build checks this), so a value's byte is start[k] or start[k] + 1, and one
// comparison with lower[start[k] + 1] decides. Every value with a byte from 1
// to 254 lies in some bucket: lower[1] > 2^-13 and lower[255] <= 1.
inline constexpr int kSrgbBucketBits{7};
inline constexpr std::int64_t kSrgbBucketBase{(1023 - 13) << kSrgbBucketBits};
inline constexpr int kSrgbBuckets{13 << kSrgbBucketBits};
struct SrgbTable {
    std::array<double, 256> lower;
    std::array<std::uint8_t, kSrgbBuckets> start;
};
const SrgbTable& srgbTable();

// writePpm (image/ppm.cpp:47-85) from bytes already encoded: "P6", the size and
// 255, then width*height RGB byte triples, rows from the top. On failure the
// partial file is removed (when it is a regular file) and std::runtime_error
// carries the reference's messages.
void writePpm(const std::filesystem::path& path, const std::uint8_t* rgb, int width, int height);

} // namespace albedo_b200
