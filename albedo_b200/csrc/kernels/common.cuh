// Device math shared by every kernel: float3 arithmetic, the per-pixel PCG32
// stream, stratified camera rays and the sampling warps.
//
// Floating-point policy: directions, points and radiance are FP32; the random
// stream is integer and bit-exact with the reference; per-pixel sums are FP64.
#pragma once

#include "../device_layout.hpp"

#include <cstdint>
#include <cuda_runtime.h>

namespace albedo_b200 {

#define ALB_DEV __device__ __forceinline__

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kInvPiF = 0.318309886183790671538f;

// ------------------------------------------------------------------ float3

ALB_DEV float3 mk(float x, float y, float z) { return make_float3(x, y, z); }
ALB_DEV float3 operator+(float3 a, float3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
ALB_DEV float3 operator-(float3 a, float3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
ALB_DEV float3 operator-(float3 a) { return mk(-a.x, -a.y, -a.z); }
ALB_DEV float3 operator*(float3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
ALB_DEV float3 operator*(float s, float3 a) { return mk(a.x * s, a.y * s, a.z * s); }
ALB_DEV float3 operator*(float3 a, float3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
ALB_DEV float3 operator/(float3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
ALB_DEV float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
ALB_DEV float3 cross(float3 a, float3 b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
ALB_DEV float lengthSquared(float3 v) { return dot(v, v); }
ALB_DEV float3 normalized(float3 v) { return v / sqrtf(lengthSquared(v)); }
ALB_DEV bool isBlack(float3 c) { return c.x == 0.0f && c.y == 0.0f && c.z == 0.0f; }
ALB_DEV float comp(float3 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }
ALB_DEV float3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }
// True for a finite, non-zero, non-subnormal value (std::isnormal).
ALB_DEV bool isNormalF(float x)
{
    const float a = fabsf(x);
    return a >= 1.17549435e-38f && a <= 3.40282347e38f;
}

// ------------------------------------------------------------------ random numbers

// PCG32 (XSH-RR, 64-bit state) seeded as pcg32_srandom_r; restates
// sampling/pcg32.hpp:30-50. The integer stream is bit-exact with the reference.
struct Pcg32 {
    std::uint64_t state;
    std::uint64_t inc;

    ALB_DEV std::uint32_t next()
    {
        const std::uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        const std::uint32_t xorshifted = static_cast<std::uint32_t>(((old >> 18u) ^ old) >> 27u);
        const std::uint32_t rot = static_cast<std::uint32_t>(old >> 59u);
        return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
    }

    ALB_DEV static Pcg32 seeded(std::uint64_t seed, std::uint64_t stream)
    {
        Pcg32 g{0, (stream << 1u) | 1u};
        g.next();
        g.state += seed;
        g.next();
        return g;
    }

    // A value in [0, 1): the reference's u32 * 2^-32 (double) truncated to FP32,
    // i.e. the top 24 bits, so 1.0f is never produced (rounding to nearest would
    // give 1.0f for the largest 128 outputs).
    ALB_DEV float next1D() { return static_cast<float>(next() >> 8u) * 5.9604644775390625e-8f; }
};

// SplitMix64 output function (sampling/sample_generator.hpp:17-22).
ALB_DEV std::uint64_t mixBits(std::uint64_t v)
{
    v = (v ^ (v >> 30u)) * 0xbf58476d1ce4e5b9ULL;
    v = (v ^ (v >> 27u)) * 0x94d049bb133111ebULL;
    return v ^ (v >> 31u);
}

// SampleGenerator::forPixel (sampling/sample_generator.hpp:35-45).
ALB_DEV Pcg32 pixelGenerator(std::uint64_t seed, std::uint32_t x, std::uint32_t y, std::uint32_t width)
{
    const std::uint64_t index = static_cast<std::uint64_t>(y) * width + x;
    return Pcg32::seeded(seed, mixBits(index));
}

// ------------------------------------------------------------------ camera

// PerspectiveCamera::generateRay (camera/perspective_camera.cpp:74-87): film
// (0,0) is the top-left corner; the direction is normalized.
ALB_DEV void cameraRay(const DevCamera& cam, float fx, float fy, float3& origin, float3& dir)
{
    const float horizontal = 2.0f * fx - 1.0f;
    const float vertical = 1.0f - 2.0f * fy;
    const float3 d = ld3(cam.forward) + ld3(cam.half_width) * horizontal + ld3(cam.half_height) * vertical;
    origin = ld3(cam.origin);
    dir = normalized(d);
}

// ------------------------------------------------------------------ warps (sampling/warps.cpp)

// Shirley-Chiu concentric disk, sampling/warps.cpp:8-28.
ALB_DEV float2 concentricDisk(float ux, float uy)
{
    const float ox = 2.0f * ux - 1.0f;
    const float oy = 2.0f * uy - 1.0f;
    if (ox == 0.0f && oy == 0.0f) {
        return make_float2(0.0f, 0.0f);
    }
    float radius;
    float angle;
    if (fabsf(ox) > fabsf(oy)) {
        radius = ox;
        angle = (kPiF / 4.0f) * (oy / ox);
    } else {
        radius = oy;
        angle = (kPiF / 2.0f) - (kPiF / 4.0f) * (ox / oy);
    }
    float s, c;
    sincosf(angle, &s, &c);
    return make_float2(radius * c, radius * s);
}

// Malley's method, sampling/warps.cpp:30-36.
ALB_DEV float3 cosineHemisphere(float ux, float uy)
{
    const float2 d = concentricDisk(ux, uy);
    const float z = sqrtf(fmaxf(0.0f, 1.0f - d.x * d.x - d.y * d.y));
    return mk(d.x, d.y, z);
}

// sampling/warps.cpp:38-45.
ALB_DEV float3 uniformSphere(float ux, float uy)
{
    const float z = 1.0f - 2.0f * ux;
    const float radius = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    const float phi = 2.0f * kPiF * uy;
    float s, c;
    sincosf(phi, &s, &c);
    return mk(radius * c, radius * s, z);
}

ALB_DEV float uniformSpherePdf() { return kInvPiF / 4.0f; }

// ------------------------------------------------------------------ orthonormal basis

// Duff et al. 2017, as core/orthonormal_basis.cpp:17-35.
struct Onb {
    float3 t, b, n;
    ALB_DEV static Onb fromNormal(float3 n)
    {
        const float sign = copysignf(1.0f, n.z);
        const float a = -1.0f / (sign + n.z);
        const float bb = n.x * n.y * a;
        Onb o;
        o.t = mk(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
        o.b = mk(bb, sign + n.y * n.y * a, -n.y);
        o.n = n;
        return o;
    }
    ALB_DEV float3 toLocal(float3 w) const { return mk(dot(w, t), dot(w, b), dot(w, n)); }
    ALB_DEV float3 toWorld(float3 l) const { return t * l.x + b * l.y + n * l.z; }
};

} // namespace albedo_b200
