// The film's resolve: per-pixel FP64 accumulators to 8-bit sRGB, 3 bytes a pixel,
// rows from the top — the bytes the reference's writePpm writes for
// PixelBuffer::average (image/ppm.cpp:22-33, image/pixel_buffer.cpp:37-45,
// color/srgb.cpp:18-36).
//
// The average is sum / count in FP64, correctly rounded as on the host; a count
// that is a power of two multiplies by its exact reciprocal instead, which rounds
// the same real number the same way. The byte comes from the host's tables: 255
// thresholds (the smallest double of each byte, found with the reference's own
// transfer function) and a start byte per bucket of doubles (exponent and top 7
// mantissa bits) that holds at most one threshold. One table read and one
// comparison settle a channel, so the result is the reference's byte exactly and
// the kernel evaluates no power function. A pure stream: 32 bytes read and 3
// written per pixel.
#include "launch.hpp"

#include <algorithm>
#include <cstdint>

namespace albedo_b200 {

namespace {

// Build-time launch shape: pixels per thread (a multiple of 4, so a thread's
// output is whole aligned 32-bit words) and the minimum resident blocks per SM
// the register budget must allow.
#ifndef ALBEDO_RESOLVE_GROUP
#define ALBEDO_RESOLVE_GROUP 4
#endif
#ifndef ALBEDO_RESOLVE_MIN_BLOCKS
#define ALBEDO_RESOLVE_MIN_BLOCKS 1
#endif

constexpr int kResolveThreads{256};
constexpr int kResolveGroup{ALBEDO_RESOLVE_GROUP};
static_assert(kResolveGroup % 4 == 0, "a thread's pixels must fill whole 32-bit words");

__device__ __forceinline__ unsigned int srgbByteOf(double v, double lowest, double highest, const double* lower,
                                                   const unsigned char* start)
{
    // NaN, zero and negative averages fail the first test (byte 0); 1.0 and
    // above pass the second (byte 255). Between them v lies in a bucket:
    // lower[1] > 2^-13 and lower[255] <= 1.
    if (!(v >= lowest)) {
        return 0u;
    }
    if (v >= highest) {
        return 255u;
    }
    const int bucket{static_cast<int>((__double_as_longlong(v) >> kResolveBucketShift) - kResolveBucketBase)};
    const unsigned int b{start[bucket]};
    return b + (v >= lower[b + 1] ? 1u : 0u);
}

// PixelBuffer::average (image/pixel_buffer.cpp:37-45): the count is unsigned.
struct Divisor {
    unsigned long long count;
    double reciprocal;  // 2^-k when count = 2^k, else 0
};

__device__ __forceinline__ Divisor divisorOf(unsigned long long count)
{
    const bool power_of_two{count != 0 && (count & (count - 1)) == 0};
    const long long k{63 - __clzll(static_cast<long long>(count))};
    return {count, power_of_two ? __longlong_as_double((1023 - k) << 52) : 0.0};
}

__device__ __forceinline__ double averageOf(double sum, const Divisor& d)
{
    if (d.count == 0) {
        return 0.0;
    }
    return d.reciprocal != 0.0 ? sum * d.reciprocal : sum / static_cast<double>(d.count);
}

// ALIGNED: accumulators 16-byte aligned (two 16-byte loads a pixel) and the
// output 4-byte aligned (word stores); otherwise 8-byte loads and byte stores.
// Each thread resolves kResolveGroup consecutive pixels per grid-stride turn.
template <bool ALIGNED>
__global__ void __launch_bounds__(kResolveThreads, ALBEDO_RESOLVE_MIN_BLOCKS) resolveSrgbKernel(const PixelAccum* __restrict__ accum,
                                                                      long long pixels,
                                                                      unsigned char* __restrict__ out,
                                                                      SrgbThresholds table)
{
    __shared__ double lower[256];
    __shared__ unsigned char start[kResolveBuckets];
    for (int i{static_cast<int>(threadIdx.x)}; i < 256; i += blockDim.x) {
        lower[i] = table.lower[i];
    }
    for (int i{static_cast<int>(threadIdx.x)}; i < kResolveBuckets; i += blockDim.x) {
        start[i] = table.start[i];
    }
    __syncthreads();
    const double lowest{lower[1]};
    const double highest{lower[255]};

    const long long groups{(pixels + kResolveGroup - 1) / kResolveGroup};
    const long long stride{static_cast<long long>(gridDim.x) * blockDim.x};
    for (long long g{static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x}; g < groups; g += stride) {
        const long long first{g * kResolveGroup};
        const int n{static_cast<int>(min(static_cast<long long>(kResolveGroup), pixels - first))};
        unsigned int bytes[3 * kResolveGroup];
#pragma unroll
        for (int p{0}; p < kResolveGroup; ++p) {
            double r{0.0}, gr{0.0}, bl{0.0};
            unsigned long long count{0};
            if (p < n) {
                const PixelAccum* a{accum + first + p};
                if constexpr (ALIGNED) {
                    const double2 rg{__ldcs(reinterpret_cast<const double2*>(a))};
                    const double2 bc{__ldcs(reinterpret_cast<const double2*>(a) + 1)};
                    r = rg.x;
                    gr = rg.y;
                    bl = bc.x;
                    count = static_cast<unsigned long long>(__double_as_longlong(bc.y));
                } else {
                    r = __ldcs(&a->r);
                    gr = __ldcs(&a->g);
                    bl = __ldcs(&a->b);
                    count = static_cast<unsigned long long>(__ldcs(&a->count));
                }
            }
            const Divisor d{divisorOf(count)};
            bytes[3 * p + 0] = srgbByteOf(averageOf(r, d), lowest, highest, lower, start);
            bytes[3 * p + 1] = srgbByteOf(averageOf(gr, d), lowest, highest, lower, start);
            bytes[3 * p + 2] = srgbByteOf(averageOf(bl, d), lowest, highest, lower, start);
        }
        unsigned char* dst{out + 3 * first};
        if (ALIGNED && n == kResolveGroup) {
            unsigned int* words{reinterpret_cast<unsigned int*>(dst)};
#pragma unroll
            for (int w{0}; w < 3 * kResolveGroup / 4; ++w) {
                __stcs(words + w, bytes[4 * w] | bytes[4 * w + 1] << 8 | bytes[4 * w + 2] << 16 |
                                      bytes[4 * w + 3] << 24);
            }
        } else {
#pragma unroll
            for (int i{0}; i < 3 * kResolveGroup; ++i) {
                if (i < 3 * n) {
                    dst[i] = static_cast<unsigned char>(bytes[i]);
                }
            }
        }
    }
}

} // namespace

cudaError_t launchResolveSrgb(const PixelAccum* accum, long long pixels, unsigned char* out,
                              const SrgbThresholds& table, cudaStream_t stream)
{
    if (pixels <= 0) {
        return cudaSuccess;
    }
    int device{0};
    int sms{0};
    cudaError_t e{cudaGetDevice(&device)};
    if (e == cudaSuccess) {
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    }
    if (e != cudaSuccess) {
        return e;
    }
    // A grid-stride stream, one wave of resident blocks: all of them keep
    // loads in flight, enough to saturate HBM.
    const bool aligned{(reinterpret_cast<std::uintptr_t>(accum) & 15) == 0 &&
                       (reinterpret_cast<std::uintptr_t>(out) & 3) == 0};
    const auto kernel{aligned ? resolveSrgbKernel<true> : resolveSrgbKernel<false>};
    int per_sm{0};
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kResolveThreads, 0);
    if (e != cudaSuccess) {
        return e;
    }
    const long long groups{(pixels + kResolveGroup - 1) / kResolveGroup};
    const long long wanted{(groups + kResolveThreads - 1) / kResolveThreads};
    const int blocks{static_cast<int>(std::min(wanted, static_cast<long long>(std::max(per_sm, 1)) * sms))};
    kernel<<<blocks, kResolveThreads, 0, stream>>>(accum, pixels, out, table);
    return cudaGetLastError();
}

} // namespace albedo_b200
