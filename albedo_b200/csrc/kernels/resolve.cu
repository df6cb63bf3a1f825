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
// comparison settle a channel (the tiled kernel packs both tables into one
// 64-bit entry per bucket), so the result is the reference's byte exactly and
// the kernel evaluates no power function. A pure stream: 32 bytes read and 3
// written per pixel, the reads as one coalesced 256-bit load per pixel.
#include "launch.hpp"

#include <algorithm>
#include <cstdint>

namespace albedo_b200 {

namespace {

// Build-time launch shape: pixels per lane in a warp's tile and the minimum
// resident blocks per SM the register budget must allow.
#ifndef ALBEDO_RESOLVE_GROUP
#define ALBEDO_RESOLVE_GROUP 4
#endif
#ifndef ALBEDO_RESOLVE_MIN_BLOCKS
#define ALBEDO_RESOLVE_MIN_BLOCKS 4
#endif

constexpr int kResolveThreads{256};
constexpr int kResolveGroup{ALBEDO_RESOLVE_GROUP};

__device__ __forceinline__ unsigned int srgbByteOf(double v, double lowest, double highest, const double* lower,
                                                   const unsigned char* start)
{
    // Without branches: NaN, zero and negative averages fail `in_range` (byte
    // 0); 1.0 and above pass `saturated` (byte 255). Between them v lies in a
    // bucket, since lower[1] > 2^-13 and lower[255] <= 1; outside, the bucket
    // and the start byte are clamped so every table read stays in bounds, and
    // the selects discard what they give. The bucket is the high word of v
    // shifted right by kResolveBucketShift - 32.
    const bool in_range{v >= lowest};
    const bool saturated{v >= highest};
    const int bucket{min(max((__double2hiint(v) >> (kResolveBucketShift - 32)) -
                                 static_cast<int>(kResolveBucketBase),
                             0),
                         kResolveBuckets - 1)};
    const unsigned int b{min(static_cast<unsigned int>(start[bucket]), 254u)};
    const unsigned int byte{b + (v >= lower[b + 1] ? 1u : 0u)};
    return saturated ? 255u : (in_range ? byte : 0u);
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

// The tables into shared memory; every thread takes part.
__device__ __forceinline__ void loadTables(const SrgbThresholds& table, double* lower, unsigned char* start)
{
    for (int i{static_cast<int>(threadIdx.x)}; i < 256; i += blockDim.x) {
        lower[i] = table.lower[i];
    }
    for (int i{static_cast<int>(threadIdx.x)}; i < kResolveBuckets; i += blockDim.x) {
        start[i] = table.start[i];
    }
    __syncthreads();
}

// One pixel's accumulator in one 256-bit load (sm_100 global vector load), marked
// streaming: each accumulator is read once. The address is 32-byte aligned.
__device__ __forceinline__ void loadPixel(const PixelAccum* a, double& r, double& g, double& b,
                                          unsigned long long& count)
{
    double c;
    asm("ld.global.cs.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(r), "=d"(g), "=d"(b), "=d"(c)
                 : "l"(a));
    count = static_cast<unsigned long long>(__double_as_longlong(c));
}

constexpr int kResolveWarps{kResolveThreads / 32};
constexpr int kTilePixels{32 * kResolveGroup};
constexpr int kTileBytes{3 * kTilePixels};  // 96 * kResolveGroup: whole 16-byte units

// The tiled kernel's form of the tables: one 64-bit entry per bucket, read
// with one shared-memory load. Bits 48-55 hold the bucket's start byte s;
// bits 0-45 hold the low kResolveBucketShift bits of lower[s + 1] when that
// threshold lies in the bucket, else 2^kResolveBucketShift (above every value's
// low bits). Doubles of one bucket share their high bits, so comparing low bits
// compares the values.
constexpr unsigned long long kLowBits{(1ull << kResolveBucketShift) - 1};
constexpr unsigned long long kNoThreshold{1ull << kResolveBucketShift};

__device__ __forceinline__ void packBuckets(const SrgbThresholds& table, unsigned long long* packed)
{
    for (int k{static_cast<int>(threadIdx.x)}; k < kResolveBuckets; k += blockDim.x) {
        const unsigned int s{table.start[k]};
        unsigned long long low{kNoThreshold};
        if (s < 255) {
            const long long t{__double_as_longlong(table.lower[s + 1])};
            if ((t >> kResolveBucketShift) == kResolveBucketBase + k) {
                low = static_cast<unsigned long long>(t) & kLowBits;
            }
        }
        packed[k] = static_cast<unsigned long long>(s) << 48 | low;
    }
    __syncthreads();
}

// srgbByteOf with the packed table: one table read per channel.
__device__ __forceinline__ unsigned int srgbBytePacked(double v, double lowest, double highest,
                                                       const unsigned long long* packed)
{
    const bool in_range{v >= lowest};
    const bool saturated{v >= highest};
    const int bucket{min(max((__double2hiint(v) >> (kResolveBucketShift - 32)) -
                                 static_cast<int>(kResolveBucketBase),
                             0),
                         kResolveBuckets - 1)};
    const unsigned long long entry{packed[bucket]};
    const unsigned long long low{static_cast<unsigned long long>(__double_as_longlong(v)) & kLowBits};
    const unsigned int byte{static_cast<unsigned int>(entry >> 48) +
                            (low >= (entry & (kNoThreshold | kLowBits)) ? 1u : 0u)};
    return saturated ? 255u : (in_range ? byte : 0u);
}

// One warp tile into the warp's stage: lane l resolves pixels l, l + 32, ...
// of the tile's n. FULL tiles (n == kTilePixels) need no bounds tests, so the
// loads and the byte computations run as straight-line code the compiler can
// interleave.
template <bool FULL>
__device__ __forceinline__ void resolveTile(const PixelAccum* tile, int n, int lane, unsigned char* stage,
                                            double lowest, double highest, const unsigned long long* packed)
{
    double r[kResolveGroup], g[kResolveGroup], b[kResolveGroup];
    unsigned long long count[kResolveGroup];
#pragma unroll
    for (int j{0}; j < kResolveGroup; ++j) {
        const int q{lane + 32 * j};
        r[j] = g[j] = b[j] = 0.0;
        count[j] = 0;
        if (FULL || q < n) {
            loadPixel(tile + q, r[j], g[j], b[j], count[j]);
        }
    }
#pragma unroll
    for (int j{0}; j < kResolveGroup; ++j) {
        const int q{lane + 32 * j};
        if (FULL || q < n) {
            const Divisor d{divisorOf(count[j])};
            stage[3 * q + 0] =
                static_cast<unsigned char>(srgbBytePacked(averageOf(r[j], d), lowest, highest, packed));
            stage[3 * q + 1] =
                static_cast<unsigned char>(srgbBytePacked(averageOf(g[j], d), lowest, highest, packed));
            stage[3 * q + 2] =
                static_cast<unsigned char>(srgbBytePacked(averageOf(b[j], d), lowest, highest, packed));
        }
    }
}

// Accumulators 32-byte aligned and output 16-byte aligned. Each warp resolves
// tiles of kTilePixels pixels: lane l takes pixels l, l + 32, ..., so each of
// its kResolveGroup loads is one coalesced 1 KB read across the warp. The bytes
// are transposed through the warp's shared-memory stage and leave as coalesced
// 16-byte stores.
__global__ void __launch_bounds__(kResolveThreads, ALBEDO_RESOLVE_MIN_BLOCKS)
    resolveSrgbTiles(const PixelAccum* __restrict__ accum, long long pixels, unsigned char* __restrict__ out,
                     SrgbThresholds table)
{
    __shared__ unsigned long long packed[kResolveBuckets];
    __shared__ __align__(16) unsigned char stage[kResolveWarps][kTileBytes];
    packBuckets(table, packed);
    const double lowest{table.lower[1]};
    const double highest{table.lower[255]};
    const int lane{static_cast<int>(threadIdx.x) & 31};
    const int warp{static_cast<int>(threadIdx.x) >> 5};
    unsigned char* my_stage{stage[warp]};

    const long long tiles{(pixels + kTilePixels - 1) / kTilePixels};
    const long long warps_total{static_cast<long long>(gridDim.x) * kResolveWarps};
    for (long long t{static_cast<long long>(blockIdx.x) * kResolveWarps + warp}; t < tiles; t += warps_total) {
        const long long first{t * kTilePixels};
        const int n{static_cast<int>(min(static_cast<long long>(kTilePixels), pixels - first))};
        if (n == kTilePixels) {
            resolveTile<true>(accum + first, n, lane, my_stage, lowest, highest, packed);
        } else {
            resolveTile<false>(accum + first, n, lane, my_stage, lowest, highest, packed);
        }
        __syncwarp();
        unsigned char* dst{out + 3 * first};
        if (n == kTilePixels) {
            for (int i{lane}; i < kTileBytes / 16; i += 32) {
                __stcs(reinterpret_cast<uint4*>(dst) + i, reinterpret_cast<const uint4*>(my_stage)[i]);
            }
        } else {
            for (int i{lane}; i < 3 * n; i += 32) {
                dst[i] = my_stage[i];
            }
        }
        __syncwarp();
    }
}

// Any other alignment (accumulators at least 8-byte aligned): one pixel per
// thread per turn, 8-byte loads and byte stores.
__global__ void __launch_bounds__(kResolveThreads) resolveSrgbAnyAlignment(const PixelAccum* __restrict__ accum,
                                                                            long long pixels,
                                                                            unsigned char* __restrict__ out,
                                                                            SrgbThresholds table)
{
    __shared__ double lower[256];
    __shared__ unsigned char start[kResolveBuckets];
    loadTables(table, lower, start);
    const double lowest{lower[1]};
    const double highest{lower[255]};
    const long long stride{static_cast<long long>(gridDim.x) * blockDim.x};
    for (long long p{static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x}; p < pixels; p += stride) {
        const PixelAccum* a{accum + p};
        const Divisor d{divisorOf(static_cast<unsigned long long>(__ldcs(&a->count)))};
        out[3 * p + 0] = static_cast<unsigned char>(srgbByteOf(averageOf(__ldcs(&a->r), d), lowest, highest, lower,
                                                               start));
        out[3 * p + 1] = static_cast<unsigned char>(srgbByteOf(averageOf(__ldcs(&a->g), d), lowest, highest, lower,
                                                               start));
        out[3 * p + 2] = static_cast<unsigned char>(srgbByteOf(averageOf(__ldcs(&a->b), d), lowest, highest, lower,
                                                               start));
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
    const bool tiled{(reinterpret_cast<std::uintptr_t>(accum) & 31) == 0 &&
                     (reinterpret_cast<std::uintptr_t>(out) & 15) == 0};
    const auto kernel{tiled ? resolveSrgbTiles : resolveSrgbAnyAlignment};
    int per_sm{0};
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kResolveThreads, 0);
    if (e != cudaSuccess) {
        return e;
    }
    const long long per_block{tiled ? static_cast<long long>(kTilePixels) * kResolveWarps : kResolveThreads};
    const long long wanted{(pixels + per_block - 1) / per_block};
    const int blocks{static_cast<int>(std::min(wanted, static_cast<long long>(std::max(per_sm, 1)) * sms))};
    kernel<<<blocks, kResolveThreads, 0, stream>>>(accum, pixels, out, table);
    return cudaGetLastError();
}

} // namespace albedo_b200
