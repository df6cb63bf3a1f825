// Host-callable launchers for the CUDA kernels (defined in the .cu files).
#pragma once

#include "../device_layout.hpp"

#include <cstdint>
#include <cuda_runtime.h>

namespace albedo_b200 {

// Per-pixel accumulator, laid out as the reference's PixelBuffer::Accumulator
// (image/pixel_buffer.hpp:53-57): FP64 RGB sum and an int64 sample count.
struct PixelAccum {
    double r, g, b;
    long long count;
};

enum Estimator : int { kEstimatorPath = 0, kEstimatorScatterOnly = 1, kEstimatorNormals = 2 };

struct RenderArgs {
    int width;
    int height;
    int samples_per_axis;
    int estimator;
    unsigned long long seed;
    int max_depth;       // PathEstimator::max_depth / ScatterOnlyEstimator::max_scatter_count
    int roulette_start;
    const int2* pixels;  // optional pixel subset (x, y); null renders the whole image
    int pixel_count;
    double* sum_squares; // optional per-pixel (or per-listed-pixel) sums of squared samples, 3 doubles each
    // Launch shape of the megakernel (the autotuner's knobs): pixel tile width
    // (8, 16 or 32; tiles hold 128 pixels) and register budget (resident blocks
    // per SM the kernel is compiled for: 3 or 4). 0 picks the default (16, 3).
    int tile_width;
    int blocks_per_sm;
    // Nonzero: the traversal is inlined into the kernel (3 blocks per SM, path
    // estimator) instead of called out of line.
    int inline_traversal;
    // Per-pixel sums inside the kernel: kAccumulateFp64, or kAccumulateKahan
    // (compensated FP32, path estimator only). Either is added to the FP64
    // accumulators at the end.
    int accumulation;
};

enum Accumulation : int { kAccumulateFp64 = 0, kAccumulateKahan = 1 };

// Stack capacity (entries per thread) of the kernel chosen for a scene, or 0 if
// the scene's hierarchy is deeper than every compiled variant supports.
int stackCapacityFor(std::uint32_t stack_need);

// Traversal-stack capacities the kernels are compiled for (8 bytes per entry per
// thread of shared memory; 48 entries keep four 128-thread blocks per SM).
template <int S>
struct StackSize {
    static constexpr int value = S;
};

// Calls f(StackSize<S>{}) for the compiled capacity S that `capacity` names.
template <typename F>
auto withStack(int capacity, F&& f)
{
    if (capacity <= 32) {
        return f(StackSize<32>{});
    }
    if (capacity <= 48) {
        return f(StackSize<48>{});
    }
    return f(StackSize<64>{});
}

// Lets `kernel` use `entries` stack entries of dynamic shared memory per thread
// in 128-thread blocks (above the 48 KB default when needed).
template <typename Kernel>
cudaError_t allowStackMemory(Kernel kernel, int entries, int entry_bytes = static_cast<int>(sizeof(uint2)))
{
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, entries * 128 * entry_bytes);
}

// The plain megakernel: one thread per pixel, serial over that pixel's n x n
// stratified samples so each pixel's PCG32 stream is consumed as the
// reference consumes it. Adds into `accum` (one PixelAccum per pixel, or per
// listed pixel when args.pixels is set).
cudaError_t launchMegakernel(const DevScene& scene, const DevCamera& camera, const RenderArgs& args, PixelAccum* accum,
                             unsigned int* error_flag, int stack_capacity, cudaStream_t stream);

// The megakernel (path estimator) counting its traversal work into
// totals[0..5] = child boxes tested, triangles tested, spheres tested,
// instances entered, queries traced, boxes the reference's binary traversal
// tests for the same queries. Not used for timing.
cudaError_t launchMegakernelCounting(const DevScene& scene, const DevCamera& camera, const RenderArgs& args,
                                     PixelAccum* accum, unsigned int* error_flag, int stack_capacity,
                                     unsigned long long* totals, cudaStream_t stream);

// Ray queries: rays are 6 floats (origin, direction). Closest hit in (t_min,
// t_max): hit flag, t, object id, triangle id within its mesh (-1 for spheres),
// point, geometric normal facing the ray, shading normal, front-face flag.
struct TraceOutputs {
    int* hit;
    float* t;
    int* object;
    int* triangle;
    float* point;
    float* normal;
    float* shading_normal;
    int* front;
};
// Closest-hit queries of given rays counting their work into totals[0..5].
cudaError_t launchTraceCounting(const DevScene& scene, const float* rays, int count, float t_min, float t_max,
                                unsigned int* error_flag, int stack_capacity, unsigned long long* totals,
                                cudaStream_t stream);
cudaError_t launchTrace(const DevScene& scene, const float* rays, int count, float t_min, float t_max,
                        const TraceOutputs& out, unsigned int* error_flag, int stack_capacity, cudaStream_t stream);
// Any hit in (0, t_max[i]).
cudaError_t launchOccluded(const DevScene& scene, const float* rays, const float* t_max, int count, int* occluded,
                           unsigned int* error_flag, int stack_capacity, cudaStream_t stream);

// The film's resolve to 8-bit sRGB (3 bytes a pixel) from per-pixel averages,
// by comparison against a table of the smallest double of each byte (lower[b],
// b = 1..255; lower[0] is unused). start[k] is the byte at the smallest double of
// bucket k: the doubles whose bits shifted right by 45 equal kResolveBucketBase +
// k, each holding at most one threshold (the host builds and checks both tables).
constexpr int kResolveBucketShift{45};
constexpr long long kResolveBucketBase{(1023 - 13) << 7};
constexpr int kResolveBuckets{13 << 7};
struct SrgbThresholds {
    double lower[256];
    unsigned char start[kResolveBuckets];
};
cudaError_t launchResolveSrgb(const PixelAccum* accum, long long pixels, unsigned char* out,
                              const SrgbThresholds& table, cudaStream_t stream);

// Probe kernels for parity tests of device arithmetic.
cudaError_t launchPixelStream(unsigned long long seed, int x, int y, int width, int count, unsigned int* out_u32,
                              float* out_real, cudaStream_t stream);
cudaError_t launchLobeEval(int kind, const float* params, const float* wo_wi, int count, float* out_f, float* out_pdf,
                           cudaStream_t stream);
cudaError_t launchLobeSample(int kind, const float* params, const float* inputs, int count, int* out_valid,
                             float* out_dir, float* out_weight, float* out_pdf, int* out_specular, cudaStream_t stream);
cudaError_t launchPerlin(const float* points, int count, float* out_noise, float* out_turbulence, cudaStream_t stream);
// Reads `bytes` (a multiple of 16, 16-byte aligned) `repeats` times through L2.
cudaError_t launchReadSweep(const void* data, long long bytes, int repeats, int blocks, void* sink,
                            cudaStream_t stream);
cudaError_t launchCameraRays(const DevCamera& camera, const float* film, int count, float* out_rays,
                             cudaStream_t stream);

} // namespace albedo_b200
