// A wavefront render that allocates nothing: its path slots, queues, control
// block and job record live in one file-scope device array, so a caller that
// cannot call cudaMalloc can still render. Who needs that: a program whose
// device memory is owned up front by another allocator (a framework's caching
// pool that has reserved the GPU), and a loop with a latency budget, where an
// allocation can synchronize the device or stall on the driver.
//
// The array is sized for kNoAllocMaxSlots path slots, one per pixel, so images
// of at most 65,536 pixels fit; larger ones are rejected. Every GPU that loads
// the library holds the array (about 17 MB) until the process exits. Every call
// shares it and it keeps the last call's contents: each call clears what must
// start at zero (queues, counters, slot ownership) before use, and calls whose
// work overlaps on the GPU race on it, so callers must not overlap them.
#include "wavefront.cuh"

#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>

namespace albedo_b200 {

namespace {

constexpr int kNoAllocMaxSlots = 65536;
constexpr std::size_t kMaxDevices = 64;

constexpr std::size_t alignUp(std::size_t n) { return (n + 255) & ~static_cast<std::size_t>(255); }

constexpr std::size_t kF4 = alignUp(sizeof(float4) * kNoAllocMaxSlots);
constexpr std::size_t kF2 = alignUp(sizeof(float2) * kNoAllocMaxSlots);
constexpr std::size_t kU2 = alignUp(sizeof(ulonglong2) * kNoAllocMaxSlots);
constexpr std::size_t kQueue = alignUp(sizeof(int) * kNoAllocMaxSlots);
constexpr std::size_t kControl = alignUp(sizeof(WfControl));
constexpr std::size_t kJob = alignUp(sizeof(WfJob));
constexpr std::size_t kJobDone = alignUp(sizeof(unsigned long long));
constexpr std::size_t kScratchBytes = 12 * kF4 + kF2 + kU2 + kQueueCount * kQueue + kControl + kJob + kJobDone;

// The scratch. In host code this name is a host-side stand-in, not a device
// address; the host passes the address cudaGetSymbolAddress returns.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_address[kMaxDevices] = {};

// Once per device, with that device current: the device address of the
// scratch. The address is kept for the life of the process, so rendering on a
// device after cudaDeviceReset (which ends the context the address belongs
// to) is not supported.
cudaError_t scratchAddress(void** out)
{
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) {
        return e;
    }
    if (device < 0 || static_cast<std::size_t>(device) >= kMaxDevices) {
        return cudaErrorInvalidDevice;
    }
    const std::lock_guard<std::mutex> lock{g_setup_mutex};
    if (g_scratch_address[device] == nullptr) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) {
            return e;
        }
        g_scratch_address[device] = ptr;
    }
    *out = g_scratch_address[device];
    return cudaSuccess;
}

WfBuffers carve(void* base, int slots, WfJob** job)
{
    auto* p = static_cast<unsigned char*>(base);
    const auto take = [&](std::size_t bytes) {
        void* r = p;
        p += bytes;
        return r;
    };
    WfBuffers b{};
    WfSlots& s = b.slots;
    s.ray_o = static_cast<float4*>(take(kF4));
    s.ray_d = static_cast<float4*>(take(kF4));
    s.throughput = static_cast<float4*>(take(kF4));
    s.result = static_cast<float4*>(take(kF4));
    s.arrival = static_cast<float4*>(take(kF4));
    s.skip = static_cast<uint4*>(take(kF4));
    s.where = static_cast<int4*>(take(kF4));
    s.hit = static_cast<float4*>(take(kF4));
    s.shadow_o = static_cast<float4*>(take(kF4));
    s.shadow_d = static_cast<float4*>(take(kF4));
    s.shadow_skip = static_cast<uint4*>(take(kF4));
    s.shadow_c = static_cast<float4*>(take(kF4));
    s.hit_b = static_cast<float2*>(take(kF2));
    s.rng = static_cast<ulonglong2*>(take(kU2));
    for (int q = 0; q < kQueueCount; ++q) {
        b.queue[q] = static_cast<int*>(take(kQueue));
    }
    b.control = static_cast<WfControl*>(take(kControl));
    *job = static_cast<WfJob*>(take(kJob));
    b.job_done = static_cast<unsigned long long*>(take(kJobDone));
    b.slot_count = slots;
    return b;
}

} // namespace

int noAllocMaxPixels() { return kNoAllocMaxSlots; }

// Renders one job with one path slot per pixel inside the static scratch.
// Returns cudaSuccess, a CUDA error, or cudaErrorLaunchTimeout if the render
// is not complete within its iteration bound.
cudaError_t renderNoAlloc(const WfJob& job, int stack, int blocks, unsigned int* error_flag, cudaStream_t stream)
{
    const long long pixels = static_cast<long long>(job.width) * job.height;
    if (pixels <= 0 || pixels > kNoAllocMaxSlots) {
        return cudaErrorInvalidValue;
    }
    void* base = nullptr;
    cudaError_t e = scratchAddress(&base);
    if (e != cudaSuccess) {
        return e;
    }
    WfJob* device_job = nullptr;
    const WfBuffers buffers = carve(base, static_cast<int>(pixels), &device_job);
    WfJob staged = job;
    staged.item_begin = 0;
    staged.item_end = pixels;
    if ((e = cudaMemcpyAsync(device_job, &staged, sizeof(WfJob), cudaMemcpyHostToDevice, stream)) != cudaSuccess) {
        return e;
    }
    if ((e = wfPrepare(stack)) != cudaSuccess) {
        return e;
    }
    const auto total = static_cast<unsigned long long>(pixels);
    if ((e = wfReset(buffers, total, 1, stream)) != cudaSuccess) {
        return e;
    }
    int per_sm = 1;
    int device = 0;
    int sms = 1;
    if ((e = wfTraceBlocksPerSm(stack, &per_sm)) != cudaSuccess || (e = cudaGetDevice(&device)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) {
        return e;
    }
    const WfLaunch launch{blocks, 128, stack, per_sm * sms, 32, 0};
    // A slot finishes its pixel within n^2 (max_depth + 2) iterations: the
    // total iteration bound (computed in 64 bits; max_depth may be near INT_MAX).
    const unsigned long long bound = static_cast<unsigned long long>(job.samples_per_axis) * job.samples_per_axis *
                                         (static_cast<unsigned long long>(job.max_depth) + 2) +
                                     16;
    constexpr int kIterationsPerCheck = 8;
    WfControl snapshot{};
    for (unsigned long long done = 0; done <= bound; done += kIterationsPerCheck) {
        for (int i = 0; i < kIterationsPerCheck; ++i) {
            if ((e = wfIteration(device_job, buffers, launch, error_flag, stream)) != cudaSuccess) {
                return e;
            }
        }
        if ((e = cudaMemcpyAsync(&snapshot, buffers.control, sizeof(WfControl), cudaMemcpyDeviceToHost, stream)) !=
            cudaSuccess) {
            return e;
        }
        if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) {
            return e;
        }
        if (snapshot.completed >= total) {
            return cudaSuccess;
        }
    }
    return cudaErrorLaunchTimeout;
}

} // namespace albedo_b200
