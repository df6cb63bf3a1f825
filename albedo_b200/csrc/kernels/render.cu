// The plain per-pixel megakernel and the ray-query kernels.
//
// renderPixel (render/render_image.cpp:27-44): each pixel owns one PCG32 stream
// and draws its n x n stratified samples from it in row-major order, so one
// thread runs one pixel's samples serially. Blocks cover tiles of 128 pixels
// (16 x 8 by default) so a warp's camera rays start coherent. The traversal stack of every thread sits in
// shared memory (STACK entries of 8 bytes).
#include "estimator.cuh"

#include <type_traits>

namespace albedo_b200 {

namespace {

constexpr int kBlock = 128;
constexpr int kTileW = 16; // default tile: 16 x 8 pixels
// Resident blocks per SM the megakernel's register budget is sized for by
// default: 3 (168 registers a thread) measured 4-12% faster than 4 (128
// registers, with local-memory spills) on the room and trefoil scenes. The
// path estimator is also compiled for 4; the autotuner picks per scene.
#ifndef ALBEDO_MEGA_BLOCKS_PER_SM
#define ALBEDO_MEGA_BLOCKS_PER_SM 3
#endif
constexpr int kMegaBlocksPerSm = ALBEDO_MEGA_BLOCKS_PER_SM;

// Per-pixel running sums: FP64, or FP32 with Kahan compensation.
template <int ACC>
struct PixelSums;

// reset() zeroes them.
template <>
struct PixelSums<kAccumulateFp64> {
    double r, g, b;
    ALB_DEV void reset() { r = g = b = 0.0; }
    ALB_DEV void add(float3 v)
    {
        r += v.x;
        g += v.y;
        b += v.z;
    }
    ALB_DEV double3 total() const { return make_double3(r, g, b); }
};

template <>
struct PixelSums<kAccumulateKahan> {
    float r, g, b;
    float cr, cg, cb;
    ALB_DEV void reset() { r = g = b = cr = cg = cb = 0.0f; }
    // Kahan 1965: c carries the low-order part lost by the previous addition.
    static ALB_DEV void kahan(float& sum, float& c, float v)
    {
        const float y = __fsub_rn(v, c);
        const float t = __fadd_rn(sum, y);
        c = __fsub_rn(__fsub_rn(t, sum), y);
        sum = t;
    }
    ALB_DEV void add(float3 v)
    {
        kahan(r, cr, v.x);
        kahan(g, cg, v.y);
        kahan(b, cb, v.z);
    }
    ALB_DEV double3 total() const
    {
        return make_double3(static_cast<double>(r) - cr, static_cast<double>(g) - cg, static_cast<double>(b) - cb);
    }
};

// A path's state kept in shared memory by the lean variants: 23 words a thread
// (an odd stride, so a warp's accesses to one field hit 32 different banks).
struct alignas(4) SharedPath {
    PathState p;
    float pad;
};
static_assert(sizeof(SharedPath) % 8 == 4, "odd word stride");

// Stack entry type of a megakernel variant: LEAN kernels keep the child
// reference alone (4 bytes).
template <bool LEAN>
using MegaStackEntry = std::conditional_t<LEAN, unsigned, uint2>;

// INL: 0 = both queries call the shared out-of-line traversal, 1 = both are
// inlined, 2 = the closest-hit query is inlined and the shadow query calls the
// out-of-line copy (a smaller kernel than 1, no register saves around the
// per-bounce call). LEAN: the path's state between bounces lives in shared
// memory rather than registers and the stack entries are 4 bytes, so fewer
// registers carry state across the traversal and more blocks fit an SM.
template <int STACK, int EST, bool COUNT = false, int MINB = kMegaBlocksPerSm, int ACC = kAccumulateFp64,
          int INL = 0, bool LEAN = false>
__global__ void __launch_bounds__(kBlock, MINB) megakernel(const DevScene scene, const DevCamera camera,
                                                          const RenderArgs args, PixelAccum* accum,
                                                          unsigned int* error_flag,
                                                          unsigned long long* totals = nullptr)
{
    using Entry = MegaStackEntry<LEAN>;
    extern __shared__ uint2 stack_memory[];
    Entry* const stack = reinterpret_cast<Entry*>(stack_memory);
    TraversalCounts counts{0, 0, 0, 0, 0, 0};
    const TraceContext<INL != 0, COUNT, INL == 1, Entry> ctx{stack + threadIdx.x, kBlock, STACK, error_flag,
                                                             COUNT ? &counts : nullptr};
    int x, y, slot;
    if (args.pixels != nullptr) {
        slot = blockIdx.x * kBlock + threadIdx.x;
        if (slot >= args.pixel_count) {
            return;
        }
        x = args.pixels[slot].x;
        y = args.pixels[slot].y;
    } else {
        const int tile_w = args.tile_width > 0 ? args.tile_width : kTileW;
        const int tile_h = kBlock / tile_w;
        const int tiles_x = (args.width + tile_w - 1) / tile_w;
        x = (blockIdx.x % tiles_x) * tile_w + static_cast<int>(threadIdx.x) % tile_w;
        y = (blockIdx.x / tiles_x) * tile_h + static_cast<int>(threadIdx.x) / tile_w;
        if (x >= args.width || y >= args.height) {
            return;
        }
        slot = y * args.width + x;
    }
    Pcg32 g = pixelGenerator(args.seed, static_cast<std::uint32_t>(x), static_cast<std::uint32_t>(y),
                             static_cast<std::uint32_t>(args.width));
    const int n = args.samples_per_axis;
    const float inv_n = 1.0f / static_cast<float>(n);
    const float width = static_cast<float>(args.width);
    const float height = static_cast<float>(args.height);
    PixelSums<ACC> sums;
    sums.reset();
    // Sums of squared samples (for two-sample tests) go straight to memory, one
    // read-modify-write per sample, only when asked for: no registers carry them
    // through the traversal calls of an ordinary render.
    double* const squares = args.sum_squares != nullptr ? args.sum_squares + 3 * slot : nullptr;
    // One bounce per iteration: a lane whose path ends starts the pixel's next
    // sample at once (drawing its jitter next from the same stream, as the
    // reference does), so a warp waits for the longest pixel, not the longest
    // path of every sample.
    const int total = n * n;
    int sample = 0;
    PathState local_path;
    PathState* path_ptr = &local_path;
    if constexpr (LEAN) {
        __shared__ SharedPath shared_paths[kBlock];
        path_ptr = &shared_paths[threadIdx.x].p;
    }
    PathState& path = *path_ptr;
    startSample(camera, path, g, x, y, 0, n, inv_n, width, height);
    for (;;) {
        if (estimatorBounce<EST>(scene, ctx, path, g, args)) {
            continue;
        }
        const float3 L = path.result;
        sums.add(L);
        if (squares != nullptr) {
            squares[0] += static_cast<double>(L.x) * L.x;
            squares[1] += static_cast<double>(L.y) * L.y;
            squares[2] += static_cast<double>(L.z) * L.z;
        }
        if (++sample == total) {
            break;
        }
        startSample(camera, path, g, x, y, sample, n, inv_n, width, height);
    }
    PixelAccum& a = accum[slot];
    const double3 total_sum = sums.total();
    a.r += total_sum.x;
    a.g += total_sum.y;
    a.b += total_sum.z;
    a.count += static_cast<long long>(n) * n;
    if constexpr (COUNT) {
        atomicAdd(totals + 0, counts.boxes);
        atomicAdd(totals + 1, counts.triangles);
        atomicAdd(totals + 2, counts.spheres);
        atomicAdd(totals + 3, counts.instances);
        atomicAdd(totals + 4, counts.rays);
        atomicAdd(totals + 5, counts.reference_boxes);
    }
}

// Closest-hit queries of given rays, counting their traversal work into
// totals[0..5] (as the counting megakernel does). Not used for timing.
template <int STACK>
__global__ void __launch_bounds__(kBlock) traceCountKernel(const DevScene scene, const float* rays, int count,
                                                           float t_min, float t_max, unsigned int* error_flag,
                                                           unsigned long long* totals)
{
    extern __shared__ uint2 stack[];
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= count) {
        return;
    }
    TraversalCounts counts{0, 0, 0, 0, 0, 0};
    const float3 o = mk(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
    const float3 d = mk(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
    TraceHit hit;
    float tmax = t_max;
    static_cast<void>(traceScene<false, false, true>(scene, o, d, t_min, tmax, SkipRule::none(), hit,
                                                     stack + threadIdx.x, kBlock, STACK, error_flag, &counts));
    atomicAdd(totals + 0, counts.boxes);
    atomicAdd(totals + 1, counts.triangles);
    atomicAdd(totals + 2, counts.spheres);
    atomicAdd(totals + 3, counts.instances);
    atomicAdd(totals + 4, counts.rays);
    atomicAdd(totals + 5, counts.reference_boxes);
}

template <int STACK>
__global__ void __launch_bounds__(kBlock) traceKernel(const DevScene scene, const float* rays, int count, float t_min,
                                                      float t_max, TraceOutputs out, unsigned int* error_flag)
{
    extern __shared__ uint2 stack[];
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= count) {
        return;
    }
    const float3 o = mk(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
    const float3 d = mk(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
    TraceHit hit;
    float tmax = t_max;
    const bool found = traceScene<false>(scene, o, d, t_min, tmax, SkipRule::none(), hit, stack + threadIdx.x, kBlock,
                                         STACK, error_flag);
    out.hit[i] = found ? 1 : 0;
    if (!found) {
        return;
    }
    Surface sf;
    resolveHit(scene, o, d, hit, sf);
    out.t[i] = static_cast<float>(refinedDistance(scene, o, d, hit));
    out.object[i] = static_cast<int>(sf.object_id);
    out.triangle[i] = -1;
    const DevObject obj = scene.objects[hit.obj_pos];
    if (obj.kind == kObjInstance) {
        out.triangle[i] = static_cast<int>(__float_as_uint(scene.triangles[hit.tri_pos].v0w));
    }
    if (out.point != nullptr) {
        out.point[3 * i] = sf.p.x;
        out.point[3 * i + 1] = sf.p.y;
        out.point[3 * i + 2] = sf.p.z;
        out.normal[3 * i] = sf.n.x;
        out.normal[3 * i + 1] = sf.n.y;
        out.normal[3 * i + 2] = sf.n.z;
        out.shading_normal[3 * i] = sf.ns.x;
        out.shading_normal[3 * i + 1] = sf.ns.y;
        out.shading_normal[3 * i + 2] = sf.ns.z;
        out.front[i] = sf.front ? 1 : 0;
    }
}

template <int STACK>
__global__ void __launch_bounds__(kBlock) occludedKernel(const DevScene scene, const float* rays, const float* t_max,
                                                         int count, int* occluded_out, unsigned int* error_flag)
{
    extern __shared__ uint2 stack[];
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i >= count) {
        return;
    }
    const float3 o = mk(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
    const float3 d = mk(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
    TraceHit hit;
    float tmax = t_max[i];
    occluded_out[i] = traceScene<true>(scene, o, d, 0.0f, tmax, SkipRule::none(), hit, stack + threadIdx.x, kBlock,
                                       STACK, error_flag)
                          ? 1
                          : 0;
}

constexpr std::size_t stackBytes(int stack, std::size_t entry_bytes = sizeof(uint2))
{
    return static_cast<std::size_t>(stack) * kBlock * entry_bytes;
}

int megaBlocks(const RenderArgs& args)
{
    if (args.pixels != nullptr) {
        return (args.pixel_count + kBlock - 1) / kBlock;
    }
    const int tile_w = args.tile_width > 0 ? args.tile_width : kTileW;
    const int tile_h = kBlock / tile_w;
    return ((args.width + tile_w - 1) / tile_w) * ((args.height + tile_h - 1) / tile_h);
}

// Launches `kernel` over `blocks` blocks with a STACK-entry shared-memory stack
// of ENTRY-byte entries.
template <int STACK, int ENTRY = static_cast<int>(sizeof(uint2)), typename Kernel, typename... Args>
cudaError_t launchStacked(Kernel kernel, int blocks, cudaStream_t stream, Args... args)
{
    if (blocks == 0) {
        return cudaSuccess;
    }
    const cudaError_t e = allowStackMemory(kernel, STACK, ENTRY);
    if (e != cudaSuccess) {
        return e;
    }
    kernel<<<blocks, kBlock, stackBytes(STACK, ENTRY), stream>>>(args...);
    return cudaGetLastError();
}

} // namespace

cudaError_t launchMegakernelCounting(const DevScene& scene, const DevCamera& camera, const RenderArgs& args,
                                     PixelAccum* accum, unsigned int* error_flag, int stack_capacity,
                                     unsigned long long* totals, cudaStream_t stream)
{
    return withStack(stack_capacity, [&](auto size) {
        constexpr int S = decltype(size)::value;
        return launchStacked<S>(megakernel<S, kEstimatorPath, true>, megaBlocks(args), stream, scene, camera, args,
                                accum, error_flag, totals);
    });
}

int stackCapacityFor(std::uint32_t stack_need)
{
    if (stack_need <= 32u) {
        return 32;
    }
    if (stack_need <= 48u) {
        return 48;
    }
    if (stack_need <= 64u) {
        return 64;
    }
    return 0;
}

// Path-estimator megakernel of the shape `args` names: blocks_per_sm 3 (state
// in registers, 8-byte stack entries) or 4 (lean: state in shared memory,
// 4-byte stack entries), and how its traversal is placed (inline_traversal).
template <int S, int ACC>
cudaError_t launchPathMegakernel(const DevScene& scene, const DevCamera& camera, const RenderArgs& args,
                                 PixelAccum* accum, unsigned int* error_flag, cudaStream_t stream)
{
    unsigned long long* no_totals = nullptr;
    const int blocks = megaBlocks(args);
    if (args.blocks_per_sm == 4) {
        constexpr int kEntry = static_cast<int>(sizeof(unsigned));
        if (args.inline_traversal == 1) {
            return launchStacked<S, kEntry>(megakernel<S, kEstimatorPath, false, 4, ACC, 1, true>, blocks, stream,
                                            scene, camera, args, accum, error_flag, no_totals);
        }
        return launchStacked<S, kEntry>(megakernel<S, kEstimatorPath, false, 4, ACC, 0, true>, blocks, stream, scene,
                                        camera, args, accum, error_flag, no_totals);
    }
    if (args.inline_traversal == 1) {
        return launchStacked<S>(megakernel<S, kEstimatorPath, false, kMegaBlocksPerSm, ACC, 1>, blocks, stream, scene,
                                camera, args, accum, error_flag, no_totals);
    }
    if (args.inline_traversal == 2) {
        return launchStacked<S>(megakernel<S, kEstimatorPath, false, kMegaBlocksPerSm, ACC, 2>, blocks, stream, scene,
                                camera, args, accum, error_flag, no_totals);
    }
    return launchStacked<S>(megakernel<S, kEstimatorPath, false, kMegaBlocksPerSm, ACC>, blocks, stream, scene, camera,
                            args, accum, error_flag, no_totals);
}

cudaError_t launchMegakernel(const DevScene& scene, const DevCamera& camera, const RenderArgs& args, PixelAccum* accum,
                             unsigned int* error_flag, int stack_capacity, cudaStream_t stream)
{
    return withStack(stack_capacity, [&](auto size) {
        constexpr int S = decltype(size)::value;
        unsigned long long* no_totals = nullptr;
        switch (args.estimator) {
        case kEstimatorScatterOnly:
            return launchStacked<S>(megakernel<S, kEstimatorScatterOnly>, megaBlocks(args), stream, scene, camera,
                                    args, accum, error_flag, no_totals);
        case kEstimatorNormals:
            return launchStacked<S>(megakernel<S, kEstimatorNormals>, megaBlocks(args), stream, scene, camera, args,
                                    accum, error_flag, no_totals);
        default:
            if (args.accumulation == kAccumulateKahan) {
                return launchPathMegakernel<S, kAccumulateKahan>(scene, camera, args, accum, error_flag, stream);
            }
            return launchPathMegakernel<S, kAccumulateFp64>(scene, camera, args, accum, error_flag, stream);
        }
    });
}

cudaError_t launchTrace(const DevScene& scene, const float* rays, int count, float t_min, float t_max,
                        const TraceOutputs& out, unsigned int* error_flag, int stack_capacity, cudaStream_t stream)
{
    return withStack(stack_capacity, [&](auto size) {
        constexpr int S = decltype(size)::value;
        return launchStacked<S>(traceKernel<S>, (count + kBlock - 1) / kBlock, stream, scene, rays, count, t_min,
                                t_max, out, error_flag);
    });
}

cudaError_t launchTraceCounting(const DevScene& scene, const float* rays, int count, float t_min, float t_max,
                                unsigned int* error_flag, int stack_capacity, unsigned long long* totals,
                                cudaStream_t stream)
{
    return withStack(stack_capacity, [&](auto size) {
        constexpr int S = decltype(size)::value;
        return launchStacked<S>(traceCountKernel<S>, (count + kBlock - 1) / kBlock, stream, scene, rays, count, t_min,
                                t_max, error_flag, totals);
    });
}

cudaError_t launchOccluded(const DevScene& scene, const float* rays, const float* t_max, int count, int* occluded_out,
                           unsigned int* error_flag, int stack_capacity, cudaStream_t stream)
{
    return withStack(stack_capacity, [&](auto size) {
        constexpr int S = decltype(size)::value;
        return launchStacked<S>(occludedKernel<S>, (count + kBlock - 1) / kBlock, stream, scene, rays, t_max, count,
                                occluded_out, error_flag);
    });
}

} // namespace albedo_b200
