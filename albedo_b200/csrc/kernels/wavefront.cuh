// Wavefront renderer layout: jobs, path slots and queues shared by the kernels
// in wavefront.cu and the host engine that drives them.
#pragma once

#include "launch.hpp"

#include <cstdint>

namespace albedo_b200 {

// One render job of a batch: its scene, camera, accumulators and parameters, and
// where its pixels sit in the batch's work-item range.
struct WfJob {
    DevScene scene;
    DevCamera camera;
    PixelAccum* accum;
    int width;
    int height;
    int samples_per_axis;
    int max_depth;
    int roulette_start;
    int pad;
    unsigned long long seed;
    long long item_begin;   // first work item (pixel) of this job
    long long item_end;     // one past its last
    float grid[4];          // ray-binning cells of the scene: x0, y0, z0, cells per unit (coherenceGrid)
};

// Ray binning before each extend: 2^kBinBits bins of (job, direction octant,
// origin cell) keys.
constexpr int kBinBits = 14;
constexpr int kBinCount = 1 << kBinBits;

// Path slots, one record per field group so a gather of one slot reads whole
// 16-byte records. A slot owns one pixel for all of that pixel's samples, so its
// PCG32 stream advances exactly as the reference's per-pixel generator does.
struct WfSlots {
    float4* ray_o;      // origin xyz, arrival pdf
    float4* ray_d;      // direction xyz, arrival-specular flag (0 or 1)
    float4* throughput; // xyz, unused
    float4* result;     // radiance gathered so far xyz, unused
    float4* arrival;    // previous scattering point xyz, unused
    uint4* skip;        // object position, triangle position, sphere mode, unused
    ulonglong2* rng;    // PCG32 state, increment
    int4* where;        // job (-1: idle), pixel index in the job, sample index, depth
    float4* hit;        // t, object position bits, triangle position bits, b0
    float2* hit_b;      // b1, b2
    float4* shadow_o;   // shadow ray origin xyz, range end
    float4* shadow_d;   // shadow ray direction xyz, area-light object position bits
    uint4* shadow_skip; // object position, triangle position, sphere mode, unused
    float4* shadow_c;   // contribution if unoccluded xyz, unused
};

enum WfQueueId : int {
    kQExtend0 = 0,
    kQExtend1 = 1,
    kQRegen0 = 2,
    kQRegen1 = 3,
    kQDiffuse = 4,
    kQConductor = 5,
    kQDielectric = 6,
    kQMix = 7,
    kQShadow = 8,
    kQParked = 9, // slots that found no pixel; an append puts them back to work
    kQueueCount = 10
};

struct WfControl {
    int count[kQueueCount];
    int parity;                   // current extend/regen buffers: kQExtend0 + parity, kQRegen0 + parity
    unsigned long long next_item; // next pixel work item to hand out
    unsigned long long completed; // pixels whose last sample has been accumulated
    unsigned long long iterations;
    // The batch so far: work items (pixels) and jobs in the job table. A server
    // appends jobs between iterations, growing both.
    unsigned long long total_items;
    int job_count;
    int pad;
    // Queue entries handed out so far in this iteration by the extend and shadow
    // kernels (which take rays in warp batches as lanes finish).
    int fetch_extend;
    int fetch_shadow;
    unsigned long long rays_traced; // closest-hit plus shadow queries since the batch opened
};

struct WfBuffers {
    WfSlots slots;
    int* queue[kQueueCount]; // each `slot_count` entries
    WfControl* control;
    unsigned long long* job_done; // per job: pixels whose last sample has been accumulated
    int slot_count;
    // Ray binning (null where an engine has none): per extend-queue entry its
    // bin key, the queue reordered by bin, bin counts (zero between iterations)
    // and bin cursors.
    unsigned int* bin_key;
    int* binned;
    unsigned int* bin_count;
    unsigned int* bin_cursor;
};

struct WfLaunch {
    int blocks;       // grid of the queue kernels (a multiple of the SM count)
    int threads;      // threads per block
    int stack;        // traversal stack entries per thread
    int trace_blocks; // grid of the persistent traversal kernels (blocks resident at once), or 0 for `blocks`
    int fetch_batch;  // queue entries a traversal warp claims at once (0: 32)
    int trace_loop;   // traversal turn shape of the persistent kernels (TraceLoop)
    int ray_sort;     // 1: the extend queue is binned by ray coherence before the extend kernel; 2: the shadow
                      // queue too
};

// Opts the traversal kernels into `stack` entries of dynamic shared memory; call
// before capturing iterations into a graph.
cudaError_t wfPrepare(int stack);
// Puts every slot in the regeneration queue with no job, clears the counters and
// the first `job_count` per-job counters, and sets the batch's size.
cudaError_t wfReset(const WfBuffers& b, unsigned long long total_items, int job_count, cudaStream_t stream);
// The allocation-free variant (noalloc.cu): one job, one path slot per pixel, all
// scratch in a static device array; at most noAllocMaxPixels() pixels.
int noAllocMaxPixels();
cudaError_t renderNoAlloc(const WfJob& job, int stack, int blocks, unsigned int* error_flag, cudaStream_t stream);
// Enqueues one iteration (regenerate, extend, shade x 4, shadow, advance). The
// batch's size is read from the control block, so iterations captured in a graph
// keep serving jobs appended later.
// Blocks per SM of the persistent traversal kernels that fit at once with
// `stack` entries per thread (after wfPrepare).
cudaError_t wfTraceBlocksPerSm(int stack, int* out);
// Probe for parity tests: closest-hit (any = false) or any-hit queries of given
// rays, traced one query per thread (mode 0) or the wavefront's way (mode 1:
// nodes then leaf per turn, 2: one step per turn; `counter` is an int zeroed
// before the launch), writing raw hits.
cudaError_t launchTraceModes(const DevScene& scene, const float* rays, int count, float t_min, float t_max, bool any,
                             int mode, int stack, int* counter, unsigned int* error_flag, int* out_hit,
                             unsigned int* out_t, unsigned int* out_obj, unsigned int* out_tri, cudaStream_t stream);
// Side streams and events for running the per-class shade kernels of an
// iteration as parallel branches (they touch disjoint slots and push through
// atomics); without them the kernels run one after another.
struct WfSide {
    cudaStream_t stream[3];
    cudaEvent_t fork;
    cudaEvent_t join[3];
};
cudaError_t wfIteration(const WfJob* jobs, const WfBuffers& b, const WfLaunch& launch, unsigned int* error_flag,
                        cudaStream_t stream, const WfSide* side = nullptr);
// Appends jobs [first, first + count) of the (already uploaded) job table to a
// running batch: zeroes their completion counters and grows the batch's size.
cudaError_t wfAppend(const WfBuffers& b, int first, int count, unsigned long long new_total_items,
                     cudaStream_t stream);

} // namespace albedo_b200
