// The wavefront renderer: path slots advanced one bounce per iteration by
// stage kernels over compacted queues.
//
//   regenerate   finished paths are added to their pixel (PixelBuffer::addSample);
//                the slot starts its pixel's next stratified sample, or claims the
//                batch's next pixel (render/render_image.cpp:27-44)
//   extend       closest hit of every queued ray; misses add the MIS-weighted sky
//   shade x 4    one kernel per material class (diffuse / conductor / dielectric /
//                mix): emission, next-event estimation (a shadow-ray candidate),
//                BSDF sampling and roulette (estimator/path_estimator.cpp:153-185)
//   shadow       any-hit test of the candidates; unoccluded ones are added
//   advance      swaps the double-buffered extend / regenerate queues
//
// Every push is warp-aggregated: one ballot, one atomicAdd per warp, and each
// lane writes at the prefix count of the lanes below it. Random numbers are drawn
// in the same order as the megakernel (jitter, then per bounce 3 NEE, 3 BSDF,
// 1 roulette), so each pixel's stream matches the reference's.
#include "estimator.cuh"
#include "fetch.cuh"
#include "wavefront.cuh"

namespace albedo_b200 {

namespace {

ALB_DEV void pushSlot(int* queue, int* counter, int slot, bool pred)
{
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, pred);
    if (mask == 0u) {
        return;
    }
    const int lane = static_cast<int>(threadIdx.x & 31u);
    const int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) {
        base = atomicAdd(counter, __popc(mask));
    }
    base = __shfl_sync(active, base, leader);
    if (pred) {
        queue[base + __popc(mask & ((1u << lane) - 1u))] = slot;
    }
}

// Hands out work items with one atomicAdd per warp.
ALB_DEV unsigned long long claimItem(unsigned long long* next, bool want)
{
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, want);
    if (mask == 0u) {
        return ~0ull;
    }
    const int lane = static_cast<int>(threadIdx.x & 31u);
    const int leader = __ffs(mask) - 1;
    unsigned long long base = 0;
    if (lane == leader) {
        base = atomicAdd(next, static_cast<unsigned long long>(__popc(mask)));
    }
    base = __shfl_sync(active, base, leader);
    return want ? base + static_cast<unsigned long long>(__popc(mask & ((1u << lane) - 1u))) : ~0ull;
}

// Resident blocks per SM the traversal kernels' register budget is sized for:
// 5 (96 registers a thread, no spills). With 4-byte stack entries five blocks'
// stacks fit in shared memory; 5 measured 6-10% faster than 4 on the trefoil,
// icosphere and 64-job workloads.
#ifndef ALBEDO_TRACE_BLOCKS_PER_SM
#define ALBEDO_TRACE_BLOCKS_PER_SM 5
#endif
constexpr int kTraceBlocksPerSm = ALBEDO_TRACE_BLOCKS_PER_SM;

ALB_DEV int findJob(const WfJob* jobs, int job_count, long long item)
{
    int lo = 0;
    int hi = job_count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (jobs[mid].item_begin <= item) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

ALB_DEV void storeRay(const WfSlots& sl, int s, const PathState& p)
{
    sl.ray_o[s] = make_float4(p.o.x, p.o.y, p.o.z, p.arrival_pdf);
    sl.ray_d[s] = make_float4(p.d.x, p.d.y, p.d.z, p.arrival_specular ? 1.0f : 0.0f);
    sl.throughput[s] = make_float4(p.throughput.x, p.throughput.y, p.throughput.z, 0.0f);
    sl.result[s] = make_float4(p.result.x, p.result.y, p.result.z, 0.0f);
    sl.arrival[s] = make_float4(p.arrival_origin.x, p.arrival_origin.y, p.arrival_origin.z, 0.0f);
    sl.skip[s] = make_uint4(p.skip.object_pos, p.skip.tri_pos, static_cast<unsigned>(p.skip.sphere_mode), 0u);
}

ALB_DEV void loadPath(const WfSlots& sl, int s, int depth, PathState& p)
{
    const float4 o = sl.ray_o[s];
    const float4 d = sl.ray_d[s];
    const float4 t = sl.throughput[s];
    const float4 r = sl.result[s];
    const float4 a = sl.arrival[s];
    const uint4 k = sl.skip[s];
    p.o = mk(o.x, o.y, o.z);
    p.arrival_pdf = o.w;
    p.d = mk(d.x, d.y, d.z);
    p.arrival_specular = d.w != 0.0f;
    p.throughput = mk(t.x, t.y, t.z);
    p.result = mk(r.x, r.y, r.z);
    p.arrival_origin = mk(a.x, a.y, a.z);
    p.skip = {k.x, k.y, static_cast<int>(k.z), kNoPrim};
    p.depth = depth;
}

__global__ void __launch_bounds__(128) regenKernel(const WfJob* __restrict__ jobs, WfBuffers b)
{
    WfControl* ctl = b.control;
    const int parity = ctl->parity;
    const unsigned long long total_items = ctl->total_items;
    const int job_count = ctl->job_count;
    const int in = kQRegen0 + parity;
    const int out = kQExtend0 + parity;
    const int count = ctl->count[in];
    const WfSlots& sl = b.slots;
    const int stride = static_cast<int>(gridDim.x * blockDim.x);
    for (int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x); i < count; i += stride) {
        const int s = b.queue[in][i];
        int4 w = sl.where[s];
        bool start = false;
        Pcg32 g;
        if (w.x >= 0) {
            const WfJob& job = jobs[w.x];
            const float4 r = sl.result[s];
            PixelAccum& acc = job.accum[w.y];
            acc.r += r.x;
            acc.g += r.y;
            acc.b += r.z;
            acc.count += 1;
            w.z += 1;
            if (w.z < job.samples_per_axis * job.samples_per_axis) {
                start = true;
                const ulonglong2 st = sl.rng[s];
                g = {st.x, st.y};
            } else {
                atomicAdd(&ctl->completed, 1ull);
                atomicAdd(&b.job_done[w.x], 1ull);
                w.x = -1;
            }
        }
        const unsigned long long item = claimItem(&ctl->next_item, w.x < 0);
        if (w.x < 0 && item < total_items) {
            const int j = findJob(jobs, job_count, static_cast<long long>(item));
            const WfJob& job = jobs[j];
            const int pixel = static_cast<int>(static_cast<long long>(item) - job.item_begin);
            w = make_int4(j, pixel, 0, 0);
            g = pixelGenerator(job.seed, static_cast<std::uint32_t>(pixel % job.width),
                               static_cast<std::uint32_t>(pixel / job.width), static_cast<std::uint32_t>(job.width));
            start = true;
        }
        if (start) {
            const WfJob& job = jobs[w.x];
            const int n = job.samples_per_axis;
            PathState p;
            startSample(job.camera, p, g, w.y % job.width, w.y / job.width, w.z, n, 1.0f / static_cast<float>(n),
                        static_cast<float>(job.width), static_cast<float>(job.height));
            storeRay(sl, s, p);
            sl.rng[s] = make_ulonglong2(g.state, g.inc);
            w.w = 0;
        }
        sl.where[s] = w;
        pushSlot(b.queue[out], &ctl->count[out], s, start);
        pushSlot(b.queue[kQParked], &ctl->count[kQParked], s, !start);
    }
}

// Ray binning. Between regeneration and extension the extend queue is
// reordered so that a traversal warp's rays start in the same region of the
// scene and point into the same octant, and so visit similar nodes in the same
// order: a counting sort by a 14-bit key of (job, direction octant, origin cell
// of an 8 x 8 x 8 grid over the scene's core, in Morton order). Each query's
// result does not depend on when it is traced, so images are the same with or
// without binning, and in any order within a bin.
ALB_DEV unsigned int rayBinKey(const WfJob& job, int job_index, float4 o, float4 d)
{
    const auto cell = [&](float v, float lo) {
        const int c = __float2int_rd((v - lo) * job.grid[3]);
        return static_cast<unsigned int>(min(max(c, 0), 7));
    };
    const unsigned int cx = cell(o.x, job.grid[0]);
    const unsigned int cy = cell(o.y, job.grid[1]);
    const unsigned int cz = cell(o.z, job.grid[2]);
    unsigned int morton = 0u;
    for (int bit = 2; bit >= 0; --bit) {
        morton = (morton << 3) | (((cx >> bit) & 1u) << 2) | (((cy >> bit) & 1u) << 1) | ((cz >> bit) & 1u);
    }
    const unsigned int octant = (d.x < 0.0f ? 4u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 1u : 0u);
    return (static_cast<unsigned int>(job_index & 3) << 12) | (octant << 9) | morton;
}

// Adds `amount` to counter[key] once per group of lanes with the same key and
// returns the counter's old value plus the lane's rank in its group.
ALB_DEV unsigned int groupedAdd(unsigned int* counter, unsigned int key)
{
    const unsigned int active = __activemask();
    const unsigned int peers = __match_any_sync(active, key);
    const int lane = static_cast<int>(threadIdx.x & 31u);
    const int leader = __ffs(peers) - 1;
    unsigned int base = 0u;
    if (lane == leader) {
        base = atomicAdd(counter + key, static_cast<unsigned int>(__popc(peers)));
    }
    base = __shfl_sync(active, base, leader);
    return base + static_cast<unsigned int>(__popc(peers & ((1u << lane) - 1u)));
}

// The queue a binning pass reorders: the extend queue of this iteration, or
// the shadow queue (SHADOW), whose rays are the shadow origins and directions.
template <bool SHADOW>
ALB_DEV int binnedQueue(const WfControl* ctl)
{
    return SHADOW ? static_cast<int>(kQShadow) : static_cast<int>(kQExtend0) + ctl->parity;
}

template <bool SHADOW>
__global__ void __launch_bounds__(128) binKeysKernel(const WfJob* __restrict__ jobs, WfBuffers b)
{
    const WfControl* ctl = b.control;
    const int in = binnedQueue<SHADOW>(ctl);
    const int count = ctl->count[in];
    const int stride = static_cast<int>(gridDim.x * blockDim.x);
    for (int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x); i < count; i += stride) {
        const int s = b.queue[in][i];
        const int job = b.slots.where[s].x;
        const float4 o = SHADOW ? b.slots.shadow_o[s] : b.slots.ray_o[s];
        const float4 d = SHADOW ? b.slots.shadow_d[s] : b.slots.ray_d[s];
        const unsigned int key = rayBinKey(jobs[job], job, o, d);
        b.bin_key[i] = key;
        static_cast<void>(groupedAdd(b.bin_count, key));
    }
}

// One block of 1024 threads: exclusive prefix sums of the bin counts into the
// cursors, and the counts back to zero for the next iteration.
__global__ void __launch_bounds__(1024) binScanKernel(WfBuffers b)
{
    constexpr int kPerThread = kBinCount / 1024;
    __shared__ unsigned int warp_total[32];
    const int t = static_cast<int>(threadIdx.x);
    unsigned int local[kPerThread];
    unsigned int sum = 0u;
    for (int k = 0; k < kPerThread; ++k) {
        local[k] = b.bin_count[t * kPerThread + k];
        sum += local[k];
    }
    // Inclusive scan of the threads' sums: within each warp, then over warps.
    const int lane = t & 31;
    const int warp = t >> 5;
    unsigned int inclusive = sum;
    for (int offset = 1; offset < 32; offset <<= 1) {
        const unsigned int up = __shfl_up_sync(0xFFFFFFFFu, inclusive, offset);
        if (lane >= offset) {
            inclusive += up;
        }
    }
    if (lane == 31) {
        warp_total[warp] = inclusive;
    }
    __syncthreads();
    if (warp == 0) {
        unsigned int w = warp_total[lane];
        for (int offset = 1; offset < 32; offset <<= 1) {
            const unsigned int up = __shfl_up_sync(0xFFFFFFFFu, w, offset);
            if (lane >= offset) {
                w += up;
            }
        }
        warp_total[lane] = w;
    }
    __syncthreads();
    unsigned int running = inclusive - sum + (warp > 0 ? warp_total[warp - 1] : 0u);
    for (int k = 0; k < kPerThread; ++k) {
        b.bin_cursor[t * kPerThread + k] = running;
        running += local[k];
        b.bin_count[t * kPerThread + k] = 0u;
    }
}

template <bool SHADOW>
__global__ void __launch_bounds__(128) binScatterKernel(WfBuffers b)
{
    const WfControl* ctl = b.control;
    const int in = binnedQueue<SHADOW>(ctl);
    const int count = ctl->count[in];
    const int stride = static_cast<int>(gridDim.x * blockDim.x);
    for (int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x); i < count; i += stride) {
        const unsigned int position = groupedAdd(b.bin_cursor, b.bin_key[i]);
        b.binned[position] = b.queue[in][i];
    }
}

// Closest hit of every ray in the extend queue. The kernel is persistent: a lane
// whose query ends files the result and takes the next queued ray, so a warp is
// not held by its slowest ray. Each query runs the same traversal steps, in the
// same order, as a query traced alone.
template <int STACK, int LOOP>
__global__ void __launch_bounds__(128, kTraceBlocksPerSm) extendKernel(const WfJob* __restrict__ jobs, WfBuffers b,
                                                                        unsigned int* error_flag, int fetch_batch,
                                                                        bool binned)
{
    extern __shared__ unsigned ref_stack[];
    WfControl* ctl = b.control;
    const int parity = ctl->parity;
    const int in = kQExtend0 + parity;
    const int* const order = binned ? b.binned : b.queue[in];
    const int ended = kQRegen0 + (parity ^ 1);
    const int count = ctl->count[in];
    const WfSlots& sl = b.slots;
    unsigned* const lane_stack = ref_stack + threadIdx.x;
    const int stride = static_cast<int>(blockDim.x);
    WarpFetch fetch{0, 0, fetch_batch, false};
    TraceState q;
    SkipRule skip = SkipRule::none();
    const DevScene* scene = nullptr;
    int s = -1;
    bool active = false;
    for (;;) {
        const int i = fetch.take(&ctl->fetch_extend, count, !active);
        bool finished = false;
        if (i >= 0) {
            s = order[i];
            scene = &jobs[sl.where[s].x].scene;
            const float4 o = sl.ray_o[s];
            const float4 d = sl.ray_d[s];
            const uint4 k = sl.skip[s];
            skip = {k.x, k.y, static_cast<int>(k.z), kNoPrim};
            active = traceBegin(*scene, q, mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), 0.0f, INFINITY);
            finished = !active;
        }
        if (__ballot_sync(0xFFFFFFFFu, active || finished) == 0u) {
            break;
        }
        if (active && !traceAdvance<LOOP>(*scene, q, skip, lane_stack, stride, STACK, error_flag, nullptr, false)) {
            active = false;
            finished = true;
        }
        if (finished) {
            int cls = -1;
            if (q.found) {
                sl.hit[s] = make_float4(q.hit.t, __uint_as_float(q.hit.obj_pos), __uint_as_float(q.hit.tri_pos),
                                        q.hit.b0);
                sl.hit_b[s] = make_float2(q.hit.b1, q.hit.b2);
                cls = materialClass(*scene, q.hit.obj_pos);
            } else {
                const float4 o = sl.ray_o[s];
                const float4 d = sl.ray_d[s];
                PathState p;
                p.d = mk(d.x, d.y, d.z);
                p.arrival_pdf = o.w;
                p.arrival_specular = d.w != 0.0f;
                const float4 t = sl.throughput[s];
                const float3 e = weightedSky(*scene, p);
                float4 r = sl.result[s];
                r.x += t.x * e.x;
                r.y += t.y * e.y;
                r.z += t.z * e.z;
                sl.result[s] = r;
            }
            pushSlot(b.queue[ended], &ctl->count[ended], s, !q.found);
            pushSlot(b.queue[kQDiffuse], &ctl->count[kQDiffuse], s, cls == kClassDiffuse);
            pushSlot(b.queue[kQConductor], &ctl->count[kQConductor], s, cls == kClassConductor);
            pushSlot(b.queue[kQDielectric], &ctl->count[kQDielectric], s, cls == kClassDielectric);
            pushSlot(b.queue[kQMix], &ctl->count[kQMix], s, cls == kClassMix);
        }
    }
}

template <int CLASS>
__global__ void __launch_bounds__(128) shadeKernel(const WfJob* __restrict__ jobs, WfBuffers b)
{
    WfControl* ctl = b.control;
    const int parity = ctl->parity;
    const int in = kQDiffuse + CLASS;
    const int next = kQExtend0 + (parity ^ 1);
    const int ended = kQRegen0 + (parity ^ 1);
    const int count = ctl->count[in];
    const WfSlots& sl = b.slots;
    const int stride = static_cast<int>(gridDim.x * blockDim.x);
    for (int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x); i < count; i += stride) {
        const int s = b.queue[in][i];
        int4 w = sl.where[s];
        const WfJob& job = jobs[w.x];
        const DevScene& scene = job.scene;
        PathState p;
        loadPath(sl, s, w.w, p);
        const float4 h = sl.hit[s];
        const float2 hb = sl.hit_b[s];
        const TraceHit hit{h.x, __float_as_uint(h.y), __float_as_uint(h.z), h.w, hb.x, hb.y};
        const ulonglong2 st = sl.rng[s];
        Pcg32 g{st.x, st.y};
        Surface sf;
        resolveHit(scene, p.o, p.d, hit, sf);
        p.result = p.result + p.throughput * weightedEmission(scene, p, sf);
        bool alive = false;
        bool shadow = false;
        if (p.depth < job.max_depth) {
            const Scattering sc = scatteringAtClass<CLASS>(scene, sf);
            const float3 wo = -p.d;
            const NeeCandidate nc = directLightCandidate(scene, sf, sc, wo, g);
            if (nc.valid) {
                const float3 c = p.throughput * nc.contribution;
                if (nc.needs_test) {
                    shadow = true;
                    sl.shadow_o[s] = make_float4(nc.origin.x, nc.origin.y, nc.origin.z, nc.range_max);
                    sl.shadow_d[s] = make_float4(nc.dir.x, nc.dir.y, nc.dir.z, __uint_as_float(nc.skip.light_object_pos));
                    sl.shadow_skip[s] = make_uint4(nc.skip.object_pos, nc.skip.tri_pos,
                                                   static_cast<unsigned>(nc.skip.sphere_mode), 0u);
                    sl.shadow_c[s] = make_float4(c.x, c.y, c.z, 0.0f);
                } else {
                    p.result = p.result + c;
                }
            }
            const float u_choice = g.next1D();
            const float ux = g.next1D();
            const float uy = g.next1D();
            ScatterSample smp;
            if (sc.sample(wo, u_choice, ux, uy, smp)) {
                p.throughput = p.throughput * smp.weight;
                if (!isBlack(p.throughput)) {
                    alive = true;
                    if (p.depth >= job.roulette_start) {
                        const float survival =
                            fminf(0.95f, fmaxf(p.throughput.x, fmaxf(p.throughput.y, p.throughput.z)));
                        if (g.next1D() >= survival) {
                            alive = false;
                        } else {
                            p.throughput = p.throughput / survival;
                        }
                    }
                    if (alive) {
                        p.arrival_origin = sf.p;
                        p.arrival_pdf = smp.pdf;
                        p.arrival_specular = smp.specular;
                        rayLeaving(sf, smp.dir, p.o, p.skip);
                        p.d = smp.dir;
                        w.w = p.depth + 1;
                    }
                }
            }
        }
        storeRay(sl, s, p);
        sl.rng[s] = make_ulonglong2(g.state, g.inc);
        sl.where[s] = w;
        pushSlot(b.queue[kQShadow], &ctl->count[kQShadow], s, shadow);
        pushSlot(b.queue[next], &ctl->count[next], s, alive);
        pushSlot(b.queue[ended], &ctl->count[ended], s, !alive);
    }
}

// Any-hit test of every shadow candidate; unoccluded candidates are added to
// their path. Persistent, like extendKernel.
template <int STACK, int LOOP>
__global__ void __launch_bounds__(128, kTraceBlocksPerSm) shadowKernel(const WfJob* __restrict__ jobs, WfBuffers b,
                                                                        unsigned int* error_flag, int fetch_batch,
                                                                        bool binned)
{
    extern __shared__ unsigned ref_stack[];
    WfControl* ctl = b.control;
    const int count = ctl->count[kQShadow];
    const int* const order = binned ? b.binned : b.queue[kQShadow];
    const WfSlots& sl = b.slots;
    unsigned* const lane_stack = ref_stack + threadIdx.x;
    const int stride = static_cast<int>(blockDim.x);
    WarpFetch fetch{0, 0, fetch_batch, false};
    TraceState q;
    SkipRule skip = SkipRule::none();
    const DevScene* scene = nullptr;
    int s = -1;
    bool active = false;
    for (;;) {
        const int i = fetch.take(&ctl->fetch_shadow, count, !active);
        bool finished = false;
        if (i >= 0) {
            s = order[i];
            scene = &jobs[sl.where[s].x].scene;
            const float4 o = sl.shadow_o[s];
            const float4 d = sl.shadow_d[s];
            const uint4 k = sl.shadow_skip[s];
            skip = {k.x, k.y, static_cast<int>(k.z), __float_as_uint(d.w)};
            active = traceBegin(*scene, q, mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), 0.0f, o.w);
            finished = !active;
        }
        if (__ballot_sync(0xFFFFFFFFu, active || finished) == 0u) {
            break;
        }
        if (active && !traceAdvance<LOOP>(*scene, q, skip, lane_stack, stride, STACK, error_flag, nullptr, true)) {
            active = false;
            finished = true;
        }
        if (finished && !q.found) {
            const float4 c = sl.shadow_c[s];
            float4 r = sl.result[s];
            r.x += c.x;
            r.y += c.y;
            r.z += c.z;
            sl.result[s] = r;
        }
    }
}

__global__ void advanceKernel(WfControl* ctl)
{
    const int parity = ctl->parity;
    ctl->rays_traced += static_cast<unsigned long long>(ctl->count[kQExtend0 + parity]) +
                        static_cast<unsigned long long>(ctl->count[kQShadow]);
    ctl->count[kQExtend0 + parity] = 0;
    ctl->count[kQRegen0 + parity] = 0;
    ctl->count[kQDiffuse] = 0;
    ctl->count[kQConductor] = 0;
    ctl->count[kQDielectric] = 0;
    ctl->count[kQMix] = 0;
    ctl->count[kQShadow] = 0;
    ctl->fetch_extend = 0;
    ctl->fetch_shadow = 0;
    ctl->parity = parity ^ 1;
    ctl->iterations += 1;
}

__global__ void resetKernel(WfBuffers b, unsigned long long total_items, int job_count)
{
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (i < b.slot_count) {
        b.slots.where[i] = make_int4(-1, 0, 0, 0);
        b.queue[kQRegen0][i] = i;
    }
    if (i < job_count) {
        b.job_done[i] = 0;
    }
    if (b.bin_count != nullptr && i < kBinCount) {
        b.bin_count[i] = 0u;
    }
    if (i == 0) {
        WfControl* ctl = b.control;
        for (int q = 0; q < kQueueCount; ++q) {
            ctl->count[q] = 0;
        }
        ctl->count[kQRegen0] = b.slot_count;
        ctl->parity = 0;
        ctl->next_item = 0;
        ctl->completed = 0;
        ctl->iterations = 0;
        ctl->total_items = total_items;
        ctl->job_count = job_count;
        ctl->fetch_extend = 0;
        ctl->fetch_shadow = 0;
        ctl->rays_traced = 0;
    }
}

// Appending jobs, step 1: parked slots rejoin the current regeneration queue and
// the new jobs' completion counters start at zero.
__global__ void appendCopyKernel(WfBuffers b, int first, int count)
{
    const WfControl* ctl = b.control;
    const int parity = ctl->parity;
    const int parked = ctl->count[kQParked];
    const int base = ctl->count[kQRegen0 + parity];
    const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (i < parked) {
        b.queue[kQRegen0 + parity][base + i] = b.queue[kQParked][i];
    }
    if (i < count) {
        b.job_done[first + i] = 0;
    }
}

// Appending jobs, step 2 (one thread, after step 1): queue counts and the batch's
// size. Claims past the old end only happened once every old item was claimed, so
// handing out resumes at the old end.
__global__ void appendFinishKernel(WfBuffers b, int first, int count, unsigned long long new_total_items)
{
    WfControl* ctl = b.control;
    const int parity = ctl->parity;
    ctl->count[kQRegen0 + parity] += ctl->count[kQParked];
    ctl->count[kQParked] = 0;
    if (ctl->next_item > ctl->total_items) {
        ctl->next_item = ctl->total_items;
    }
    ctl->total_items = new_total_items;
    ctl->job_count = first + count;
}

// Probe: queries of given rays traced either as the wavefront traces them
// (persistent, warp fetch, node-then-leaf steps) or one query per thread through
// the shared out-of-line traversal, writing the raw hits (hit flag, FP32 t bits,
// object leaf position, triangle table position) for a bit-for-bit comparison.
template <int STACK>
__global__ void __launch_bounds__(128, kTraceBlocksPerSm) traceModesKernel(const DevScene scene, const float* rays,
                                                                         int count, float t_min, float t_max,
                                                                         bool any, int mode, int* counter,
                                                                         unsigned int* error_flag, int* out_hit,
                                                                         unsigned int* out_t, unsigned int* out_obj,
                                                                         unsigned int* out_tri)
{
    extern __shared__ uint2 stack[];
    uint2* const lane_stack = stack + threadIdx.x;
    // The persistent modes use the 4-byte stack entries of the wavefront's kernels.
    unsigned* const lane_refs = reinterpret_cast<unsigned*>(stack) + threadIdx.x;
    const int stride = static_cast<int>(blockDim.x);
    const auto store = [&](int i, bool found, const TraceHit& hit) {
        out_hit[i] = found ? 1 : 0;
        out_t[i] = found ? __float_as_uint(hit.t) : 0u;
        out_obj[i] = found ? hit.obj_pos : kNoPrim;
        out_tri[i] = found ? hit.tri_pos : kNoPrim;
    };
    if (mode == 0) {
        const int i = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
        if (i < count) {
            TraceHit hit;
            float tmax = t_max;
            const float3 o = mk(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
            const float3 d = mk(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
            const bool found = traceQuery(scene, o, d, t_min, tmax, SkipRule::none(), hit, lane_stack, stride, STACK,
                                          error_flag, nullptr, any);
            store(i, found, hit);
        }
        return;
    }
    WarpFetch fetch{0, 0, 32, false};
    TraceState q;
    int i = -1;
    bool active = false;
    for (;;) {
        const int next = fetch.take(counter, count, !active);
        bool finished = false;
        if (next >= 0) {
            i = next;
            const float3 o = mk(rays[6 * i], rays[6 * i + 1], rays[6 * i + 2]);
            const float3 d = mk(rays[6 * i + 3], rays[6 * i + 4], rays[6 * i + 5]);
            active = traceBegin(scene, q, o, d, t_min, t_max);
            finished = !active;
        }
        if (__ballot_sync(0xFFFFFFFFu, active || finished) == 0u) {
            break;
        }
        bool more = false;
        if (active) {
            if (mode == 3) {
                more = traceAdvance<kLoopQuery>(scene, q, SkipRule::none(), lane_refs, stride, STACK, error_flag,
                                                nullptr, any);
            } else if (mode == 2) {
                more = traceAdvance<kLoopOneStep>(scene, q, SkipRule::none(), lane_refs, stride, STACK, error_flag,
                                                  nullptr, any);
            } else {
                more = traceAdvance<kLoopNodesThenLeaf>(scene, q, SkipRule::none(), lane_refs, stride, STACK,
                                                        error_flag, nullptr, any);
            }
        }
        if (active && !more) {
            active = false;
            finished = true;
        }
        if (finished) {
            store(i, q.found, q.hit);
        }
    }
}

} // namespace

cudaError_t launchTraceModes(const DevScene& scene, const float* rays, int count, float t_min, float t_max, bool any,
                             int mode, int stack, int* counter, unsigned int* error_flag, int* out_hit,
                             unsigned int* out_t, unsigned int* out_obj, unsigned int* out_tri, cudaStream_t stream)
{
    return withStack(stack, [&](auto size) {
        constexpr int S = decltype(size)::value;
        const std::size_t smem = static_cast<std::size_t>(S) * 128 * sizeof(uint2);
        const cudaError_t e = allowStackMemory(traceModesKernel<S>, S);
        if (e != cudaSuccess) {
            return e;
        }
        const int blocks = mode != 0 ? 148 * 4 : (count + 127) / 128;
        traceModesKernel<S><<<blocks, 128, smem, stream>>>(scene, rays, count, t_min, t_max, any, mode, counter,
                                                           error_flag, out_hit, out_t, out_obj, out_tri);
        return cudaGetLastError();
    });
}

cudaError_t wfPrepare(int stack)
{
    return withStack(stack, [&](auto size) {
        constexpr int S = decltype(size)::value;
        constexpr int kRef = static_cast<int>(sizeof(unsigned));
        cudaError_t e = allowStackMemory(extendKernel<S, kLoopNodesThenLeaf>, S, kRef);
        if (e == cudaSuccess) {
            e = allowStackMemory(shadowKernel<S, kLoopNodesThenLeaf>, S, kRef);
        }
        if (e == cudaSuccess) {
            e = allowStackMemory(extendKernel<S, kLoopOneStep>, S, kRef);
        }
        if (e == cudaSuccess) {
            e = allowStackMemory(shadowKernel<S, kLoopOneStep>, S, kRef);
        }
        if (e == cudaSuccess) {
            e = allowStackMemory(extendKernel<S, kLoopQuery>, S, kRef);
        }
        return e != cudaSuccess ? e : allowStackMemory(shadowKernel<S, kLoopQuery>, S, kRef);
    });
}

cudaError_t wfTraceBlocksPerSm(int stack, int* out)
{
    *out = 1;
    return withStack(stack, [&](auto size) {
        constexpr int S = decltype(size)::value;
        const std::size_t smem = static_cast<std::size_t>(S) * 128 * sizeof(unsigned);
        int extend = 0;
        int shadow = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&extend, extendKernel<S, kLoopNodesThenLeaf>,
                                                                      128, smem);
        if (e == cudaSuccess) {
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&shadow, shadowKernel<S, kLoopNodesThenLeaf>, 128, smem);
        }
        const int blocks = extend < shadow ? extend : shadow;
        *out = blocks > 0 ? blocks : 1;
        return e;
    });
}

cudaError_t wfReset(const WfBuffers& b, unsigned long long total_items, int job_count, cudaStream_t stream)
{
    int n = b.slot_count > job_count ? b.slot_count : job_count;
    n = n > kBinCount ? n : kBinCount;
    resetKernel<<<(n + 255) / 256, 256, 0, stream>>>(b, total_items, job_count);
    return cudaGetLastError();
}

cudaError_t wfAppend(const WfBuffers& b, int first, int count, unsigned long long new_total_items,
                     cudaStream_t stream)
{
    const int n = b.slot_count > count ? b.slot_count : count;
    appendCopyKernel<<<(n + 255) / 256, 256, 0, stream>>>(b, first, count);
    appendFinishKernel<<<1, 1, 0, stream>>>(b, first, count, new_total_items);
    return cudaGetLastError();
}

cudaError_t wfIteration(const WfJob* jobs, const WfBuffers& b, const WfLaunch& launch, unsigned int* error_flag,
                        cudaStream_t stream, const WfSide* side)
{
    const int g = launch.blocks;
    const int tg = launch.trace_blocks > 0 ? launch.trace_blocks : launch.blocks;
    const int fetch = launch.fetch_batch > 0 ? launch.fetch_batch : 32;
    // The persistent traversal kernels keep 4-byte stack entries (references only).
    const auto smemFor = [](int entries) { return static_cast<std::size_t>(entries) * 128 * sizeof(unsigned); };
    regenKernel<<<g, 128, 0, stream>>>(jobs, b);
    const bool binned = launch.ray_sort != 0 && b.binned != nullptr;
    if (binned) {
        binKeysKernel<false><<<g, 128, 0, stream>>>(jobs, b);
        binScanKernel<<<1, 1024, 0, stream>>>(b);
        binScatterKernel<false><<<g, 128, 0, stream>>>(b);
    }
    withStack(launch.stack, [&](auto size) {
        constexpr int S = decltype(size)::value;
        if (launch.trace_loop == kLoopOneStep) {
            extendKernel<S, kLoopOneStep><<<tg, 128, smemFor(S), stream>>>(jobs, b, error_flag, fetch, binned);
        } else if (launch.trace_loop == kLoopQuery) {
            extendKernel<S, kLoopQuery><<<tg, 128, smemFor(S), stream>>>(jobs, b, error_flag, fetch, binned);
        } else {
            extendKernel<S, kLoopNodesThenLeaf><<<tg, 128, smemFor(S), stream>>>(jobs, b, error_flag, fetch, binned);
        }
        return 0;
    });
    if (side != nullptr) {
        cudaError_t e = cudaEventRecord(side->fork, stream);
        for (int k = 0; k < 3 && e == cudaSuccess; ++k) {
            e = cudaStreamWaitEvent(side->stream[k], side->fork, 0);
        }
        if (e != cudaSuccess) {
            return e;
        }
        shadeKernel<kClassDiffuse><<<g, 128, 0, stream>>>(jobs, b);
        shadeKernel<kClassConductor><<<g, 128, 0, side->stream[0]>>>(jobs, b);
        shadeKernel<kClassDielectric><<<g, 128, 0, side->stream[1]>>>(jobs, b);
        shadeKernel<kClassMix><<<g, 128, 0, side->stream[2]>>>(jobs, b);
        for (int k = 0; k < 3 && e == cudaSuccess; ++k) {
            e = cudaEventRecord(side->join[k], side->stream[k]);
            if (e == cudaSuccess) {
                e = cudaStreamWaitEvent(stream, side->join[k], 0);
            }
        }
        if (e != cudaSuccess) {
            return e;
        }
    } else {
        shadeKernel<kClassDiffuse><<<g, 128, 0, stream>>>(jobs, b);
        shadeKernel<kClassConductor><<<g, 128, 0, stream>>>(jobs, b);
        shadeKernel<kClassDielectric><<<g, 128, 0, stream>>>(jobs, b);
        shadeKernel<kClassMix><<<g, 128, 0, stream>>>(jobs, b);
    }
    // The shadow rays too, when binning is 2. The binned buffer is free again:
    // the extend kernel has read it.
    const bool binned_shadows = launch.ray_sort == 2 && b.binned != nullptr;
    if (binned_shadows) {
        binKeysKernel<true><<<g, 128, 0, stream>>>(jobs, b);
        binScanKernel<<<1, 1024, 0, stream>>>(b);
        binScatterKernel<true><<<g, 128, 0, stream>>>(b);
    }
    withStack(launch.stack, [&](auto size) {
        constexpr int S = decltype(size)::value;
        if (launch.trace_loop == kLoopOneStep) {
            shadowKernel<S, kLoopOneStep><<<tg, 128, smemFor(S), stream>>>(jobs, b, error_flag, fetch,
                                                                           binned_shadows);
        } else if (launch.trace_loop == kLoopQuery) {
            shadowKernel<S, kLoopQuery><<<tg, 128, smemFor(S), stream>>>(jobs, b, error_flag, fetch,
                                                                         binned_shadows);
        } else {
            shadowKernel<S, kLoopNodesThenLeaf><<<tg, 128, smemFor(S), stream>>>(jobs, b, error_flag, fetch,
                                                                                 binned_shadows);
        }
        return 0;
    });
    advanceKernel<<<1, 1, 0, stream>>>(b.control);
    return cudaGetLastError();
}

} // namespace albedo_b200
