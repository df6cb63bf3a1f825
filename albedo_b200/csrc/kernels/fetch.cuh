// Warp-level work distribution for persistent kernels.
#pragma once

#include "common.cuh"

namespace albedo_b200 {

// Deals work items [0, count) to the lanes of a warp that want one, in lane
// order; the warp claims `batch` items at a time with one atomicAdd on `counter`
// (global or shared memory). All 32 lanes call take() together.
struct WarpFetch {
    int next;
    int end;
    int batch;
    bool drained;

    ALB_DEV int take(int* counter, int count, bool want)
    {
        const int lane = static_cast<int>(threadIdx.x & 31u);
        const unsigned below = (1u << lane) - 1u;
        unsigned need = __ballot_sync(0xFFFFFFFFu, want);
        int got = -1;
        while (need != 0u && !drained) {
            if (next >= end) {
                int base = 0;
                if (lane == 0) {
                    base = atomicAdd(counter, batch);
                }
                base = __shfl_sync(0xFFFFFFFFu, base, 0);
                if (base >= count) {
                    drained = true;
                    break;
                }
                next = base;
                end = base + batch < count ? base + batch : count;
            }
            const int avail = end - next;
            const int rank = __popc(need & below);
            if (((need >> lane) & 1u) != 0u && rank < avail) {
                got = next + rank;
            }
            const int wanted = __popc(need);
            next += wanted < avail ? wanted : avail;
            need = __ballot_sync(0xFFFFFFFFu, want && got < 0);
        }
        return got;
    }
};

} // namespace albedo_b200
