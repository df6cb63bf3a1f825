// Host side of the wavefront renderer: owns the path slots, queues and job table
// on one device and drives iterations, either for one batch of jobs (render) or
// continuously while jobs keep arriving (open / submit / step / poll).
#pragma once

#include "kernels/wavefront.cuh"

#include <cuda_runtime_api.h>

#include <cstdint>
#include <string>
#include <vector>

namespace albedo_b200 {

// Launch shape of the wavefront iteration (the autotuner's knobs).
struct WfShape {
    int blocks_per_sm{8};         // queue kernels (regenerate, shade): blocks per SM
    int iterations_per_graph{4};  // iterations captured in one CUDA graph
    int trace_blocks_per_sm{0};   // persistent traversal kernels: blocks per SM, 0 = as many as fit
    int fetch_batch{32};          // queue entries a traversal warp claims at once
    int trace_loop{2};            // traversal turn shape of the persistent kernels: 0 nodes then leaf, 1 one step,
                                  // 2 the whole query through the out-of-line traversal
    int ray_sort{0};              // 1: bin each bounce's rays by coherence before they are traced; 2: the
                                  // shadow rays too
};

class WavefrontEngine {
public:
    // `slot_count` path slots (264 bytes each, queues and ray binning included)
    // and a table of `job_capacity`
    // jobs on the current device.
    WavefrontEngine(int slot_count, int job_capacity);
    ~WavefrontEngine();
    WavefrontEngine(const WavefrontEngine&) = delete;
    WavefrontEngine& operator=(const WavefrontEngine&) = delete;

    // Renders `jobs` into their (device) accumulators, adding width*height*n^2
    // samples per job; returns when all are done. Work is ordered after the
    // caller's stream and before anything the caller enqueues next.
    void render(const std::vector<WfJob>& jobs, int stack, unsigned int* error_flag, cudaStream_t caller);

    // Continuous batching. open() starts an empty batch whose iterations are
    // captured once into a CUDA graph; submit() appends a job (returning its
    // index) between graph launches, while earlier jobs are in flight; step()
    // launches one graph of iterations; poll() waits for the step before the
    // last and returns the indices of jobs that have finished since the
    // previous poll. A job's accumulators are complete once poll reports it.
    void open(int stack, unsigned int* error_flag);
    int submit(const WfJob& job);
    void step();
    std::vector<int> poll();
    bool isOpen() const { return open_; }
    int jobsInFlight() const { return static_cast<int>(in_flight_.size()); }
    // Jobs whose pixels have all been handed out to slots, so that a new job
    // added now would start being worked on at once.
    bool saturated() const;
    void close();

    int slotCount() const { return buffers_.slot_count; }
    int jobCapacity() const { return job_capacity_; }
    std::size_t deviceBytes() const { return device_bytes_; }
    unsigned long long lastIterations() const { return last_iterations_; }
    // Ray queries (closest hit and shadow) the last render traced, or the open
    // batch has traced as of the last poll.
    unsigned long long lastRays() const { return last_rays_; }

    // Launch shape; the autotuner sets it. Takes effect at the next open() or
    // render().
    void setShape(const WfShape& shape);
    const WfShape& shape() const { return shape_; }

private:
    cudaStream_t stream_{nullptr};
    WfSide side_{};     // branches for the shade kernels
    bool parallel_shade_{true};
    cudaEvent_t ordering_{nullptr};
    cudaEvent_t step_done_[2]{nullptr, nullptr};
    WfBuffers buffers_{};
    void* slab_{nullptr};
    std::size_t device_bytes_{0};
    WfJob* device_jobs_{nullptr};
    WfJob* staging_jobs_{nullptr};     // pinned, one entry per job-table slot
    WfControl* host_control_{nullptr}; // pinned: a snapshot per step parity
    unsigned long long* host_done_{nullptr}; // pinned: per step parity, job_capacity counters
    int job_capacity_{0};
    WfShape shape_{};
    int sm_count_{148};
    unsigned long long last_iterations_{0};
    unsigned long long last_rays_{0};

    // The open batch.
    bool open_{false};
    cudaGraphExec_t graph_{nullptr};
    int job_count_{0};
    unsigned long long total_items_{0};
    std::vector<long long> job_pixels_;
    std::vector<int> in_flight_;
    int steps_launched_{0};
    int steps_polled_{0};
    unsigned long long stall_limit_{16};
    unsigned long long last_completed_{0};
    unsigned long long last_progress_iteration_{0};
};

} // namespace albedo_b200
