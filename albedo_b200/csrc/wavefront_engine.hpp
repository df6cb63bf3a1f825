// Host side of the wavefront renderer: owns the path slots and queues on one
// device and drives iterations until every pixel of a batch of jobs is done.
#pragma once

#include "kernels/wavefront.cuh"

#include <cuda_runtime_api.h>

#include <vector>

namespace albedo_b200 {

class WavefrontEngine {
public:
    // `slot_count` path slots (about 240 bytes each) on the current device.
    explicit WavefrontEngine(int slot_count);
    ~WavefrontEngine();
    WavefrontEngine(const WavefrontEngine&) = delete;
    WavefrontEngine& operator=(const WavefrontEngine&) = delete;

    // Renders `jobs` into their (device) accumulators, adding width*height*n^2
    // samples per job. Iterations are captured once into a CUDA graph of
    // `iterations_per_graph` iterations and replayed; completion is polled one
    // graph behind, so the device never waits for the host. Returns when all
    // pixels are done (the stream is then idle).
    void render(const std::vector<WfJob>& jobs, int stack, unsigned int* error_flag, cudaStream_t stream);

    int slotCount() const { return buffers_.slot_count; }
    unsigned long long lastIterations() const { return last_iterations_; }

    // Launch shape of the queue kernels; the autotuner sets it.
    void setLaunch(int blocks_per_sm, int iterations_per_graph);

private:
    void renderOnOwnStream(const std::vector<WfJob>& jobs, int stack, unsigned int* error_flag);

    cudaStream_t stream_{nullptr};
    cudaEvent_t ordering_{nullptr};
    WfBuffers buffers_{};
    void* slab_{nullptr};
    WfJob* device_jobs_{nullptr};
    int job_capacity_{0};
    WfJob* staging_jobs_{nullptr};
    WfControl* host_control_{nullptr}; // pinned: two snapshots for pipelined polling
    int blocks_per_sm_{8};
    int iterations_per_graph_{4};
    int sm_count_{148};
    unsigned long long last_iterations_{0};
};

} // namespace albedo_b200
