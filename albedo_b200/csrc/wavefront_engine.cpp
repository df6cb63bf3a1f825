// Wavefront engine: slot and queue allocation, job upload, graph capture and
// pipelined completion polling.
#include "wavefront_engine.hpp"

#include <algorithm>
#include <cstring>
#include <format>
#include <string>
#include <new>
#include <stdexcept>

namespace albedo_b200 {

namespace {

void cudaCheck(cudaError_t e, const char* what)
{
    if (e == cudaErrorMemoryAllocation) {
        throw std::bad_alloc{};
    }
    if (e != cudaSuccess) {
        throw std::runtime_error{std::format("{}: {}", what, cudaGetErrorString(e))};
    }
}

std::size_t align256(std::size_t n) { return (n + 255) & ~std::size_t{255}; }

} // namespace

WavefrontEngine::WavefrontEngine(int slot_count)
{
    if (slot_count <= 0) {
        throw std::invalid_argument{"the wavefront engine needs at least one slot"};
    }
    const auto n{static_cast<std::size_t>(slot_count)};
    const std::size_t f4{align256(n * sizeof(float4))};
    const std::size_t f2{align256(n * sizeof(float2))};
    const std::size_t u2{align256(n * sizeof(ulonglong2))};
    const std::size_t q{align256(n * sizeof(int))};
    const std::size_t total{12 * f4 + f2 + u2 + kQueueCount * q + align256(sizeof(WfControl))};
    cudaCheck(cudaMalloc(&slab_, total), "wavefront slots");
    auto* p{static_cast<char*>(slab_)};
    const auto take = [&](std::size_t bytes) {
        void* r{p};
        p += bytes;
        return r;
    };
    WfSlots& s{buffers_.slots};
    s.ray_o = static_cast<float4*>(take(f4));
    s.ray_d = static_cast<float4*>(take(f4));
    s.throughput = static_cast<float4*>(take(f4));
    s.result = static_cast<float4*>(take(f4));
    s.arrival = static_cast<float4*>(take(f4));
    s.skip = static_cast<uint4*>(take(f4));
    s.where = static_cast<int4*>(take(f4));
    s.hit = static_cast<float4*>(take(f4));
    s.shadow_o = static_cast<float4*>(take(f4));
    s.shadow_d = static_cast<float4*>(take(f4));
    s.shadow_skip = static_cast<uint4*>(take(f4));
    s.shadow_c = static_cast<float4*>(take(f4));
    s.hit_b = static_cast<float2*>(take(f2));
    s.rng = static_cast<ulonglong2*>(take(u2));
    for (int i{0}; i < kQueueCount; ++i) {
        buffers_.queue[i] = static_cast<int*>(take(q));
    }
    buffers_.control = static_cast<WfControl*>(take(align256(sizeof(WfControl))));
    buffers_.slot_count = slot_count;
    cudaCheck(cudaMallocHost(&host_control_, 2 * sizeof(WfControl)), "pinned control");
    std::memset(host_control_, 0, 2 * sizeof(WfControl));
    int device{0};
    cudaCheck(cudaGetDevice(&device), "cudaGetDevice");
    cudaCheck(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device), "SM count");
    cudaCheck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "engine stream");
    cudaCheck(cudaEventCreateWithFlags(&ordering_, cudaEventDisableTiming), "engine event");
}

WavefrontEngine::~WavefrontEngine()
{
    cudaStreamSynchronize(stream_);
    cudaEventDestroy(ordering_);
    cudaStreamDestroy(stream_);
    cudaFree(slab_);
    cudaFree(device_jobs_);
    cudaFreeHost(staging_jobs_);
    cudaFreeHost(host_control_);
}

void WavefrontEngine::setLaunch(int blocks_per_sm, int iterations_per_graph)
{
    if (blocks_per_sm <= 0 || iterations_per_graph <= 0) {
        throw std::invalid_argument{"launch shape must be positive"};
    }
    blocks_per_sm_ = blocks_per_sm;
    iterations_per_graph_ = iterations_per_graph;
}

void WavefrontEngine::render(const std::vector<WfJob>& input, int stack, unsigned int* error_flag,
                             cudaStream_t caller)
{
    if (input.empty()) {
        return;
    }
    // Work runs on the engine's own stream (graphs cannot be captured on the
    // legacy default stream), ordered after the caller's stream and before
    // anything the caller enqueues next.
    cudaCheck(cudaEventRecord(ordering_, caller), "ordering event");
    cudaCheck(cudaStreamWaitEvent(stream_, ordering_, 0), "ordering wait");
    renderOnOwnStream(input, stack, error_flag);
    cudaCheck(cudaEventRecord(ordering_, stream_), "ordering event");
    cudaCheck(cudaStreamWaitEvent(caller, ordering_, 0), "ordering wait");
}

void WavefrontEngine::renderOnOwnStream(const std::vector<WfJob>& input, int stack, unsigned int* error_flag)
{
    const cudaStream_t stream{stream_};
    const auto count{static_cast<int>(input.size())};
    if (count > job_capacity_) {
        cudaFree(device_jobs_);
        cudaFreeHost(staging_jobs_);
        device_jobs_ = nullptr;
        staging_jobs_ = nullptr;
        job_capacity_ = 0;
        cudaCheck(cudaMalloc(&device_jobs_, static_cast<std::size_t>(count) * sizeof(WfJob)), "job table");
        cudaCheck(cudaMallocHost(&staging_jobs_, static_cast<std::size_t>(count) * sizeof(WfJob)), "job staging");
        job_capacity_ = count;
    }
    // The stream may still read the staging copy of a previous render.
    cudaCheck(cudaStreamSynchronize(stream), "stream");
    unsigned long long total{0};
    for (int j{0}; j < count; ++j) {
        staging_jobs_[j] = input[static_cast<std::size_t>(j)];
        staging_jobs_[j].item_begin = static_cast<long long>(total);
        total += static_cast<unsigned long long>(input[static_cast<std::size_t>(j)].width) *
                 static_cast<unsigned long long>(input[static_cast<std::size_t>(j)].height);
        staging_jobs_[j].item_end = static_cast<long long>(total);
    }
    cudaCheck(cudaMemcpyAsync(device_jobs_, staging_jobs_, static_cast<std::size_t>(count) * sizeof(WfJob),
                              cudaMemcpyHostToDevice, stream),
              "job upload");
    cudaCheck(wfReset(buffers_, total, stream), "wavefront reset");

    const WfLaunch launch{sm_count_ * blocks_per_sm_, 128, stack};
    cudaCheck(wfPrepare(stack), "wavefront kernel attributes");
    cudaGraph_t graph{nullptr};
    cudaGraphExec_t exec{nullptr};
    cudaCheck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capture begin");
    cudaError_t captured{cudaSuccess};
    for (int i{0}; i < iterations_per_graph_ && captured == cudaSuccess; ++i) {
        captured = wfIteration(device_jobs_, count, total, buffers_, launch, error_flag, stream);
    }
    const cudaError_t ended{cudaStreamEndCapture(stream, &graph)};
    cudaCheck(captured, "wavefront iteration");
    cudaCheck(ended, "capture end");
    cudaCheck(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
    cudaGraphDestroy(graph);

    // Poll one graph behind: launch graph k + 1 before looking at graph k's snapshot.
    cudaEvent_t done[2];
    cudaCheck(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming), "event");
    cudaCheck(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming), "event");
    // A slot finishes its pixel within n^2 (max_depth + 2) iterations, so a batch
    // that completes no pixel for longer than that is stuck (a defect, reported
    // instead of looping forever).
    unsigned long long stall_limit{16};
    for (const WfJob& j : input) {
        const auto n2{static_cast<unsigned long long>(j.samples_per_axis) * static_cast<unsigned long long>(j.samples_per_axis)};
        stall_limit = std::max(stall_limit, n2 * static_cast<unsigned long long>(j.max_depth + 2) + 16);
    }
    unsigned long long last_completed{0};
    unsigned long long last_progress_iteration{0};
    int launched{0};
    bool finished{false};
    std::string failure;
    while (!finished) {
        const int slot{launched & 1};
        cudaCheck(cudaGraphLaunch(exec, stream), "graph launch");
        cudaCheck(cudaMemcpyAsync(&host_control_[slot], buffers_.control, sizeof(WfControl), cudaMemcpyDeviceToHost,
                                  stream),
                  "control snapshot");
        cudaCheck(cudaEventRecord(done[slot], stream), "event record");
        ++launched;
        if (launched >= 2) {
            const int previous{(launched - 2) & 1};
            cudaCheck(cudaEventSynchronize(done[previous]), "event sync");
            const WfControl& snapshot{host_control_[previous]};
            finished = snapshot.completed >= total;
            if (snapshot.completed != last_completed) {
                last_completed = snapshot.completed;
                last_progress_iteration = snapshot.iterations;
            } else if (snapshot.iterations - last_progress_iteration > stall_limit) {
                failure = std::format("wavefront batch made no progress for {} iterations ({} of {} pixels done)",
                                      snapshot.iterations - last_progress_iteration, snapshot.completed, total);
                finished = true;
            }
        }
    }
    cudaCheck(cudaEventSynchronize(done[(launched - 1) & 1]), "event sync");
    last_iterations_ = host_control_[(launched - 1) & 1].iterations;
    cudaEventDestroy(done[0]);
    cudaEventDestroy(done[1]);
    cudaGraphExecDestroy(exec);
    if (!failure.empty()) {
        throw std::runtime_error{failure};
    }
}

} // namespace albedo_b200
