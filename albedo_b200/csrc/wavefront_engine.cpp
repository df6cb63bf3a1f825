// Wavefront engine: slot, queue and job-table allocation, graph capture, job
// submission between graph launches, and pipelined completion polling.
#include "wavefront_engine.hpp"

#include <algorithm>
#include <cstring>
#include <format>
#include <new>
#include <stdexcept>
#include <string>

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

WavefrontEngine::WavefrontEngine(int slot_count, int job_capacity)
{
    if (slot_count <= 0 || job_capacity <= 0) {
        throw std::invalid_argument{"the wavefront engine needs at least one slot and one job"};
    }
    const auto n{static_cast<std::size_t>(slot_count)};
    const std::size_t f4{align256(n * sizeof(float4))};
    const std::size_t f2{align256(n * sizeof(float2))};
    const std::size_t u2{align256(n * sizeof(ulonglong2))};
    const std::size_t q{align256(n * sizeof(int))};
    const auto jobs{static_cast<std::size_t>(job_capacity)};
    const std::size_t bins{align256(kBinCount * sizeof(unsigned int))};
    const std::size_t total{12 * f4 + f2 + u2 + kQueueCount * q + align256(sizeof(WfControl)) +
                            align256(jobs * sizeof(unsigned long long)) + align256(jobs * sizeof(WfJob)) + 2 * q +
                            2 * bins};
    cudaCheck(cudaMalloc(&slab_, total), "wavefront slots");
    device_bytes_ = total;
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
    buffers_.job_done = static_cast<unsigned long long*>(take(align256(jobs * sizeof(unsigned long long))));
    device_jobs_ = static_cast<WfJob*>(take(align256(jobs * sizeof(WfJob))));
    buffers_.bin_key = static_cast<unsigned int*>(take(q));
    buffers_.binned = static_cast<int*>(take(q));
    buffers_.bin_count = static_cast<unsigned int*>(take(bins));
    buffers_.bin_cursor = static_cast<unsigned int*>(take(bins));
    buffers_.slot_count = slot_count;
    job_capacity_ = job_capacity;
    cudaCheck(cudaMallocHost(&host_control_, 2 * sizeof(WfControl)), "pinned control");
    cudaCheck(cudaMallocHost(&host_done_, 2 * jobs * sizeof(unsigned long long)), "pinned counters");
    cudaCheck(cudaMallocHost(&staging_jobs_, jobs * sizeof(WfJob)), "pinned jobs");
    std::memset(host_control_, 0, 2 * sizeof(WfControl));
    int device{0};
    cudaCheck(cudaGetDevice(&device), "cudaGetDevice");
    cudaCheck(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device), "SM count");
    cudaCheck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "engine stream");
    for (int k{0}; k < 3; ++k) {
        cudaCheck(cudaStreamCreateWithFlags(&side_.stream[k], cudaStreamNonBlocking), "engine side stream");
        cudaCheck(cudaEventCreateWithFlags(&side_.join[k], cudaEventDisableTiming), "engine event");
    }
    cudaCheck(cudaEventCreateWithFlags(&side_.fork, cudaEventDisableTiming), "engine event");
    cudaCheck(cudaEventCreateWithFlags(&ordering_, cudaEventDisableTiming), "engine event");
    cudaCheck(cudaEventCreateWithFlags(&step_done_[0], cudaEventDisableTiming), "engine event");
    cudaCheck(cudaEventCreateWithFlags(&step_done_[1], cudaEventDisableTiming), "engine event");
}

WavefrontEngine::~WavefrontEngine()
{
    cudaStreamSynchronize(stream_);
    if (graph_ != nullptr) {
        cudaGraphExecDestroy(graph_);
    }
    cudaEventDestroy(step_done_[0]);
    cudaEventDestroy(step_done_[1]);
    cudaEventDestroy(ordering_);
    for (int k{0}; k < 3; ++k) {
        cudaEventDestroy(side_.join[k]);
        cudaStreamDestroy(side_.stream[k]);
    }
    cudaEventDestroy(side_.fork);
    cudaStreamDestroy(stream_);
    cudaFree(slab_);
    cudaFreeHost(staging_jobs_);
    cudaFreeHost(host_done_);
    cudaFreeHost(host_control_);
}

void WavefrontEngine::setShape(const WfShape& shape)
{
    if (shape.blocks_per_sm <= 0 || shape.iterations_per_graph <= 0 || shape.trace_blocks_per_sm < 0 ||
        shape.fetch_batch <= 0 || shape.trace_loop < 0 || shape.trace_loop > 2 || shape.ray_sort < 0 ||
        shape.ray_sort > 2) {
        throw std::invalid_argument{"wavefront launch shape values must be positive"};
    }
    shape_ = shape;
}

void WavefrontEngine::open(int stack, unsigned int* error_flag)
{
    if (open_) {
        throw std::logic_error{"the wavefront batch is already open"};
    }
    cudaCheck(cudaStreamSynchronize(stream_), "engine stream");
    job_count_ = 0;
    total_items_ = 0;
    job_pixels_.clear();
    in_flight_.clear();
    steps_launched_ = 0;
    steps_polled_ = 0;
    stall_limit_ = 16;
    last_completed_ = 0;
    last_progress_iteration_ = 0;
    cudaCheck(wfReset(buffers_, 0, 0, stream_), "wavefront reset");
    cudaCheck(wfPrepare(stack), "wavefront kernel attributes");
    int trace_per_sm{1};
    cudaCheck(wfTraceBlocksPerSm(stack, &trace_per_sm), "traversal residency");
    if (shape_.trace_blocks_per_sm > 0) {
        trace_per_sm = std::min(trace_per_sm, shape_.trace_blocks_per_sm);
    }
    const WfLaunch launch{sm_count_ * shape_.blocks_per_sm, 128, stack, sm_count_ * trace_per_sm, shape_.fetch_batch,
                          shape_.trace_loop, shape_.ray_sort};
    cudaGraph_t graph{nullptr};
    cudaCheck(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture begin");
    cudaError_t captured{cudaSuccess};
    for (int i{0}; i < shape_.iterations_per_graph && captured == cudaSuccess; ++i) {
        captured = wfIteration(device_jobs_, buffers_, launch, error_flag, stream_,
                               parallel_shade_ ? &side_ : nullptr);
    }
    const cudaError_t ended{cudaStreamEndCapture(stream_, &graph)};
    cudaCheck(captured, "wavefront iteration");
    cudaCheck(ended, "capture end");
    const cudaError_t instantiated{cudaGraphInstantiate(&graph_, graph, 0)};
    cudaGraphDestroy(graph);
    cudaCheck(instantiated, "graph instantiate");
    open_ = true;
}

int WavefrontEngine::submit(const WfJob& input)
{
    if (!open_) {
        throw std::logic_error{"submit needs an open wavefront batch"};
    }
    if (job_count_ >= job_capacity_) {
        throw std::length_error{std::format("the job table holds {} jobs", job_capacity_)};
    }
    const int index{job_count_};
    // The staging entry of a job index is written once per batch, so no copy in
    // flight can still be reading it.
    WfJob& staged{staging_jobs_[index]};
    staged = input;
    const long long pixels{static_cast<long long>(input.width) * input.height};
    staged.item_begin = static_cast<long long>(total_items_);
    staged.item_end = staged.item_begin + pixels;
    cudaCheck(cudaMemcpyAsync(&device_jobs_[index], &staged, sizeof(WfJob), cudaMemcpyHostToDevice, stream_),
              "job upload");
    total_items_ += static_cast<unsigned long long>(pixels);
    cudaCheck(wfAppend(buffers_, index, 1, total_items_, stream_), "job append");
    ++job_count_;
    job_pixels_.push_back(pixels);
    in_flight_.push_back(index);
    const auto n2{static_cast<unsigned long long>(input.samples_per_axis) * input.samples_per_axis};
    stall_limit_ = std::max(stall_limit_, n2 * (static_cast<unsigned long long>(input.max_depth) + 2) + 16);
    return index;
}

void WavefrontEngine::step()
{
    if (!open_) {
        throw std::logic_error{"step needs an open wavefront batch"};
    }
    const int slot{steps_launched_ & 1};
    cudaCheck(cudaGraphLaunch(graph_, stream_), "graph launch");
    cudaCheck(cudaMemcpyAsync(&host_control_[slot], buffers_.control, sizeof(WfControl), cudaMemcpyDeviceToHost,
                              stream_),
              "control snapshot");
    if (job_count_ > 0) {
        cudaCheck(cudaMemcpyAsync(host_done_ + static_cast<std::size_t>(slot) * job_capacity_, buffers_.job_done,
                                  static_cast<std::size_t>(job_count_) * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, stream_),
                  "counter snapshot");
    }
    cudaCheck(cudaEventRecord(step_done_[slot], stream_), "event record");
    ++steps_launched_;
}

std::vector<int> WavefrontEngine::poll()
{
    std::vector<int> finished;
    // Look at the step before the last, so the device always has a graph queued.
    const int target{steps_launched_ - (steps_launched_ >= 2 ? 2 : 1)};
    if (target < steps_polled_ || steps_launched_ == 0) {
        return finished;
    }
    const int slot{target & 1};
    cudaCheck(cudaEventSynchronize(step_done_[slot]), "event sync");
    steps_polled_ = target + 1;
    const WfControl& snapshot{host_control_[slot]};
    const unsigned long long* done{host_done_ + static_cast<std::size_t>(slot) * job_capacity_};
    last_iterations_ = snapshot.iterations;
    last_rays_ = snapshot.rays_traced;
    std::vector<int> still;
    for (const int j : in_flight_) {
        // A job submitted after this snapshot was taken is not in it yet.
        if (j < snapshot.job_count && static_cast<long long>(done[j]) >= job_pixels_[static_cast<std::size_t>(j)]) {
            finished.push_back(j);
        } else {
            still.push_back(j);
        }
    }
    in_flight_.swap(still);
    if (snapshot.completed != last_completed_) {
        last_completed_ = snapshot.completed;
        last_progress_iteration_ = snapshot.iterations;
    } else if (!in_flight_.empty() && snapshot.iterations - last_progress_iteration_ > stall_limit_) {
        throw std::runtime_error{std::format("wavefront batch made no progress for {} iterations ({} of {} pixels done)",
                                             snapshot.iterations - last_progress_iteration_, snapshot.completed,
                                             total_items_)};
    }
    return finished;
}

bool WavefrontEngine::saturated() const
{
    if (steps_polled_ == 0) {
        return false;
    }
    const WfControl& snapshot{host_control_[(steps_polled_ - 1) & 1]};
    return snapshot.next_item >= snapshot.total_items;
}

void WavefrontEngine::close()
{
    if (!open_) {
        return;
    }
    cudaStreamSynchronize(stream_);
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
    open_ = false;
}

void WavefrontEngine::render(const std::vector<WfJob>& jobs, int stack, unsigned int* error_flag, cudaStream_t caller)
{
    if (jobs.empty()) {
        return;
    }
    if (static_cast<int>(jobs.size()) > job_capacity_) {
        throw std::invalid_argument{std::format("a batch holds at most {} jobs", job_capacity_)};
    }
    cudaCheck(cudaEventRecord(ordering_, caller), "ordering event");
    cudaCheck(cudaStreamWaitEvent(stream_, ordering_, 0), "ordering wait");
    open(stack, error_flag);
    try {
        // Longest pixels first: a pixel's samples run in sequence on one slot,
        // so the jobs with the most samples per pixel are handed out first and
        // the batch does not end on a tail of their pixels alone. Each job's
        // image does not depend on the order.
        std::vector<std::size_t> order(jobs.size());
        for (std::size_t i{0}; i < order.size(); ++i) {
            order[i] = i;
        }
        std::stable_sort(order.begin(), order.end(), [&](std::size_t a, std::size_t b) {
            const auto work = [&](const WfJob& j) {
                // In 64 bits: max_depth may be near INT_MAX.
                return static_cast<long long>(j.samples_per_axis) * j.samples_per_axis *
                       (static_cast<long long>(j.max_depth) + 1);
            };
            return work(jobs[a]) > work(jobs[b]);
        });
        for (const std::size_t i : order) {
            submit(jobs[i]);
        }
        while (!in_flight_.empty()) {
            step();
            static_cast<void>(poll());
        }
    } catch (...) {
        close();
        throw;
    }
    // Drain the graph still queued after the last poll.
    cudaCheck(cudaStreamSynchronize(stream_), "engine stream");
    last_iterations_ = host_control_[(steps_launched_ - 1) & 1].iterations;
    last_rays_ = host_control_[(steps_launched_ - 1) & 1].rays_traced;
    close();
    cudaCheck(cudaEventRecord(ordering_, stream_), "ordering event");
    cudaCheck(cudaStreamWaitEvent(caller, ordering_, 0), "ordering wait");
}

} // namespace albedo_b200
