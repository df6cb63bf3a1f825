// The C ABI (include/albedo_b200.h): scene building and upload, renders and ray
// queries. Exceptions from the host scene code become status codes with a
// thread-local message; CUDA errors become ALBEDO_DEVICE_ERROR.
#include "../../include/albedo_b200.h"

#include "autotune.hpp"
#include "host/flatten.hpp"
#include "host/scene_file.hpp"
#include "host/srgb.hpp"
#include "kernels/launch.hpp"
#include "wavefront_engine.hpp"

#include <algorithm>
#include <array>
#include <deque>
#include <limits>
#include <map>
#include <mutex>
#include <set>

#include <cuda_runtime_api.h>

#include <cstring>
#include <format>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

using namespace albedo_b200;

namespace {

thread_local std::string g_last_error;

class DeviceError : public std::runtime_error {
public:
    explicit DeviceError(const std::string& what) : std::runtime_error{what} {}
};
class Unsupported : public std::runtime_error {
public:
    explicit Unsupported(const std::string& what) : std::runtime_error{what} {}
};
class TraversalError : public std::runtime_error {
public:
    explicit TraversalError(const std::string& what) : std::runtime_error{what} {}
};

void check(cudaError_t e, const char* what)
{
    if (e == cudaErrorMemoryAllocation) {
        throw std::bad_alloc{};
    }
    if (e != cudaSuccess) {
        throw DeviceError{std::format("{}: {}", what, cudaGetErrorString(e))};
    }
}

template <typename F>
int guarded(F&& body)
{
    try {
        body();
        return ALBEDO_OK;
    } catch (const SceneParseError& e) {
        g_last_error = e.what();
        return ALBEDO_PARSE_ERROR;
    } catch (const std::invalid_argument& e) {
        g_last_error = e.what();
        return ALBEDO_INVALID_ARGUMENT;
    } catch (const std::out_of_range& e) {
        g_last_error = e.what();
        return ALBEDO_OUT_OF_RANGE;
    } catch (const std::bad_alloc&) {
        g_last_error = "out of memory";
        return ALBEDO_OUT_OF_MEMORY;
    } catch (const DeviceError& e) {
        g_last_error = e.what();
        return ALBEDO_DEVICE_ERROR;
    } catch (const Unsupported& e) {
        g_last_error = e.what();
        return ALBEDO_UNSUPPORTED;
    } catch (const LayoutLimitError& e) {
        g_last_error = e.what();
        return ALBEDO_UNSUPPORTED;
    } catch (const TraversalError& e) {
        g_last_error = e.what();
        return ALBEDO_TRAVERSAL_ERROR;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return ALBEDO_IO_ERROR;
    } catch (...) {
        g_last_error = "unknown error";
        return ALBEDO_IO_ERROR;
    }
}

// A device allocation freed on destruction.
struct DeviceBuffer {
    void* ptr{nullptr};
    std::size_t bytes{0};
    DeviceBuffer() = default;
    explicit DeviceBuffer(std::size_t n) : bytes{n}
    {
        if (n > 0) {
            check(cudaMalloc(&ptr, n), "cudaMalloc");
        }
    }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr{o.ptr}, bytes{o.bytes}
    {
        o.ptr = nullptr;
        o.bytes = 0;
    }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept
    {
        std::swap(ptr, o.ptr);
        std::swap(bytes, o.bytes);
        return *this;
    }
    ~DeviceBuffer()
    {
        if (ptr != nullptr) {
            cudaFree(ptr);
        }
    }
    template <typename T>
    T* as() const
    {
        return static_cast<T*>(ptr);
    }
};

template <typename T>
DeviceBuffer upload(const std::vector<T>& host)
{
    DeviceBuffer buffer{host.size() * sizeof(T)};
    if (!host.empty()) {
        check(cudaMemcpy(buffer.ptr, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
    }
    return buffer;
}

template <typename T>
DeviceBuffer uploadRaw(const T* data, std::size_t count)
{
    DeviceBuffer buffer{count * sizeof(T)};
    if (count > 0) {
        check(cudaMemcpy(buffer.ptr, data, count * sizeof(T), cudaMemcpyHostToDevice), "upload");
    }
    return buffer;
}

template <typename T>
void download(T* host, const DeviceBuffer& buffer, std::size_t count)
{
    if (count > 0 && host != nullptr) {
        check(cudaMemcpy(host, buffer.ptr, count * sizeof(T), cudaMemcpyDeviceToHost), "download");
    }
}

// The staging buffer of albedo_render_host on one device.
struct HostStaging {
    std::mutex mutex;
    DeviceBuffer buffer;
};

HostStaging& hostStaging(int device)
{
    static std::mutex table_mutex;
    // Never destroyed: freeing device memory from a static destructor at exit
    // would run after the CUDA runtime has shut down.
    static auto* table{new std::map<int, std::unique_ptr<HostStaging>>};
    const std::lock_guard lock{table_mutex};
    std::unique_ptr<HostStaging>& entry{(*table)[device]};
    if (!entry) {
        entry = std::make_unique<HostStaging>();
    }
    return *entry;
}

Vec3 vec(const double* v) { return {v[0], v[1], v[2]}; }
Rgb rgb(const double* v) { return {v[0], v[1], v[2]}; }

BasicMaterialDesc basicFrom(const albedo_basic_material& m)
{
    BasicMaterialDesc b;
    if (m.kind < 0 || m.kind > 2 || m.texture < 0 || m.texture > 2) {
        throw std::invalid_argument{"unknown material or texture kind"};
    }
    b.kind = static_cast<BasicKind>(m.kind);
    b.texture.kind = static_cast<TextureKind>(m.texture);
    b.texture.a = rgb(m.a);
    b.texture.b = rgb(m.b);
    b.texture.frequency_or_scale = m.frequency_or_scale;
    b.texture.veins = m.veins;
    b.eta = rgb(m.a);
    b.k = rgb(m.b);
    b.ior = m.ior;
    b.roughness = m.roughness;
    return b;
}

} // namespace

struct albedo_scene {
    HostScene host;
    bool prepared{false};
    bool committed{false};
    DeviceImage image;
    DevScene dev{};
    int stack_capacity{0};
    std::vector<DeviceBuffer> buffers;
    DeviceBuffer error_flag;
    // Ray-binning cells of the scene (coherenceGrid), for the wavefront.
    std::array<float, 4> grid{};
    // Megakernel launch shape the autotuner kept for this scene (0: default).
    int mega_tile_width{0};
    int mega_blocks_per_sm{0};
    int mega_inline{0}; // 0 out-of-line traversal, 1 both queries inlined, 2 the closest-hit query inlined

    void requireOpen() const
    {
        if (committed || prepared) {
            throw std::invalid_argument{"the scene is committed and can no longer change"};
        }
    }
    void requireCommitted() const
    {
        if (!committed) {
            throw std::invalid_argument{"the scene has not been committed"};
        }
    }

    // Builds the TLAS and the device tables on the host.
    void prepare()
    {
        if (prepared) {
            return;
        }
        host.finalize();
        image = flattenScene(host);
        grid = coherenceGrid(host);
        stack_capacity = stackCapacityFor(image.stack_need);
        if (stack_capacity == 0) {
            throw Unsupported{std::format("scene hierarchy needs {} traversal stack entries; the device kernels hold 64",
                                          image.stack_need)};
        }
        prepared = true;
    }

    void commit()
    {
        prepare();
        commitPrepared();
    }

    // Uploads the prepared tables to the current device.
    void commitPrepared()
    {
        const auto add = [&](DeviceBuffer&& b) -> void* {
            buffers.push_back(std::move(b));
            return buffers.back().ptr;
        };
        dev.nodes = static_cast<const DevNode*>(add(upload(image.nodes)));
        dev.objects = static_cast<const DevObject*>(add(upload(image.objects)));
        dev.spheres = static_cast<const DevSphere*>(add(upload(image.spheres)));
        dev.triangles = static_cast<const DevTriangle*>(add(upload(image.triangles)));
        dev.attrs = static_cast<const DevTriangleAttr*>(add(upload(image.attrs)));
        dev.instances = static_cast<const DevInstance*>(add(upload(image.instances)));
        dev.materials = static_cast<const DevMaterial*>(add(upload(image.materials)));
        dev.lights = static_cast<const DevLight*>(add(upload(image.lights)));
        dev.object_light = static_cast<const std::int32_t*>(add(upload(image.object_light)));
        dev.instance_to_object64 = static_cast<const double*>(add(upload(image.instance_to_object64)));
        dev.tlas_root = image.tlas_root;
        dev.light_count = static_cast<std::uint32_t>(image.lights.size());
        dev.sky_light = image.sky_light;
        dev.object_count = static_cast<std::uint32_t>(image.objects.size());
        error_flag = DeviceBuffer{sizeof(unsigned int)};
        check(cudaMemset(error_flag.ptr, 0, sizeof(unsigned int)), "cudaMemset");
        committed = true;
    }

    std::size_t deviceBytes() const
    {
        std::size_t total{0};
        for (const DeviceBuffer& b : buffers) {
            total += b.bytes;
        }
        return total;
    }

    // Reads and clears the kernel error flag.
    void collectKernelError() const
    {
        unsigned int flag{0};
        check(cudaMemcpy(&flag, error_flag.ptr, sizeof(flag), cudaMemcpyDeviceToHost), "error flag");
        if (flag != 0) {
            check(cudaMemset(error_flag.ptr, 0, sizeof(flag)), "cudaMemset");
            throw TraversalError{"a traversal stack overflowed; the affected rays were ended"};
        }
    }
};

namespace {

// renderImage's argument checks (render/render_image.cpp:60-67) and
// PixelBuffer's size check (image/pixel_buffer.hpp:30-38).
RenderArgs renderArgsFor(const albedo_scene& scene, const albedo_render_job& job)
{
    scene.requireCommitted();
    if (job.samples_per_axis <= 0) {
        throw std::invalid_argument{std::format("samples per axis must be positive, got {}", job.samples_per_axis)};
    }
    if (job.width <= 0 || job.height <= 0 ||
        static_cast<std::uint64_t>(job.width) > (std::uint64_t{1} << 28) / static_cast<std::uint64_t>(job.height)) {
        throw std::invalid_argument{std::format(
            "invalid image size {}x{}: dimensions must be positive and the image at most {} pixels", job.width,
            job.height, std::uint64_t{1} << 28)};
    }
    if (job.max_depth < 0 || job.roulette_start < 0) {
        throw std::invalid_argument{"path limits must not be negative"};
    }
    if (job.estimator < 0 || job.estimator > 2) {
        throw std::invalid_argument{"unknown estimator"};
    }
    if (!scene.host.has_camera) {
        throw std::invalid_argument{"the scene has no camera"};
    }
    if (job.method != ALBEDO_MEGAKERNEL && job.method != ALBEDO_WAVEFRONT) {
        throw std::invalid_argument{"unknown render method"};
    }
    if (job.method == ALBEDO_WAVEFRONT && job.estimator != ALBEDO_PATH) {
        throw Unsupported{"the wavefront renderer implements the path estimator only"};
    }
    if (job.accumulation != ALBEDO_ACCUMULATE_FP64 && job.accumulation != ALBEDO_ACCUMULATE_KAHAN_FP32) {
        throw std::invalid_argument{"unknown accumulation"};
    }
    if (job.accumulation == ALBEDO_ACCUMULATE_KAHAN_FP32 &&
        (job.method != ALBEDO_MEGAKERNEL || job.estimator != ALBEDO_PATH)) {
        throw Unsupported{"compensated FP32 accumulation is implemented for the megakernel's path estimator only"};
    }
    RenderArgs args{};
    args.width = job.width;
    args.height = job.height;
    args.samples_per_axis = job.samples_per_axis;
    args.estimator = job.estimator;
    args.seed = job.seed;
    args.max_depth = job.max_depth;
    args.roulette_start = job.roulette_start;
    args.tile_width = scene.mega_tile_width;
    args.blocks_per_sm = scene.mega_blocks_per_sm;
    args.accumulation = job.accumulation;
    // The inlined-traversal kernel exists for the path estimator; the other
    // estimators keep the out-of-line traversal (images do not depend on it).
    args.inline_traversal = job.estimator == ALBEDO_PATH ? scene.mega_inline : 0;
    return args;
}

CameraSettings cameraFrom(const albedo_camera& c)
{
    const auto v = [](const double* p) { return Vec3{p[0], p[1], p[2]}; };
    return CameraSettings{v(c.look_from), v(c.look_at), v(c.up), c.vertical_fov_degrees};
}

// The device camera of a render: the request's view, else the scene's camera.
DevCamera cameraFor(const albedo_scene& scene, const albedo_render_job& job, const albedo_camera* view)
{
    if (view != nullptr) {
        return deviceCamera(cameraFrom(*view), job.width, job.height);
    }
    return deviceCamera(scene.host, job.width, job.height);
}

// The process's wavefront engine on the current device, created on first use.
constexpr int kDefaultSlots{1 << 20};
constexpr int kBatchJobCapacity{4096};
std::mutex g_engine_mutex;
std::unique_ptr<WavefrontEngine> g_engine;
int g_engine_slots{kDefaultSlots};
WfShape g_engine_shape{};
unsigned long long g_last_iterations{0};
unsigned long long g_last_rays{0};

void configureEngine(int slots, int blocks_per_sm, int iterations_per_graph)
{
    if (slots <= 0 || blocks_per_sm <= 0 || iterations_per_graph <= 0) {
        throw std::invalid_argument{"wavefront configuration values must be positive"};
    }
    const std::lock_guard lock{g_engine_mutex};
    if (g_engine && g_engine->slotCount() != slots) {
        g_engine.reset();
    }
    g_engine_slots = slots;
    g_engine_shape = WfShape{};
    g_engine_shape.blocks_per_sm = blocks_per_sm;
    g_engine_shape.iterations_per_graph = iterations_per_graph;
}

WfShape engineShape()
{
    const std::lock_guard lock{g_engine_mutex};
    return g_engine_shape;
}

unsigned long long lastEngineIterations()
{
    const std::lock_guard lock{g_engine_mutex};
    return g_last_iterations;
}

WfJob wavefrontJob(const albedo_scene& scene, const albedo_render_job& job, PixelAccum* accum,
                   const albedo_camera* view = nullptr)
{
    albedo_render_job wf{job};
    wf.method = ALBEDO_WAVEFRONT;
    static_cast<void>(renderArgsFor(scene, wf));
    WfJob j{};
    j.scene = scene.dev;
    j.camera = cameraFor(scene, job, view);
    j.accum = accum;
    j.width = job.width;
    j.height = job.height;
    j.samples_per_axis = job.samples_per_axis;
    j.max_depth = job.max_depth;
    j.roulette_start = job.roulette_start;
    j.seed = job.seed;
    for (int k{0}; k < 4; ++k) {
        j.grid[k] = scene.grid[k];
    }
    return j;
}

void runWavefront(const std::vector<WfJob>& jobs, int stack, unsigned int* error_flag, cudaStream_t stream)
{
    const std::lock_guard lock{g_engine_mutex};
    try {
        if (!g_engine) {
            g_engine = std::make_unique<WavefrontEngine>(g_engine_slots, kBatchJobCapacity);
        }
        g_engine->setShape(g_engine_shape);
        g_engine->render(jobs, stack, error_flag, stream);
        g_last_iterations = g_engine->lastIterations();
        g_last_rays = g_engine->lastRays();
    } catch (const std::bad_alloc&) {
        throw;
    } catch (const std::invalid_argument&) {
        throw;
    } catch (const std::exception& e) {
        throw DeviceError{e.what()};
    }
}

} // namespace

// A request server: continuous batching over one wavefront engine, with
// admission against a device-memory budget.
struct albedo_server {
    struct Request {
        std::int64_t ticket{};
        const albedo_scene* scene{};
        WfJob job{};
        RenderArgs megakernel_args{}; // the same render as a megakernel launch (express route)
        std::int64_t bytes{};
    };
    // A request on the express route: rendered by the megakernel on the
    // server's own stream, done when its event completes.
    struct Express {
        std::int64_t ticket{};
        const albedo_scene* scene{};
        std::int64_t bytes{};
        cudaEvent_t done{nullptr};
    };
    static constexpr std::size_t kMaxExpress{8};
    // The wavefront batch counts as lightly loaded below this many pixels in flight.
    static constexpr std::int64_t kLightPixels{std::int64_t{1} << 18};

    std::unique_ptr<WavefrontEngine> engine;
    // The engine's traversal error flag: the server's own, since requests of
    // any scene share the engine and scenes may be released and destroyed.
    DeviceBuffer error_flag;
    std::int64_t budget{0};
    std::int64_t used{0};
    int stack{32};
    std::int64_t next_ticket{1};
    std::deque<Request> waiting;
    std::map<int, Request> running; // engine job index -> request
    std::set<const albedo_scene*> resident;
    std::deque<std::int64_t> finished; // tickets not yet handed to the caller
    std::vector<Express> express;      // in launch order
    cudaStream_t express_stream{nullptr};
    std::int64_t express_max_pixels{65536};
    std::int64_t routed_batch{0};   // requests admitted to the batch so far
    std::int64_t routed_express{0}; // requests admitted to the express route so far

    albedo_server() = default;
    albedo_server(const albedo_server&) = delete;
    albedo_server& operator=(const albedo_server&) = delete;
    ~albedo_server()
    {
        if (express_stream != nullptr) {
            cudaStreamSynchronize(express_stream);
            for (const Express& e : express) {
                cudaEventDestroy(e.done);
            }
            cudaStreamDestroy(express_stream);
        }
    }

    std::int64_t wavefrontPixels() const
    {
        std::int64_t pixels{0};
        for (const auto& [index, request] : running) {
            pixels += request.bytes / static_cast<std::int64_t>(sizeof(PixelAccum));
        }
        return pixels;
    }

    // A small request goes to the megakernel when the batch is lightly loaded,
    // or when it cannot join the batch now (it needs a deeper traversal stack
    // or the job table is full, so it would wait for the batch to drain): its
    // pixels' samples run in sequence either way, and the megakernel runs them
    // in one launch where the wavefront needs an iteration per bounce.
    bool takesExpress(const Request& r) const
    {
        const std::int64_t pixels{r.bytes / static_cast<std::int64_t>(sizeof(PixelAccum))};
        if (express_max_pixels <= 0 || pixels > express_max_pixels || express.size() >= kMaxExpress) {
            return false;
        }
        const bool batch_blocked{engine->isOpen() && !running.empty() &&
                                 (r.scene->stack_capacity > stack || submitted_in_batch >= engine->jobCapacity())};
        return batch_blocked || wavefrontPixels() < kLightPixels;
    }

    // Collects finished express renders in order; with `wait_oldest` it first
    // waits for the oldest.
    void pollExpress(bool wait_oldest)
    {
        for (auto it{express.begin()}; it != express.end();) {
            const cudaError_t e{wait_oldest && it == express.begin() ? cudaEventSynchronize(it->done)
                                                                     : cudaEventQuery(it->done)};
            if (e == cudaErrorNotReady) {
                ++it;
                continue;
            }
            check(e, "express render");
            finished.push_back(it->ticket);
            used -= it->bytes;
            cudaEventDestroy(it->done);
            it = express.erase(it);
        }
    }

    std::int64_t sceneBytes(const albedo_scene* scene) const
    {
        return resident.contains(scene) ? 0 : static_cast<std::int64_t>(scene->deviceBytes());
    }

    // Admits waiting requests in arrival order while they fit the budget.
    void admit()
    {
        while (!waiting.empty()) {
            Request& head{waiting.front()};
            const std::int64_t need{head.bytes + sceneBytes(head.scene)};
            if (used + need > budget) {
                return;
            }
            if (takesExpress(head)) {
                check(launchMegakernel(head.scene->dev, head.job.camera, head.megakernel_args, head.job.accum,
                                       error_flag.as<unsigned int>(), head.scene->stack_capacity, express_stream),
                      "express render");
                cudaEvent_t done{nullptr};
                check(cudaEventCreateWithFlags(&done, cudaEventDisableTiming), "express event");
                const cudaError_t recorded{cudaEventRecord(done, express_stream)};
                if (recorded != cudaSuccess) {
                    cudaEventDestroy(done);
                    check(recorded, "express event");
                }
                express.push_back({head.ticket, head.scene, head.bytes, done});
                ++routed_express;
                used += need;
                resident.insert(head.scene);
                waiting.pop_front();
                continue;
            }
            const int head_stack{head.scene->stack_capacity};
            const bool table_full{submitted_in_batch >= engine->jobCapacity()};
            if (engine->isOpen() && (head_stack > stack || table_full)) {
                if (!running.empty()) {
                    return; // wait for the batch to drain, then reopen
                }
                engine->close();
            }
            if (!engine->isOpen()) {
                stack = std::max(stack, head_stack);
                engine->open(stack, error_flag.as<unsigned int>());
                submitted_in_batch = 0;
            }
            used += need;
            resident.insert(head.scene);
            const int index{engine->submit(head.job)};
            ++submitted_in_batch;
            ++routed_batch;
            running.emplace(index, head);
            waiting.pop_front();
        }
    }

    int submitted_in_batch{0};
};

namespace {

void renderOnDevice(const albedo_scene& scene, const albedo_render_job& job, PixelAccum* accum, cudaStream_t stream,
                    const albedo_camera* view = nullptr)
{
    const RenderArgs args{renderArgsFor(scene, job)};
    if (job.method == ALBEDO_WAVEFRONT) {
        runWavefront({wavefrontJob(scene, job, accum, view)}, scene.stack_capacity,
                     scene.error_flag.as<unsigned int>(), stream);
        return;
    }
    const DevCamera camera{cameraFor(scene, job, view)};
    check(launchMegakernel(scene.dev, camera, args, accum, scene.error_flag.as<unsigned int>(), scene.stack_capacity,
                           stream),
          "render launch");
}

} // namespace

namespace {

// Events and a stream for timing candidate shapes.
class TuneTimer {
public:
    TuneTimer()
    {
        check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "tuning stream");
        check(cudaEventCreate(&start_), "tuning event");
        check(cudaEventCreate(&stop_), "tuning event");
    }
    ~TuneTimer()
    {
        cudaStreamSynchronize(stream_);
        cudaEventDestroy(start_);
        cudaEventDestroy(stop_);
        cudaStreamDestroy(stream_);
    }
    TuneTimer(const TuneTimer&) = delete;
    TuneTimer& operator=(const TuneTimer&) = delete;

    cudaStream_t stream() const { return stream_; }

    // One untimed run, then the fastest of `repeats` timed runs, in ms.
    template <typename Run>
    double time(Run&& run, int repeats)
    {
        run();
        check(cudaStreamSynchronize(stream_), "tuning run");
        double best{std::numeric_limits<double>::infinity()};
        for (int i{0}; i < repeats; ++i) {
            check(cudaEventRecord(start_, stream_), "event record");
            run();
            check(cudaEventRecord(stop_, stream_), "event record");
            check(cudaEventSynchronize(stop_), "event sync");
            float ms{0};
            check(cudaEventElapsedTime(&ms, start_, stop_), "event time");
            best = std::min(best, static_cast<double>(ms));
        }
        return best;
    }

private:
    cudaStream_t stream_{nullptr};
    cudaEvent_t start_{nullptr};
    cudaEvent_t stop_{nullptr};
};

// The tuning work: the caller's job at a quarter of its samples.
albedo_render_job tuningJob(const albedo_render_job& job)
{
    albedo_render_job probe{job};
    probe.samples_per_axis = std::max(1, job.samples_per_axis / 2);
    return probe;
}

void fillTuning(albedo_tuning* out, const TuneOutcome& outcome)
{
    out->evaluations = outcome.evaluations;
    out->best_ms = outcome.best_ms;
    out->default_ms = outcome.start_ms;
}

} // namespace

namespace {

// A render into host accumulators through the per-device staging buffer: one
// copy in, the render, one copy out, then a synchronize. After the first call
// of a size, a host render allocates nothing (an allocation can wait on the
// driver for as long as a render takes); host renders on one device take turns
// on the buffer.
void renderThroughStaging(const albedo_scene& scene, const albedo_render_job& job, const albedo_camera* camera,
                          albedo_accumulator* accumulators)
{
    static_cast<void>(renderArgsFor(scene, job));
    const std::size_t bytes{static_cast<std::size_t>(job.width) * static_cast<std::size_t>(job.height) *
                            sizeof(PixelAccum)};
    int device{0};
    check(cudaGetDevice(&device), "cudaGetDevice");
    HostStaging& staging{hostStaging(device)};
    const std::lock_guard lock{staging.mutex};
    if (staging.buffer.bytes < bytes) {
        staging.buffer = DeviceBuffer{};
        staging.buffer = DeviceBuffer{bytes};
    }
    check(cudaMemcpyAsync(staging.buffer.ptr, accumulators, bytes, cudaMemcpyHostToDevice, nullptr), "upload");
    renderOnDevice(scene, job, staging.buffer.as<PixelAccum>(), nullptr, camera);
    check(cudaMemcpyAsync(accumulators, staging.buffer.ptr, bytes, cudaMemcpyDeviceToHost, nullptr), "download");
    check(cudaStreamSynchronize(nullptr), "render");
    scene.collectKernelError();
}

} // namespace

extern "C" {

const char* albedo_last_error(void) { return g_last_error.c_str(); }

int albedo_scene_read(const char* path, albedo_scene** out)
{
    *out = nullptr;
    return guarded([&] {
        auto scene{std::make_unique<albedo_scene>()};
        scene->host = readSceneFile(path);
        scene->prepare();
        *out = scene.release();
    });
}

const void* albedo_scene_host_view(const albedo_scene* scene) { return &scene->host; }

int albedo_scene_create(albedo_scene** out)
{
    return guarded([&] { *out = new albedo_scene{}; });
}

int albedo_scene_load(const char* path, albedo_scene** out)
{
    *out = nullptr;
    return guarded([&] {
        auto scene{std::make_unique<albedo_scene>()};
        scene->host = readSceneFile(path);
        scene->commit();
        *out = scene.release();
    });
}

void albedo_scene_destroy(albedo_scene* scene) { delete scene; }

int albedo_scene_set_camera(albedo_scene* scene, const double look_from[3], const double look_at[3],
                            const double up[3], double vertical_fov_degrees)
{
    return guarded([&] {
        scene->requireOpen();
        CameraSettings settings{vec(look_from), vec(look_at), vec(up), vertical_fov_degrees};
        static_cast<void>(buildCameraFrame(settings, 16.0 / 9.0));
        scene->host.camera = settings;
        scene->host.has_camera = true;
    });
}

int albedo_scene_add_material(albedo_scene* scene, const albedo_material* material, uint32_t* out_material)
{
    return guarded([&] {
        scene->requireOpen();
        MaterialDesc m;
        m.mix = material->mix != 0;
        m.first = basicFrom(material->first);
        m.second = m.mix ? basicFrom(material->second) : m.first;
        m.scale = material->scale;
        m.veins = material->veins;
        m.threshold = material->threshold;
        const std::uint32_t id{scene->host.addMaterial(m)};
        if (out_material != nullptr) {
            *out_material = id;
        }
    });
}

namespace {
void requireMaterial(const albedo_scene* scene, uint32_t material)
{
    if (material >= scene->host.materials.size()) {
        throw std::invalid_argument{std::format("material {} is not defined", material)};
    }
}
} // namespace

int albedo_scene_add_sphere(albedo_scene* scene, const double center[3], double radius, uint32_t material,
                            uint32_t* out_object)
{
    return guarded([&] {
        scene->requireOpen();
        requireMaterial(scene, material);
        const std::uint32_t id{scene->host.addSphere(vec(center), radius, material)};
        if (out_object != nullptr) {
            *out_object = id;
        }
    });
}

int albedo_scene_add_area_light(albedo_scene* scene, const double center[3], double radius, const double radiance[3],
                                uint32_t material, uint32_t* out_object)
{
    return guarded([&] {
        scene->requireOpen();
        requireMaterial(scene, material);
        const std::uint32_t id{scene->host.addAreaLight(vec(center), radius, rgb(radiance), material)};
        if (out_object != nullptr) {
            *out_object = id;
        }
    });
}

int albedo_scene_add_point_light(albedo_scene* scene, const double position[3], const double intensity[3])
{
    return guarded([&] {
        scene->requireOpen();
        scene->host.addPointLight(vec(position), rgb(intensity));
    });
}

int albedo_scene_set_sky(albedo_scene* scene, const double nadir[3], const double zenith[3])
{
    return guarded([&] {
        scene->requireOpen();
        scene->host.setSky(rgb(nadir), rgb(zenith));
    });
}

namespace {
std::vector<Vec3> positionsFrom(const double* positions, int64_t count)
{
    std::vector<Vec3> out(static_cast<std::size_t>(count));
    for (int64_t i{0}; i < count; ++i) {
        out[static_cast<std::size_t>(i)] = vec(positions + 3 * i);
    }
    return out;
}
std::vector<std::array<std::uint32_t, 3>> facesFrom(const uint32_t* faces, int64_t count)
{
    std::vector<std::array<std::uint32_t, 3>> out(static_cast<std::size_t>(count));
    for (int64_t i{0}; i < count; ++i) {
        out[static_cast<std::size_t>(i)] = {faces[3 * i], faces[3 * i + 1], faces[3 * i + 2]};
    }
    return out;
}
} // namespace

int albedo_scene_add_mesh(albedo_scene* scene, const double* positions, int64_t position_count, const uint32_t* faces,
                          int64_t face_count, const double* texture_coordinates, int64_t texture_coordinate_count,
                          const uint32_t* texture_faces, int64_t texture_face_count, int32_t smooth, uint32_t* out_mesh)
{
    return guarded([&] {
        scene->requireOpen();
        std::vector<std::array<double, 2>> uvs(static_cast<std::size_t>(texture_coordinate_count));
        for (int64_t i{0}; i < texture_coordinate_count; ++i) {
            uvs[static_cast<std::size_t>(i)] = {texture_coordinates[2 * i], texture_coordinates[2 * i + 1]};
        }
        const std::uint32_t id{scene->host.addMesh(positionsFrom(positions, position_count),
                                                   facesFrom(faces, face_count), uvs,
                                                   facesFrom(texture_faces, texture_face_count), smooth != 0)};
        if (out_mesh != nullptr) {
            *out_mesh = id;
        }
    });
}

int albedo_scene_add_instance(albedo_scene* scene, uint32_t mesh, const double to_world[12],
                              const double to_object[12], uint32_t material, uint32_t* out_object)
{
    return guarded([&] {
        scene->requireOpen();
        requireMaterial(scene, material);
        Affine forward;
        Affine backward;
        for (int row{0}; row < 3; ++row) {
            for (int col{0}; col < 3; ++col) {
                forward.linear[row][col] = to_world[4 * row + col];
                backward.linear[row][col] = to_object[4 * row + col];
            }
        }
        forward.offset = {to_world[3], to_world[7], to_world[11]};
        backward.offset = {to_object[3], to_object[7], to_object[11]};
        const std::uint32_t id{
            scene->host.addInstance(mesh, Transform::fromMaps(forward, backward), material)};
        if (out_object != nullptr) {
            *out_object = id;
        }
    });
}

int albedo_scene_add_triangles(albedo_scene* scene, const double* positions, int64_t position_count,
                               const uint32_t* faces, int64_t face_count, uint32_t material)
{
    return guarded([&] {
        scene->requireOpen();
        requireMaterial(scene, material);
        scene->host.addTriangles(positionsFrom(positions, position_count), facesFrom(faces, face_count), {}, {},
                                 material);
    });
}

int albedo_scene_prepare(albedo_scene* scene)
{
    return guarded([&] { scene->prepare(); });
}

int albedo_scene_commit(albedo_scene* scene)
{
    return guarded([&] {
        if (scene->committed) {
            throw std::invalid_argument{"the scene is already committed"};
        }
        scene->prepare();
        scene->commitPrepared();
    });
}

int albedo_scene_get_info(const albedo_scene* scene, albedo_scene_info* out)
{
    return guarded([&] {
        if (!scene->prepared) {
            throw std::invalid_argument{"the scene has not been prepared"};
        }
        out->objects = static_cast<int64_t>(scene->host.objects.size());
        out->lights = static_cast<int64_t>(scene->host.lights.size());
        out->triangles = static_cast<int64_t>(scene->image.triangles.size());
        out->nodes = static_cast<int64_t>(scene->image.nodes.size());
        out->device_bytes = static_cast<int64_t>(scene->deviceBytes());
        out->stack_need = static_cast<int32_t>(scene->image.stack_need);
        out->stack_capacity = scene->stack_capacity;
    });
}

int albedo_render(const albedo_scene* scene, const albedo_render_job* job, albedo_accumulator* accumulators,
                  void* stream)
{
    return guarded([&] {
        renderOnDevice(*scene, *job, reinterpret_cast<PixelAccum*>(accumulators), static_cast<cudaStream_t>(stream));
    });
}

int albedo_render_view(const albedo_scene* scene, const albedo_render_job* job, const albedo_camera* camera,
                       albedo_accumulator* accumulators, void* stream)
{
    return guarded([&] {
        renderOnDevice(*scene, *job, reinterpret_cast<PixelAccum*>(accumulators), static_cast<cudaStream_t>(stream),
                       camera);
    });
}

int albedo_render_host(const albedo_scene* scene, const albedo_render_job* job, albedo_accumulator* accumulators)
{
    return guarded([&] { renderThroughStaging(*scene, *job, nullptr, accumulators); });
}

int albedo_render_view_host(const albedo_scene* scene, const albedo_render_job* job, const albedo_camera* camera,
                            albedo_accumulator* accumulators)
{
    return guarded([&] { renderThroughStaging(*scene, *job, camera, accumulators); });
}

int albedo_render_batch(const albedo_batch_item* items, int32_t count, void* stream)
{
    return guarded([&] {
        if (count <= 0) {
            throw std::invalid_argument{"a batch needs at least one job"};
        }
        std::vector<WfJob> jobs;
        jobs.reserve(static_cast<std::size_t>(count));
        int stack{32};
        for (int32_t i{0}; i < count; ++i) {
            const albedo_batch_item& item{items[i]};
            jobs.push_back(wavefrontJob(*item.scene, item.job, reinterpret_cast<PixelAccum*>(item.accumulators)));
            stack = std::max(stack, item.scene->stack_capacity);
        }
        // The batch reports a traversal error through its first job's scene.
        runWavefront(jobs, stack, items[0].scene->error_flag.as<unsigned int>(), static_cast<cudaStream_t>(stream));
        items[0].scene->collectKernelError();
    });
}

int albedo_render_noalloc(const albedo_scene* scene, const albedo_render_job* job, albedo_accumulator* accumulators,
                          void* stream)
{
    return guarded([&] {
        const long long pixels{static_cast<long long>(job->width) * static_cast<long long>(job->height)};
        if (job->width > 0 && job->height > 0 && pixels > noAllocMaxPixels()) {
            throw std::invalid_argument{std::format(
                "albedo_render_noalloc renders images of at most {} pixels (one path slot per pixel in its static "
                "scratch); {}x{} has {}",
                noAllocMaxPixels(), job->width, job->height, pixels)};
        }
        const WfJob wf{wavefrontJob(*scene, *job, reinterpret_cast<PixelAccum*>(accumulators))};
        int device{0};
        int sms{0};
        check(cudaGetDevice(&device), "cudaGetDevice");
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
        const cudaError_t e{renderNoAlloc(wf, scene->stack_capacity, 4 * sms, scene->error_flag.as<unsigned int>(),
                                          static_cast<cudaStream_t>(stream))};
        if (e == cudaErrorLaunchTimeout) {
            throw DeviceError{"albedo_render_noalloc exceeded its iteration bound before the image was complete"};
        }
        check(e, "albedo_render_noalloc");
        // The render is complete on the stream: report a kernel-side error
        // (a traversal stack overflow) now, as the host-buffer render does.
        scene->collectKernelError();
    });
}

namespace {

// PixelBuffer's size check (image/pixel_buffer.hpp:30-38) for the film output calls.
std::size_t filmPixels(int32_t width, int32_t height)
{
    if (width <= 0 || height <= 0 ||
        static_cast<std::uint64_t>(width) > (std::uint64_t{1} << 28) / static_cast<std::uint64_t>(height)) {
        throw std::invalid_argument{
            std::format("invalid image size {}x{}: dimensions must be positive and the image at most {} pixels",
                        width, height, std::uint64_t{1} << 28)};
    }
    return static_cast<std::size_t>(width) * static_cast<std::size_t>(height);
}

const SrgbThresholds& deviceSrgbTable()
{
    static_assert(kResolveBucketBase == kSrgbBucketBase && kResolveBuckets == kSrgbBuckets &&
                  kResolveBucketShift == 52 - kSrgbBucketBits);
    static const SrgbThresholds table{[] {
        SrgbThresholds t{};
        std::copy(srgbTable().lower.begin(), srgbTable().lower.end(), t.lower);
        std::copy(srgbTable().start.begin(), srgbTable().start.end(), t.start);
        return t;
    }()};
    return table;
}

void resolveOnDevice(const albedo_accumulator* accumulators, std::size_t pixels, uint8_t* out_rgb,
                     cudaStream_t stream)
{
    if (accumulators == nullptr || out_rgb == nullptr) {
        throw std::invalid_argument{"null accumulator or output pointer"};
    }
    if ((reinterpret_cast<std::uintptr_t>(accumulators) & 7) != 0) {
        throw std::invalid_argument{"accumulators must be 8-byte aligned"};
    }
    check(launchResolveSrgb(reinterpret_cast<const PixelAccum*>(accumulators), static_cast<long long>(pixels),
                            out_rgb, deviceSrgbTable(), stream),
          "albedo_resolve_srgb");
}

// Resolves device accumulators into a temporary device buffer, reads the bytes
// back and writes the file.
void savePpm(const char* path, const albedo_accumulator* device_accumulators, int32_t width, int32_t height,
             cudaStream_t stream)
{
    if (path == nullptr) {
        throw std::invalid_argument{"null path"};
    }
    const std::size_t pixels{filmPixels(width, height)};
    DeviceBuffer bytes{3 * pixels};
    resolveOnDevice(device_accumulators, pixels, bytes.as<uint8_t>(), stream);
    std::vector<uint8_t> rgb(3 * pixels);
    check(cudaMemcpyAsync(rgb.data(), bytes.ptr, rgb.size(), cudaMemcpyDeviceToHost, stream), "download");
    check(cudaStreamSynchronize(stream), "albedo_resolve_srgb");
    writePpm(path, rgb.data(), width, height);
}

} // namespace

int albedo_resolve_srgb(const albedo_accumulator* accumulators, int32_t width, int32_t height, uint8_t* out_rgb,
                        void* stream)
{
    return guarded([&] {
        resolveOnDevice(accumulators, filmPixels(width, height), out_rgb, static_cast<cudaStream_t>(stream));
    });
}

int albedo_srgb_tables(double* out_lower, uint8_t* out_start)
{
    return guarded([&] {
        if (out_lower == nullptr) {
            throw std::invalid_argument{"null output pointer"};
        }
        std::copy(srgbTable().lower.begin(), srgbTable().lower.end(), out_lower);
        if (out_start != nullptr) {
            std::copy(srgbTable().start.begin(), srgbTable().start.end(), out_start);
        }
    });
}

int albedo_write_ppm(const char* path, const uint8_t* rgb, int32_t width, int32_t height)
{
    return guarded([&] {
        if (path == nullptr || rgb == nullptr) {
            throw std::invalid_argument{"null path or pixel pointer"};
        }
        writePpm(path, rgb, width, height);
    });
}

int albedo_save_ppm(const char* path, const albedo_accumulator* accumulators, int32_t width, int32_t height,
                    void* stream)
{
    return guarded([&] { savePpm(path, accumulators, width, height, static_cast<cudaStream_t>(stream)); });
}

int albedo_save_ppm_host(const char* path, const albedo_accumulator* accumulators, int32_t width, int32_t height)
{
    return guarded([&] {
        const std::size_t bytes{filmPixels(width, height) * sizeof(PixelAccum)};
        if (accumulators == nullptr) {
            throw std::invalid_argument{"null accumulator pointer"};
        }
        int device{0};
        check(cudaGetDevice(&device), "cudaGetDevice");
        HostStaging& staging{hostStaging(device)};
        const std::lock_guard lock{staging.mutex};
        if (staging.buffer.bytes < bytes) {
            staging.buffer = DeviceBuffer{};
            staging.buffer = DeviceBuffer{bytes};
        }
        check(cudaMemcpyAsync(staging.buffer.ptr, accumulators, bytes, cudaMemcpyHostToDevice, nullptr), "upload");
        savePpm(path, staging.buffer.as<albedo_accumulator>(), width, height, nullptr);
    });
}

int albedo_wavefront_configure(int32_t slot_count, int32_t blocks_per_sm, int32_t iterations_per_graph)
{
    return guarded([&] { configureEngine(slot_count, blocks_per_sm, iterations_per_graph); });
}

int albedo_autotune_megakernel(albedo_scene* scene, const albedo_render_job* job, albedo_tuning* out)
{
    return guarded([&] {
        *out = albedo_tuning{};
        albedo_render_job probe{tuningJob(*job)};
        probe.method = ALBEDO_MEGAKERNEL;
        static_cast<void>(renderArgsFor(*scene, probe));
        const std::size_t pixels{static_cast<std::size_t>(probe.width) * static_cast<std::size_t>(probe.height)};
        DeviceBuffer scratch{pixels * sizeof(PixelAccum)};
        TuneTimer timer;
        // Kernel variants: 0 = 3 blocks/SM, 1 = 4 blocks/SM (both with the
        // out-of-line traversal), 2 = 3 blocks/SM with both queries' traversal
        // inlined, 3 = 3 blocks/SM with the closest-hit traversal inlined and
        // the shadow query out of line, 4 = 4 blocks/SM with both inlined
        // (path estimator only). The 4-blocks/SM kernels of the path estimator
        // keep the path's state in shared memory.
        const bool can_inline{probe.estimator == ALBEDO_PATH};
        const std::vector<TuneKnob> knobs{
            {"tile_width", {8, 16, 32}},
            {"variant", can_inline ? std::vector<int>{0, 1, 2, 3, 4} : std::vector<int>{0, 1}}};
        const int kept_tile{scene->mega_tile_width};
        const int kept_blocks{scene->mega_blocks_per_sm};
        const int kept_inline{scene->mega_inline};
        const auto apply = [&](const std::vector<int>& v) {
            scene->mega_tile_width = v[0];
            scene->mega_blocks_per_sm = v[1] == 1 || v[1] == 4 ? 4 : 3;
            scene->mega_inline = v[1] == 2 || v[1] == 4 ? 1 : (v[1] == 3 ? 2 : 0);
        };
        TuneOutcome outcome;
        try {
            outcome = tuneExhaustive(knobs, {16, 0}, [&](const std::vector<int>& v) {
                apply(v);
                return timer.time([&] { renderOnDevice(*scene, probe, scratch.as<PixelAccum>(), timer.stream()); },
                                  2);
            });
        } catch (...) {
            scene->mega_tile_width = kept_tile;
            scene->mega_blocks_per_sm = kept_blocks;
            scene->mega_inline = kept_inline;
            throw;
        }
        apply(outcome.best);
        scene->collectKernelError();
        out->tile_width = scene->mega_tile_width;
        out->blocks_per_sm = scene->mega_blocks_per_sm;
        out->inline_traversal = scene->mega_inline;
        fillTuning(out, outcome);
    });
}

int albedo_autotune_batch(const albedo_batch_item* items, int32_t count, albedo_tuning* out)
{
    return guarded([&] {
        *out = albedo_tuning{};
        if (count <= 0) {
            throw std::invalid_argument{"tuning needs at least one job"};
        }
        std::size_t pixels{0};
        int stack{32};
        for (int32_t i{0}; i < count; ++i) {
            const albedo_render_job probe{tuningJob(items[i].job)};
            static_cast<void>(wavefrontJob(*items[i].scene, probe, nullptr));
            pixels += static_cast<std::size_t>(probe.width) * static_cast<std::size_t>(probe.height);
            stack = std::max(stack, items[i].scene->stack_capacity);
        }
        DeviceBuffer scratch{pixels * sizeof(PixelAccum)};
        std::vector<WfJob> jobs;
        std::size_t offset{0};
        for (int32_t i{0}; i < count; ++i) {
            const albedo_render_job probe{tuningJob(items[i].job)};
            jobs.push_back(wavefrontJob(*items[i].scene, probe, scratch.as<PixelAccum>() + offset));
            offset += static_cast<std::size_t>(probe.width) * static_cast<std::size_t>(probe.height);
        }
        unsigned int* error_flag{items[0].scene->error_flag.as<unsigned int>()};
        TuneTimer timer;
        const std::vector<TuneKnob> knobs{{"trace_blocks_per_sm", {3, 4, 5}},
                                          {"fetch_batch", {16, 32, 64, 128}},
                                          {"trace_loop", {0, 1, 2}},
                                          {"blocks_per_sm", {4, 8, 16}},
                                          {"iterations_per_graph", {2, 4, 8}},
                                          {"slot_count", {1 << 17, 1 << 18, 1 << 19, 1 << 20, 1 << 21, 1 << 22}},
                                          {"ray_sort", {0, 1, 2}}};
        const WfShape kept_shape{engineShape()};
        int kept_slots{0};
        {
            const std::lock_guard lock{g_engine_mutex};
            kept_slots = g_engine_slots;
        }
        const auto apply = [](const std::vector<int>& v) {
            WfShape shape{};
            shape.trace_blocks_per_sm = v[0];
            shape.fetch_batch = v[1];
            shape.trace_loop = v[2];
            shape.blocks_per_sm = v[3];
            shape.iterations_per_graph = v[4];
            shape.ray_sort = v[6];
            const std::lock_guard lock{g_engine_mutex};
            if (g_engine && g_engine->slotCount() != v[5]) {
                g_engine.reset();
            }
            g_engine_slots = v[5];
            g_engine_shape = shape;
        };
        const std::vector<int> start{kept_shape.trace_blocks_per_sm > 0 ? kept_shape.trace_blocks_per_sm : 5,
                                     kept_shape.fetch_batch, kept_shape.trace_loop, kept_shape.blocks_per_sm,
                                     kept_shape.iterations_per_graph, kept_slots, kept_shape.ray_sort};
        TuneOutcome outcome;
        try {
            outcome = tuneCoordinateDescent(knobs, start, [&](const std::vector<int>& v) {
                apply(v);
                return timer.time([&] { runWavefront(jobs, stack, error_flag, timer.stream()); }, 2);
            }, 1);
        } catch (...) {
            apply(start);
            throw;
        }
        apply(outcome.best);
        for (int32_t i{0}; i < count; ++i) {
            items[i].scene->collectKernelError();
        }
        out->trace_blocks_per_sm = outcome.best[0];
        out->fetch_batch = outcome.best[1];
        out->trace_loop = outcome.best[2];
        out->blocks_per_sm = outcome.best[3];
        out->iterations_per_graph = outcome.best[4];
        out->slot_count = outcome.best[5];
        out->ray_sort = outcome.best[6];
        fillTuning(out, outcome);
    });
}

int albedo_tuning_set(albedo_scene* scene, const albedo_tuning* shape)
{
    return guarded([&] {
        if (scene != nullptr) {
            if (shape->tile_width != 8 && shape->tile_width != 16 && shape->tile_width != 32) {
                throw std::invalid_argument{std::format("megakernel tile width must be 8, 16 or 32, got {}",
                                                        shape->tile_width)};
            }
            if (shape->blocks_per_sm != 3 && shape->blocks_per_sm != 4) {
                throw std::invalid_argument{std::format("megakernel blocks per SM must be 3 or 4, got {}",
                                                        shape->blocks_per_sm)};
            }
            if (shape->inline_traversal < 0 || shape->inline_traversal > 2 ||
                (shape->inline_traversal == 2 && shape->blocks_per_sm != 3)) {
                throw std::invalid_argument{"megakernel traversal placement must be 0 (out of line), 1 (inlined) or "
                                            "2 (closest hit inlined, 3 blocks per SM only)"};
            }
            scene->mega_tile_width = shape->tile_width;
            scene->mega_blocks_per_sm = shape->blocks_per_sm;
            scene->mega_inline = shape->inline_traversal;
            return;
        }
        if (shape->blocks_per_sm <= 0 || shape->trace_blocks_per_sm <= 0 || shape->fetch_batch <= 0 ||
            shape->iterations_per_graph <= 0 || shape->slot_count <= 0) {
            throw std::invalid_argument{"wavefront shape values must be positive"};
        }
        if (shape->trace_loop < 0 || shape->trace_loop > 2) {
            throw std::invalid_argument{"the traversal turn shape must be 0, 1 or 2"};
        }
        if (shape->ray_sort < 0 || shape->ray_sort > 2) {
            throw std::invalid_argument{"ray binning must be 0, 1 or 2"};
        }
        WfShape next{};
        next.blocks_per_sm = shape->blocks_per_sm;
        next.trace_blocks_per_sm = shape->trace_blocks_per_sm;
        next.fetch_batch = shape->fetch_batch;
        next.trace_loop = shape->trace_loop;
        next.ray_sort = shape->ray_sort;
        next.iterations_per_graph = shape->iterations_per_graph;
        const std::lock_guard lock{g_engine_mutex};
        if (g_engine && g_engine->slotCount() != shape->slot_count) {
            g_engine.reset();
        }
        g_engine_slots = shape->slot_count;
        g_engine_shape = next;
    });
}

int albedo_tuning_get(const albedo_scene* scene, albedo_tuning* out)
{
    return guarded([&] {
        *out = albedo_tuning{};
        if (scene != nullptr) {
            out->tile_width = scene->mega_tile_width > 0 ? scene->mega_tile_width : 16;
            out->blocks_per_sm = scene->mega_blocks_per_sm > 0 ? scene->mega_blocks_per_sm : 3;
            out->inline_traversal = scene->mega_inline;
            return;
        }
        const std::lock_guard lock{g_engine_mutex};
        out->trace_blocks_per_sm = g_engine_shape.trace_blocks_per_sm;
        out->fetch_batch = g_engine_shape.fetch_batch;
        out->trace_loop = g_engine_shape.trace_loop;
        out->ray_sort = g_engine_shape.ray_sort;
        out->blocks_per_sm = g_engine_shape.blocks_per_sm;
        out->iterations_per_graph = g_engine_shape.iterations_per_graph;
        out->slot_count = g_engine_slots;
    });
}

int albedo_server_create(int64_t memory_budget_bytes, int32_t slot_count, albedo_server** out)
{
    *out = nullptr;
    return guarded([&] {
        if (memory_budget_bytes <= 0 || slot_count <= 0) {
            throw std::invalid_argument{"the server needs a positive memory budget and slot count"};
        }
        auto server{std::make_unique<albedo_server>()};
        try {
            server->engine = std::make_unique<WavefrontEngine>(slot_count, kBatchJobCapacity);
            server->engine->setShape(engineShape());
            server->error_flag = DeviceBuffer{sizeof(unsigned int)};
            check(cudaMemset(server->error_flag.ptr, 0, sizeof(unsigned int)), "cudaMemset");
            check(cudaStreamCreateWithFlags(&server->express_stream, cudaStreamNonBlocking), "express stream");
        } catch (const std::bad_alloc&) {
            throw;
        } catch (const std::exception& e) {
            throw DeviceError{e.what()};
        }
        server->budget = memory_budget_bytes;
        server->used = static_cast<std::int64_t>(server->engine->deviceBytes());
        if (server->used > server->budget) {
            throw std::invalid_argument{std::format("the server's path slots alone ({} bytes) exceed the budget",
                                                    server->used)};
        }
        *out = server.release();
    });
}

int albedo_server_submit(albedo_server* server, const albedo_scene* scene, const albedo_render_job* job,
                         albedo_accumulator* accumulators, int64_t* out_ticket)
{
    return albedo_server_submit_view(server, scene, job, nullptr, accumulators, out_ticket);
}

int albedo_server_submit_view(albedo_server* server, const albedo_scene* scene, const albedo_render_job* job,
                              const albedo_camera* camera, albedo_accumulator* accumulators, int64_t* out_ticket)
{
    return guarded([&] {
        albedo_server::Request request;
        request.job = wavefrontJob(*scene, *job, reinterpret_cast<PixelAccum*>(accumulators), camera);
        albedo_render_job as_megakernel{*job};
        as_megakernel.method = ALBEDO_MEGAKERNEL;
        as_megakernel.accumulation = ALBEDO_ACCUMULATE_FP64;
        request.megakernel_args = renderArgsFor(*scene, as_megakernel);
        request.ticket = server->next_ticket++;
        request.scene = scene;
        request.bytes = static_cast<std::int64_t>(job->width) * job->height * static_cast<std::int64_t>(sizeof(PixelAccum));
        const std::int64_t fixed{static_cast<std::int64_t>(server->engine->deviceBytes())};
        if (fixed + request.bytes + static_cast<std::int64_t>(scene->deviceBytes()) > server->budget) {
            throw std::invalid_argument{"the request alone exceeds the server's memory budget"};
        }
        server->waiting.push_back(request);
        try {
            server->admit();
        } catch (const std::invalid_argument&) {
            throw;
        } catch (const std::bad_alloc&) {
            throw;
        } catch (const std::exception& e) {
            throw DeviceError{e.what()};
        }
        *out_ticket = request.ticket;
    });
}

int albedo_server_step(albedo_server* server, int64_t* finished, int32_t capacity, int32_t* out_finished)
{
    return guarded([&] {
        *out_finished = 0;
        const auto report = [&] {
            while (!server->finished.empty() && *out_finished < capacity) {
                finished[(*out_finished)++] = server->finished.front();
                server->finished.pop_front();
            }
        };
        try {
            server->admit();
            const bool batch_busy{server->engine->isOpen() && !server->running.empty()};
            // With no batch to advance, wait for the oldest express render.
            server->pollExpress(!batch_busy && !server->express.empty());
            if (!batch_busy) {
                server->admit();
                report();
                return;
            }
            server->engine->step();
            for (const int index : server->engine->poll()) {
                const auto found{server->running.find(index)};
                if (found == server->running.end()) {
                    continue;
                }
                server->finished.push_back(found->second.ticket);
                server->used -= found->second.bytes;
                server->running.erase(found);
            }
            server->pollExpress(false);
            server->admit();
            report();
        } catch (const std::invalid_argument&) {
            throw;
        } catch (const std::bad_alloc&) {
            throw;
        } catch (const std::exception& e) {
            throw DeviceError{e.what()};
        }
        // A traversal stack overflow in any request (none can happen with the
        // stack the engine sizes for its scenes) is reported, once, here.
        unsigned int flag{0};
        check(cudaMemcpy(&flag, server->error_flag.ptr, sizeof(flag), cudaMemcpyDeviceToHost), "error flag");
        if (flag != 0) {
            check(cudaMemset(server->error_flag.ptr, 0, sizeof(flag)), "cudaMemset");
            throw TraversalError{"a traversal stack overflowed in a served request; the affected rays were ended"};
        }
    });
}

int albedo_server_routes(const albedo_server* server, int64_t* out_batched, int64_t* out_express)
{
    return guarded([&] {
        *out_batched = server->routed_batch;
        *out_express = server->routed_express;
    });
}

int albedo_server_set_express(albedo_server* server, int64_t max_pixels)
{
    return guarded([&] {
        if (max_pixels < 0) {
            throw std::invalid_argument{"the express route's pixel limit must not be negative"};
        }
        server->express_max_pixels = max_pixels;
    });
}

int albedo_server_release_scene(albedo_server* server, const albedo_scene* scene)
{
    return guarded([&] {
        const auto uses = [&](const albedo_server::Request& r) { return r.scene == scene; };
        if (std::any_of(server->waiting.begin(), server->waiting.end(), uses) ||
            std::any_of(server->running.begin(), server->running.end(),
                        [&](const auto& entry) { return uses(entry.second); }) ||
            std::any_of(server->express.begin(), server->express.end(),
                        [&](const albedo_server::Express& e) { return e.scene == scene; })) {
            throw std::invalid_argument{"the scene still has requests waiting or running in the server"};
        }
        if (server->resident.erase(scene) > 0) {
            server->used -= static_cast<std::int64_t>(scene->deviceBytes());
            server->admit();
        }
    });
}

int albedo_server_pending(const albedo_server* server, int32_t* out_waiting, int32_t* out_running)
{
    return guarded([&] {
        *out_waiting = static_cast<int32_t>(server->waiting.size());
        *out_running = static_cast<int32_t>(server->running.size() + server->express.size());
    });
}

void albedo_server_destroy(albedo_server* server) { delete server; }

int albedo_wavefront_last_iterations(int64_t* out)
{
    return guarded([&] { *out = static_cast<int64_t>(lastEngineIterations()); });
}

int albedo_wavefront_last_rays(int64_t* out)
{
    return guarded([&] {
        const std::lock_guard lock{g_engine_mutex};
        *out = static_cast<int64_t>(g_last_rays);
    });
}

int albedo_server_rays(const albedo_server* server, int64_t* out)
{
    return guarded([&] { *out = static_cast<int64_t>(server->engine->lastRays()); });
}

int albedo_render_pixels_host(const albedo_scene* scene, const albedo_render_job* job, const int32_t* pixels,
                              int64_t pixel_count, albedo_accumulator* accumulators, double* sum_squares)
{
    return guarded([&] {
        RenderArgs args{renderArgsFor(*scene, *job)};
        for (int64_t i{0}; i < pixel_count; ++i) {
            if (pixels[2 * i] < 0 || pixels[2 * i] >= job->width || pixels[2 * i + 1] < 0 ||
                pixels[2 * i + 1] >= job->height) {
                throw std::invalid_argument{std::format("pixel {} lies outside the image", i)};
            }
        }
        const auto count{static_cast<std::size_t>(pixel_count)};
        DeviceBuffer device_pixels{uploadRaw(pixels, 2 * count)};
        DeviceBuffer device_accum{uploadRaw(accumulators, count)};
        DeviceBuffer device_squares;
        if (sum_squares != nullptr) {
            device_squares = uploadRaw(sum_squares, 3 * count);
        }
        args.pixels = device_pixels.as<int2>();
        args.pixel_count = static_cast<int>(pixel_count);
        args.sum_squares = sum_squares != nullptr ? device_squares.as<double>() : nullptr;
        const DevCamera camera{deviceCamera(scene->host, job->width, job->height)};
        check(launchMegakernel(scene->dev, camera, args, device_accum.as<PixelAccum>(),
                               scene->error_flag.as<unsigned int>(), scene->stack_capacity, nullptr),
              "render launch");
        check(cudaDeviceSynchronize(), "render");
        download(accumulators, device_accum, count);
        if (sum_squares != nullptr) {
            download(sum_squares, device_squares, 3 * count);
        }
        scene->collectKernelError();
    });
}

int albedo_render_work_counts(const albedo_scene* scene, const albedo_render_job* job, int64_t* out_counts)
{
    return guarded([&] {
        const RenderArgs args{renderArgsFor(*scene, *job)};
        const std::size_t pixels{static_cast<std::size_t>(job->width) * static_cast<std::size_t>(job->height)};
        DeviceBuffer accum{pixels * sizeof(PixelAccum)};
        DeviceBuffer totals{6 * sizeof(unsigned long long)};
        check(cudaMemset(accum.ptr, 0, accum.bytes), "cudaMemset");
        check(cudaMemset(totals.ptr, 0, totals.bytes), "cudaMemset");
        const DevCamera camera{deviceCamera(scene->host, job->width, job->height)};
        check(launchMegakernelCounting(scene->dev, camera, args, accum.as<PixelAccum>(),
                                       scene->error_flag.as<unsigned int>(), scene->stack_capacity,
                                       totals.as<unsigned long long>(), nullptr),
              "counting launch");
        check(cudaDeviceSynchronize(), "counting");
        unsigned long long host[6]{};
        check(cudaMemcpy(host, totals.ptr, sizeof(host), cudaMemcpyDeviceToHost), "download");
        for (int i{0}; i < 6; ++i) {
            out_counts[i] = static_cast<int64_t>(host[i]);
        }
        scene->collectKernelError();
    });
}

int albedo_trace_counts_host(const albedo_scene* scene, const float* rays, int64_t count, float t_min, float t_max,
                             int64_t* out_counts)
{
    return guarded([&] {
        scene->requireCommitted();
        if (count <= 0 || count > (int64_t{1} << 30)) {
            throw std::invalid_argument{"ray count must be in 1..2^30"};
        }
        const auto n{static_cast<std::size_t>(count)};
        DeviceBuffer d_rays{uploadRaw(rays, 6 * n)};
        DeviceBuffer totals{6 * sizeof(unsigned long long)};
        check(cudaMemset(totals.ptr, 0, totals.bytes), "cudaMemset");
        check(launchTraceCounting(scene->dev, d_rays.as<float>(), static_cast<int>(count), t_min, t_max,
                                  scene->error_flag.as<unsigned int>(), scene->stack_capacity,
                                  totals.as<unsigned long long>(), nullptr),
              "counting trace launch");
        check(cudaDeviceSynchronize(), "counting trace");
        unsigned long long host[6]{};
        check(cudaMemcpy(host, totals.ptr, sizeof(host), cudaMemcpyDeviceToHost), "download");
        for (int i{0}; i < 6; ++i) {
            out_counts[i] = static_cast<int64_t>(host[i]);
        }
        scene->collectKernelError();
    });
}

int albedo_scene_check(const albedo_scene* scene)
{
    return guarded([&] {
        check(cudaDeviceSynchronize(), "synchronize");
        scene->collectKernelError();
    });
}

int albedo_trace_host(const albedo_scene* scene, const float* rays, int64_t count, float t_min, float t_max,
                      int32_t* hit, float* t, int32_t* object, int32_t* triangle, float* point, float* normal,
                      float* shading_normal, int32_t* front)
{
    return guarded([&] {
        scene->requireCommitted();
        const auto n{static_cast<std::size_t>(count)};
        DeviceBuffer d_rays{uploadRaw(rays, 6 * n)};
        DeviceBuffer d_hit{n * sizeof(int)};
        DeviceBuffer d_t{n * sizeof(float)};
        DeviceBuffer d_object{n * sizeof(int)};
        DeviceBuffer d_triangle{n * sizeof(int)};
        const bool geometry{point != nullptr};
        DeviceBuffer d_point{geometry ? 3 * n * sizeof(float) : 0};
        DeviceBuffer d_normal{geometry ? 3 * n * sizeof(float) : 0};
        DeviceBuffer d_shading{geometry ? 3 * n * sizeof(float) : 0};
        DeviceBuffer d_front{geometry ? n * sizeof(int) : 0};
        TraceOutputs out{d_hit.as<int>(),   d_t.as<float>(),      d_object.as<int>(),   d_triangle.as<int>(),
                         d_point.as<float>(), d_normal.as<float>(), d_shading.as<float>(), d_front.as<int>()};
        check(launchTrace(scene->dev, d_rays.as<float>(), static_cast<int>(count), t_min, t_max, out,
                          scene->error_flag.as<unsigned int>(), scene->stack_capacity, nullptr),
              "trace launch");
        check(cudaDeviceSynchronize(), "trace");
        download(hit, d_hit, n);
        download(t, d_t, n);
        download(object, d_object, n);
        download(triangle, d_triangle, n);
        if (geometry) {
            download(point, d_point, 3 * n);
            download(normal, d_normal, 3 * n);
            download(shading_normal, d_shading, 3 * n);
            download(front, d_front, n);
        }
        scene->collectKernelError();
    });
}

int albedo_occluded_host(const albedo_scene* scene, const float* rays, const float* t_max, int64_t count,
                         int32_t* occluded)
{
    return guarded([&] {
        scene->requireCommitted();
        const auto n{static_cast<std::size_t>(count)};
        DeviceBuffer d_rays{uploadRaw(rays, 6 * n)};
        DeviceBuffer d_tmax{uploadRaw(t_max, n)};
        DeviceBuffer d_out{n * sizeof(int)};
        check(launchOccluded(scene->dev, d_rays.as<float>(), d_tmax.as<float>(), static_cast<int>(count),
                             d_out.as<int>(), scene->error_flag.as<unsigned int>(), scene->stack_capacity, nullptr),
              "occluded launch");
        check(cudaDeviceSynchronize(), "occluded");
        download(occluded, d_out, n);
        scene->collectKernelError();
    });
}

int albedo_probe_pixel_stream(uint64_t seed, int32_t x, int32_t y, int32_t width, int32_t count, uint32_t* out_u32,
                              float* out_real)
{
    return guarded([&] {
        const auto n{static_cast<std::size_t>(count)};
        DeviceBuffer u{n * sizeof(unsigned int)};
        DeviceBuffer r{n * sizeof(float)};
        check(launchPixelStream(seed, x, y, width, count, u.as<unsigned int>(), r.as<float>(), nullptr), "probe");
        check(cudaDeviceSynchronize(), "probe");
        download(out_u32, u, n);
        download(out_real, r, n);
    });
}

int albedo_probe_lobe_eval(int32_t kind, const float* params, const float* wo_wi, int32_t count, float* out_f,
                           float* out_pdf)
{
    return guarded([&] {
        const auto n{static_cast<std::size_t>(count)};
        DeviceBuffer p{uploadRaw(params, 8)};
        DeviceBuffer in{uploadRaw(wo_wi, 6 * n)};
        DeviceBuffer f{3 * n * sizeof(float)};
        DeviceBuffer pdf{n * sizeof(float)};
        check(launchLobeEval(kind, p.as<float>(), in.as<float>(), count, f.as<float>(), pdf.as<float>(), nullptr),
              "probe");
        check(cudaDeviceSynchronize(), "probe");
        download(out_f, f, 3 * n);
        download(out_pdf, pdf, n);
    });
}

int albedo_probe_lobe_sample(int32_t kind, const float* params, const float* inputs, int32_t count, int32_t* out_valid,
                             float* out_direction, float* out_weight, float* out_pdf, int32_t* out_specular)
{
    return guarded([&] {
        const auto n{static_cast<std::size_t>(count)};
        DeviceBuffer p{uploadRaw(params, 8)};
        DeviceBuffer in{uploadRaw(inputs, 6 * n)};
        DeviceBuffer valid{n * sizeof(int)};
        DeviceBuffer dir{3 * n * sizeof(float)};
        DeviceBuffer weight{3 * n * sizeof(float)};
        DeviceBuffer pdf{n * sizeof(float)};
        DeviceBuffer spec{n * sizeof(int)};
        check(cudaMemset(valid.ptr, 0, n * sizeof(int)), "memset");
        check(launchLobeSample(kind, p.as<float>(), in.as<float>(), count, valid.as<int>(), dir.as<float>(),
                               weight.as<float>(), pdf.as<float>(), spec.as<int>(), nullptr),
              "probe");
        check(cudaDeviceSynchronize(), "probe");
        download(out_valid, valid, n);
        download(out_direction, dir, 3 * n);
        download(out_weight, weight, 3 * n);
        download(out_pdf, pdf, n);
        download(out_specular, spec, n);
    });
}

int albedo_probe_perlin(const float* points, int32_t count, float* out_noise, float* out_turbulence)
{
    return guarded([&] {
        const auto n{static_cast<std::size_t>(count)};
        DeviceBuffer in{uploadRaw(points, 3 * n)};
        DeviceBuffer noise{n * sizeof(float)};
        DeviceBuffer turb{n * sizeof(float)};
        check(launchPerlin(in.as<float>(), count, noise.as<float>(), turb.as<float>(), nullptr), "probe");
        check(cudaDeviceSynchronize(), "probe");
        download(out_noise, noise, n);
        download(out_turbulence, turb, n);
    });
}

int albedo_probe_read_sweep(const void* data, int64_t bytes, int32_t repeats, int32_t blocks, void* sink,
                            void* stream)
{
    return guarded([&] {
        if (data == nullptr || sink == nullptr || bytes < 16 || bytes % 16 != 0 || repeats <= 0 || blocks <= 0 ||
            reinterpret_cast<std::uintptr_t>(data) % 16 != 0 || reinterpret_cast<std::uintptr_t>(sink) % 16 != 0) {
            throw std::invalid_argument{"read sweep: 16-byte aligned data and sink, bytes a positive multiple of 16, "
                                        "positive repeats and blocks"};
        }
        check(launchReadSweep(data, bytes, repeats, blocks, sink, static_cast<cudaStream_t>(stream)), "read sweep");
    });
}

int albedo_probe_trace_modes(const albedo_scene* scene, const float* rays, int64_t count, float t_min, float t_max,
                             int32_t any, int32_t persistent, int32_t* out_hit, uint32_t* out_t_bits,
                             uint32_t* out_object_position, uint32_t* out_triangle_position)
{
    return guarded([&] {
        scene->requireCommitted();
        if (count <= 0 || count > (int64_t{1} << 28)) {
            throw std::invalid_argument{"ray count must be in 1..2^28"};
        }
        const auto n{static_cast<std::size_t>(count)};
        DeviceBuffer d_rays{uploadRaw(rays, 6 * n)};
        DeviceBuffer counter{sizeof(int)};
        DeviceBuffer hit{n * sizeof(int)};
        DeviceBuffer t{n * sizeof(unsigned int)};
        DeviceBuffer obj{n * sizeof(unsigned int)};
        DeviceBuffer tri{n * sizeof(unsigned int)};
        check(cudaMemset(counter.ptr, 0, sizeof(int)), "cudaMemset");
        if (persistent < 0 || persistent > 3) {
            throw std::invalid_argument{"persistent must be 0, 1, 2 or 3"};
        }
        check(launchTraceModes(scene->dev, d_rays.as<float>(), static_cast<int>(count), t_min, t_max, any != 0,
                               persistent, scene->stack_capacity, counter.as<int>(),
                               scene->error_flag.as<unsigned int>(), hit.as<int>(), t.as<unsigned int>(),
                               obj.as<unsigned int>(), tri.as<unsigned int>(), nullptr),
              "probe");
        check(cudaDeviceSynchronize(), "probe");
        download(out_hit, hit, n);
        download(out_t_bits, t, n);
        download(out_object_position, obj, n);
        download(out_triangle_position, tri, n);
        scene->collectKernelError();
    });
}

int albedo_probe_camera_rays(const albedo_scene* scene, int32_t width, int32_t height, const float* film, int32_t count,
                             float* out_rays)
{
    return guarded([&] {
        const auto n{static_cast<std::size_t>(count)};
        const DevCamera camera{deviceCamera(scene->host, width, height)};
        DeviceBuffer in{uploadRaw(film, 2 * n)};
        DeviceBuffer out{6 * n * sizeof(float)};
        check(launchCameraRays(camera, in.as<float>(), count, out.as<float>(), nullptr), "probe");
        check(cudaDeviceSynchronize(), "probe");
        download(out_rays, out, 6 * n);
    });
}

} // extern "C"
