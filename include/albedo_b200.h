/*
 * albedo_b200: the C ABI of the B200 path tracer.
 *
 * A drop-in for the render path of anazli/albedo. The reference has no C or FFI
 * API of its own; these entry points replace the C++ calls its app and tests
 * make, one for one:
 *
 *   albedo_scene_load           readScene(path)                    src/albedo/scene/scene_file.hpp:142-146
 *   albedo_scene_create/...     Scene::add / addAreaLight /        src/albedo/scene/scene.hpp:31-62
 *                               addLight / setSky, TriangleMesh,   src/albedo/geometry/triangle_mesh.hpp:29-41
 *                               MeshGeometry, MeshInstance,        src/albedo/geometry/mesh_geometry.hpp:30-33
 *                               Transform factories                src/albedo/geometry/mesh_instance.hpp:24-27
 *                                                                  src/albedo/core/transform.hpp:45-66
 *   albedo_scene_set_camera     CameraSettings                     src/albedo/camera/perspective_camera.hpp:13-26
 *   albedo_render               renderImage(RenderJob, PixelBuffer) src/albedo/render/render_image.hpp:36-49
 *   albedo_render_host          renderImage with a host PixelBuffer src/albedo/render/render_image.hpp:36-49
 *   albedo_trace_host           Scene::intersect                   src/albedo/scene/scene.hpp:69-75
 *   albedo_occluded_host        Scene::occluded                    src/albedo/scene/scene.hpp:86-88
 *   albedo_resolve_srgb         writePpm's encodeRow               src/albedo/image/ppm.cpp:22-33
 *   albedo_write_ppm/save_ppm   writePpm(path, image)              src/albedo/image/ppm.cpp:61-85
 *
 * Exceptions never cross the ABI: every call returns an albedo_status and leaves
 * a message in a thread-local string (albedo_last_error). Status values map to
 * the reference's exception types (std::invalid_argument, SceneParseError,
 * std::runtime_error, std::out_of_range) plus device failures.
 *
 * Scenes are immutable once committed; any number of renders may then run on
 * them concurrently on different streams. Accumulators follow PixelBuffer's
 * Accumulator (src/albedo/image/pixel_buffer.hpp:53-57): an FP64 RGB sum and an
 * int64 sample count per pixel, row-major from the top-left pixel; renders ADD
 * samples to them, as renderImage adds to a PixelBuffer.
 */
#ifndef ALBEDO_B200_H
#define ALBEDO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct albedo_scene albedo_scene;

typedef enum albedo_status {
    ALBEDO_OK = 0,
    ALBEDO_INVALID_ARGUMENT = 1, /* std::invalid_argument */
    ALBEDO_PARSE_ERROR = 2,      /* SceneParseError, with the line number in the message */
    ALBEDO_IO_ERROR = 3,         /* std::runtime_error: a file cannot be opened or read */
    ALBEDO_OUT_OF_RANGE = 4,     /* std::out_of_range: a mesh index past its table */
    ALBEDO_DEVICE_ERROR = 5,     /* a CUDA call failed */
    ALBEDO_OUT_OF_MEMORY = 6,    /* device or host allocation failed */
    ALBEDO_UNSUPPORTED = 7,      /* beyond the device layout's limits (see message) */
    ALBEDO_TRAVERSAL_ERROR = 8   /* a kernel reported a traversal stack overflow */
} albedo_status;

/* One per pixel; 32 bytes, as PixelBuffer's Accumulator. */
typedef struct albedo_accumulator {
    double r;
    double g;
    double b;
    int64_t count;
} albedo_accumulator;

typedef enum albedo_estimator {
    ALBEDO_PATH = 0,         /* PathEstimator: NEE + MIS + Russian roulette */
    ALBEDO_SCATTER_ONLY = 1, /* ScatterOnlyEstimator (max_depth = max_scatter_count) */
    ALBEDO_NORMALS = 2       /* NormalsEstimator */
} albedo_estimator;

typedef enum albedo_method {
    ALBEDO_MEGAKERNEL = 0, /* one thread per pixel, samples in sequence */
    ALBEDO_WAVEFRONT = 1   /* path slots advanced bounce by bounce through compacted queues */
} albedo_method;

/* How the megakernel sums a pixel's samples before adding them to the FP64
 * accumulators. The reference sums in FP64 (render/render_image.cpp:27-44). */
typedef enum albedo_accumulation {
    ALBEDO_ACCUMULATE_FP64 = 0,      /* FP64 running sums (all methods) */
    ALBEDO_ACCUMULATE_KAHAN_FP32 = 1 /* FP32 with Kahan compensation (megakernel, path estimator) */
} albedo_accumulation;

/* RenderJob (src/albedo/render/render_image.hpp:17-32) minus the camera and scene. */
typedef struct albedo_render_job {
    int32_t width;
    int32_t height;
    int32_t samples_per_axis; /* n: n x n stratified samples per pixel */
    int32_t estimator;        /* albedo_estimator */
    uint64_t seed;
    int32_t max_depth;        /* PathEstimator::max_depth (default 64) */
    int32_t roulette_start;   /* PathEstimator::roulette_start (default 3) */
    int32_t method;           /* albedo_method */
    int32_t accumulation;     /* albedo_accumulation */
} albedo_render_job;

/* A view for one render in place of the scene's camera: CameraSettings
 * (src/albedo/camera/perspective_camera.hpp:13-26), validated as the
 * PerspectiveCamera constructor does. */
typedef struct albedo_camera {
    double look_from[3];
    double look_at[3];
    double up[3];
    double vertical_fov_degrees;
} albedo_camera;

/* BasicMaterial: kind 0 diffuse (texture 0 constant color a, 1 checker even a /
 * odd b / frequency, 2 Perlin low a / high b / scale / veins), kind 1 conductor
 * (eta a, k b, roughness), kind 2 dielectric (ior, roughness). */
typedef struct albedo_basic_material {
    int32_t kind;
    int32_t texture;
    double a[3];
    double b[3];
    double frequency_or_scale;
    double veins;
    double ior;
    double roughness;
} albedo_basic_material;

/* Material: a basic material, or (mix != 0) MixMaterial of two basic ones. */
typedef struct albedo_material {
    int32_t mix;
    int32_t reserved;
    albedo_basic_material first;
    albedo_basic_material second;
    double scale;
    double veins;
    double threshold;
} albedo_material;

typedef struct albedo_scene_info {
    int64_t objects;
    int64_t lights;
    int64_t triangles;       /* scene triangles plus every mesh's triangles */
    int64_t nodes;           /* device BVH nodes (4-wide form) */
    int64_t device_bytes;    /* device memory held by the committed scene */
    int32_t stack_need;      /* traversal stack entries a query can need */
    int32_t stack_capacity;  /* entries of the kernel variant chosen */
} albedo_scene_info;

const char* albedo_last_error(void);

/* Scene input. albedo_scene_load = albedo_scene_read + albedo_scene_commit. */
int albedo_scene_load(const char* path, albedo_scene** out);
/* Reads a scene file and builds its hierarchy and device tables on the host
 * only (no device needed); commit uploads it. */
int albedo_scene_read(const char* path, albedo_scene** out);
int albedo_scene_create(albedo_scene** out);
void albedo_scene_destroy(albedo_scene* scene);
int albedo_scene_set_camera(albedo_scene* scene, const double look_from[3], const double look_at[3],
                            const double up[3], double vertical_fov_degrees);
int albedo_scene_add_material(albedo_scene* scene, const albedo_material* material, uint32_t* out_material);
int albedo_scene_add_sphere(albedo_scene* scene, const double center[3], double radius, uint32_t material,
                            uint32_t* out_object);
int albedo_scene_add_area_light(albedo_scene* scene, const double center[3], double radius,
                                const double radiance[3], uint32_t material, uint32_t* out_object);
int albedo_scene_add_point_light(albedo_scene* scene, const double position[3], const double intensity[3]);
int albedo_scene_set_sky(albedo_scene* scene, const double nadir[3], const double zenith[3]);
/* A shared mesh (TriangleMesh + MeshGeometry): positions (3 per vertex), faces
 * (3 indices each), optional texture coordinates (2 each) and texture faces
 * (0 or face_count of them). smooth != 0 shades with averaged vertex normals. */
int albedo_scene_add_mesh(albedo_scene* scene, const double* positions, int64_t position_count,
                          const uint32_t* faces, int64_t face_count, const double* texture_coordinates,
                          int64_t texture_coordinate_count, const uint32_t* texture_faces,
                          int64_t texture_face_count, int32_t smooth, uint32_t* out_mesh);
/* A MeshInstance: object-to-world as a 3x4 row-major affine matrix and its exact
 * inverse, as Transform keeps both. */
int albedo_scene_add_instance(albedo_scene* scene, uint32_t mesh, const double to_world[12],
                              const double to_object[12], uint32_t material, uint32_t* out_object);
/* Scene::add(TriangleMesh, material): every triangle its own object. */
int albedo_scene_add_triangles(albedo_scene* scene, const double* positions, int64_t position_count,
                               const uint32_t* faces, int64_t face_count, uint32_t material);
/* Builds the TLAS and the device tables on the host (idempotent; no device). */
int albedo_scene_prepare(albedo_scene* scene);
/* Prepares if needed, then uploads the scene to the current CUDA device. */
int albedo_scene_commit(albedo_scene* scene);
/* The host-side scene tables (an albedo_b200::HostScene) of a prepared scene,
 * for test code built against the same headers; valid until destroy. */
const void* albedo_scene_host_view(const albedo_scene* scene);
int albedo_scene_get_info(const albedo_scene* scene, albedo_scene_info* out);

/* Rendering. albedo_render is stream-ordered and asynchronous: `accumulators`
 * is a device array of width*height entries; `stream` is a cudaStream_t (NULL:
 * the default stream). Call albedo_scene_check after synchronizing to collect a
 * kernel-reported error. albedo_render_host takes a host array, copies it in,
 * renders, copies it back and synchronizes; it stages the array in a device
 * buffer kept per device (grown to the largest image seen, never freed), so
 * repeated host renders allocate nothing, and host renders on one device run
 * one at a time. */
int albedo_render(const albedo_scene* scene, const albedo_render_job* job, albedo_accumulator* accumulators,
                  void* stream);
int albedo_render_host(const albedo_scene* scene, const albedo_render_job* job, albedo_accumulator* accumulators);
/* albedo_render from the given camera instead of the scene's (NULL: the
 * scene's). The reference builds one PerspectiveCamera per render from the
 * settings it is given (app/main.cpp); this is that call with a per-request
 * camera on a resident scene. */
int albedo_render_view(const albedo_scene* scene, const albedo_render_job* job, const albedo_camera* camera,
                       albedo_accumulator* accumulators, void* stream);
/* albedo_render_host from the given camera (NULL: the scene's): renderImage
 * (render/render_image.hpp:36-49) with a host PixelBuffer and the job's own
 * camera, as the C++ adapter include/albedo_b200_adapter.hpp calls it. */
int albedo_render_view_host(const albedo_scene* scene, const albedo_render_job* job, const albedo_camera* camera,
                            albedo_accumulator* accumulators);
/* Renders only the listed pixels (x, y pairs) into one host accumulator each,
 * optionally also returning per-pixel sums of squared samples (3 doubles each). */
int albedo_render_pixels_host(const albedo_scene* scene, const albedo_render_job* job, const int32_t* pixels,
                              int64_t pixel_count, albedo_accumulator* accumulators, double* sum_squares);
/* One job of a batch: a committed scene, its job, and a device array of its
 * width*height accumulators. */
typedef struct albedo_batch_item {
    const albedo_scene* scene;
    albedo_render_job job;
    albedo_accumulator* accumulators;
} albedo_batch_item;

/* Renders many jobs (any scenes, sizes and sample counts; path estimator) in one
 * wavefront run that shares the path slots among them, so small jobs fill the
 * GPU together. Each job's image is the one renderImage would give it alone.
 * Returns when every job is done. No counterpart in the reference, which renders
 * one job per call; this batches renderImage (render_image.hpp:36-49). */
int albedo_render_batch(const albedo_batch_item* items, int32_t count, void* stream);
/* Renders one job (path estimator) without allocating any device memory: no
 * cudaMalloc, cudaFree or allocating library call. It has no counterpart in the
 * reference, whose renderImage allocates nothing on a GPU because it has none.
 * It is for callers that cannot allocate: a program whose device memory another
 * allocator owns up front (a framework's caching pool that has reserved the
 * GPU), or a loop with a latency budget, where an allocation can stall on the
 * driver or synchronize the device. The wavefront's path slots, queues and
 * control block live in a static device array of about 17 MB that every GPU
 * loading the library holds until exit. It holds one path slot per pixel, so
 * images are limited to 65,536 pixels; larger ones are rejected with
 * ALBEDO_INVALID_ARGUMENT. The first call on a device looks up that array's
 * device address (cudaGetSymbolAddress) and should come before any stream
 * capture. All calls share the array and it keeps the last call's contents:
 * each call clears what must start at zero, and calls that overlap on the GPU
 * race, so do not overlap them. `accumulators` is a device array of width *
 * height entries. The call synchronizes `stream`: it returns once the render
 * is complete, with a kernel-reported error (ALBEDO_TRAVERSAL_ERROR) already
 * collected. The array's address is looked up once per device for the life of
 * the process, so calls after cudaDeviceReset on that device are not
 * supported. */
int albedo_render_noalloc(const albedo_scene* scene, const albedo_render_job* job, albedo_accumulator* accumulators,
                          void* stream);
/* Film output (image/ppm.cpp:22-85, color/srgb.cpp:18-36). albedo_resolve_srgb
 * turns width*height device accumulators into width*height*3 device bytes, the
 * R G B bytes writePpm writes for each pixel's average (rows from the top): the
 * average is sum / count (0 without samples), its byte toByte(encodeSrgb(.)).
 * The bytes equal the reference's exactly. It is asynchronous on `stream`;
 * accumulators must be 8-byte aligned. It replaces the reference's per-pixel
 * encodeRow loop (image/ppm.cpp:22-33) and, for a served image, the copy of 32
 * bytes a pixel to the host by one of 3. */
int albedo_resolve_srgb(const albedo_accumulator* accumulators, int32_t width, int32_t height, uint8_t* out_rgb,
                        void* stream);
/* The resolve's tables, computed on the host from the reference's transfer
 * function. out_lower (256 doubles): [b] (b = 1..255) is the smallest positive
 * double whose byte is at least b; [0] is -infinity. out_start (1664 bytes, or
 * NULL): the byte at the smallest double of each bucket, where bucket k holds the
 * doubles whose bit pattern shifted right by 45 is (1023 - 13) * 128 + k (an
 * exponent and the top 7 mantissa bits, covering [2^-13, 1)); no bucket holds
 * more than one threshold, so a value's byte is start or start + 1. */
int albedo_srgb_tables(double* out_lower, uint8_t* out_start);
/* writePpm(path, image) (image/ppm.cpp:61-85) from host bytes already encoded:
 * a binary P6 file with maxval 255. The file is truncated on open; on a failed
 * write the partial file is removed (when it is a regular file). Errors carry the
 * reference's messages: "cannot open '<path>' for writing", "failed to write
 * '<path>': failed to write PPM image" (a failure while writing) and "failed to
 * write '<path>'" (a failure on close); all are ALBEDO_IO_ERROR. */
int albedo_write_ppm(const char* path, const uint8_t* rgb, int32_t width, int32_t height);
/* writePpm(path, image) for device accumulators: resolves them on `stream`,
 * copies the bytes back, synchronizes the stream and writes the file. */
int albedo_save_ppm(const char* path, const albedo_accumulator* accumulators, int32_t width, int32_t height,
                    void* stream);
/* albedo_save_ppm for host accumulators, uploaded through the per-device staging
 * buffer that albedo_render_host uses. */
int albedo_save_ppm_host(const char* path, const albedo_accumulator* accumulators, int32_t width, int32_t height);
/* A render server: continuous batching of requests on one wavefront engine. A
 * request is admitted, in arrival order, once the device memory it needs fits
 * the budget: the engine's path slots and queues, each scene's tables (counted
 * once; scenes stay resident) and each running request's accumulators. Admitted
 * requests join the batch already on the device between graph launches, so
 * their work overlaps the work of requests admitted before them. A small
 * request admitted while the batch is lightly loaded takes the express route
 * instead: the megakernel renders it on the server's own stream, beside the
 * batch (a pixel's samples run in sequence either way, and the megakernel runs
 * them in one launch). Each result is the image the same request would get
 * alone: the same paths, equal within the tolerance between the two forms. No
 * counterpart in the reference, which renders one image per process. */
typedef struct albedo_server albedo_server;
int albedo_server_create(int64_t memory_budget_bytes, int32_t slot_count, albedo_server** out);
/* Queues a request (committed scene, job, device accumulators) and admits what
 * fits. The ticket identifies it in albedo_server_step's results. */
int albedo_server_submit(albedo_server* server, const albedo_scene* scene, const albedo_render_job* job,
                         albedo_accumulator* accumulators, int64_t* out_ticket);
/* albedo_server_submit with the request's own camera (NULL: the scene's). */
int albedo_server_submit_view(albedo_server* server, const albedo_scene* scene, const albedo_render_job* job,
                              const albedo_camera* camera, albedo_accumulator* accumulators, int64_t* out_ticket);
/* Advances the device by one graph of iterations and reports (up to `capacity`)
 * tickets whose accumulators are now complete; tickets beyond `capacity` are
 * reported by later calls. */
int albedo_server_step(albedo_server* server, int64_t* finished, int32_t capacity, int32_t* out_finished);
int albedo_server_pending(const albedo_server* server, int32_t* out_waiting, int32_t* out_running);
/* The express route's limit: requests of at most `max_pixels` pixels may take
 * it (default 65,536); 0 sends every request to the batch. */
int albedo_server_set_express(albedo_server* server, int64_t max_pixels);
/* Requests admitted so far to the batch and to the express route. */
int albedo_server_routes(const albedo_server* server, int64_t* out_batched, int64_t* out_express);
/* Stops counting a scene's tables against the server's budget (and admits what
 * then fits). The server counts each scene once, from its first admitted
 * request until this call; call it before destroying a scene the server has
 * rendered. A scene with requests still waiting or running is refused. */
int albedo_server_release_scene(albedo_server* server, const albedo_scene* scene);
void albedo_server_destroy(albedo_server* server);
/* Wavefront engine shape: path slots, blocks per SM of the queue kernels, and
 * iterations per captured CUDA graph; the traversal kernels' blocks per SM and
 * fetch batch return to their defaults (as many as fit, 32). */
int albedo_wavefront_configure(int32_t slot_count, int32_t blocks_per_sm, int32_t iterations_per_graph);
/* Autotuner. No counterpart in the reference (a CPU renderer with no launch
 * shapes). Candidate launch shapes are timed with CUDA events on the caller's
 * work rendered at a quarter of its samples (samples per axis halved) into
 * scratch accumulators; the caller's accumulators are not touched. The fastest
 * shape is kept and used by later renders: per scene for the megakernel, by the
 * process's wavefront engine and servers created afterwards for batches.
 * Images do not depend on the shape. Synchronous. */
typedef struct albedo_tuning {
    int32_t tile_width;           /* megakernel: pixel tile width (8, 16 or 32; 128-pixel tiles) */
    int32_t blocks_per_sm;        /* megakernel: register budget (3 or 4 resident blocks per SM; at 4
                                     the path estimator keeps each path's state in shared memory);
                                     wavefront: blocks per SM of the queue kernels */
    int32_t trace_blocks_per_sm;  /* wavefront: persistent traversal blocks per SM */
    int32_t fetch_batch;          /* wavefront: queue entries a traversal warp claims at once */
    int32_t iterations_per_graph; /* wavefront: iterations per captured CUDA graph */
    int32_t slot_count;           /* wavefront: path slots */
    int32_t evaluations;          /* shapes timed */
    int32_t inline_traversal;     /* megakernel: 0 = one out-of-line traversal copy serves both queries,
                                     1 = both queries' traversal inlined into the kernel, 2 = the
                                     closest-hit query's inlined and the shadow query's out of line
                                     (path estimator; 2 at 3 blocks per SM only) */
    int32_t trace_loop;           /* wavefront: 0 = a traversal turn descends nodes then handles a leaf,
                                     1 = a turn is one node or one leaf, 2 = a turn is the whole query
                                     (out-of-line traversal; same steps, same results) */
    int32_t ray_sort;             /* wavefront: 1 = the rays of each bounce are binned by job, direction
                                     octant and origin cell before they are traced, 2 = the shadow rays
                                     too (same results) */
    double best_ms;               /* the kept shape's time on the tuning work */
    double default_ms;            /* the default shape's time on the same work */
} albedo_tuning;
/* Tunes the megakernel for `scene` on `job` and keeps the result in the scene:
 * every tile width with every kernel variant (3 or 4 blocks per SM with an
 * out-of-line traversal; 3 or 4 with the traversal inlined for both queries;
 * or 3 with it inlined for the closest-hit query only: which is fastest
 * depends on the scene). */
int albedo_autotune_megakernel(albedo_scene* scene, const albedo_render_job* job, albedo_tuning* out);
/* Tunes the wavefront engine on a batch (coordinate descent over traversal
 * blocks per SM, fetch batch, traversal turn shape, queue-kernel blocks per SM,
 * iterations per graph, slot count and ray binning) and keeps the result for
 * the process. */
int albedo_autotune_batch(const albedo_batch_item* items, int32_t count, albedo_tuning* out);
/* The shape renders use now: the scene's megakernel shape (scene not NULL) or
 * the process's wavefront shape (scene NULL); timing fields are zero. */
int albedo_tuning_get(const albedo_scene* scene, albedo_tuning* out);
/* Pins a shape, as the autotuner would keep it: the scene's megakernel shape
 * (scene not NULL: tile_width 8, 16 or 32, blocks_per_sm 3 or 4, and
 * inline_traversal 0, 1 or 2, the last with 3 blocks per SM) or the
 * process's wavefront shape (scene NULL: blocks_per_sm, trace_blocks_per_sm,
 * fetch_batch, iterations_per_graph and slot_count, all positive, and
 * trace_loop 0, 1 or 2, ray_sort 0, 1 or 2). Timing fields are ignored. Images do not depend on the
 * shape. */
int albedo_tuning_set(albedo_scene* scene, const albedo_tuning* shape);
/* Iterations the last wavefront run took. */
int albedo_wavefront_last_iterations(int64_t* out);
/* Ray queries (closest hit plus shadow) the last wavefront run traced. */
int albedo_wavefront_last_rays(int64_t* out);
/* Ray queries the server's current batch has traced, as of the last step whose
 * results were polled (the count restarts when the engine reopens a batch). */
int albedo_server_rays(const albedo_server* server, int64_t* out);
/* Renders the job once (path estimator, into scratch accumulators) while counting
 * traversal work: out_counts[0..5] = child boxes the 4-wide traversal tested,
 * triangles tested, spheres tested, instances entered, ray queries traced, and
 * the boxes the reference's binary traversal (accel/bvh.hpp:239-278: one box
 * per node popped) tests for the same queries. Synchronous. No counterpart in
 * the reference. */
int albedo_render_work_counts(const albedo_scene* scene, const albedo_render_job* job, int64_t* out_counts);
/* The same six counts for closest-hit queries of given rays (6 floats each,
 * as albedo_trace_host). Synchronous. */
int albedo_trace_counts_host(const albedo_scene* scene, const float* rays, int64_t count, float t_min, float t_max,
                             int64_t* out_counts);
/* Reads and clears the scene's kernel error flag (synchronizes the device). */
int albedo_scene_check(const albedo_scene* scene);

/* Ray queries over host arrays of rays (origin xyz, direction xyz as floats).
 * trace: hit flag, t, object id (add order), triangle id within its mesh (-1 if
 * none), and optionally point / normal / shading normal (3 floats each) and
 * front-face flags. occluded: any hit in (0, t_max[i]). */
int albedo_trace_host(const albedo_scene* scene, const float* rays, int64_t count, float t_min, float t_max,
                      int32_t* hit, float* t, int32_t* object, int32_t* triangle, float* point, float* normal,
                      float* shading_normal, int32_t* front);
int albedo_occluded_host(const albedo_scene* scene, const float* rays, const float* t_max, int64_t count,
                         int32_t* occluded);

/* Probes of device arithmetic for parity tests (host arrays). */
int albedo_probe_pixel_stream(uint64_t seed, int32_t x, int32_t y, int32_t width, int32_t count, uint32_t* out_u32,
                              float* out_real);
int albedo_probe_lobe_eval(int32_t kind, const float* params, const float* wo_wi, int32_t count, float* out_f,
                           float* out_pdf);
int albedo_probe_lobe_sample(int32_t kind, const float* params, const float* inputs, int32_t count,
                             int32_t* out_valid, float* out_direction, float* out_weight, float* out_pdf,
                             int32_t* out_specular);
int albedo_probe_perlin(const float* points, int32_t count, float* out_noise, float* out_turbulence);
int albedo_probe_camera_rays(const albedo_scene* scene, int32_t width, int32_t height, const float* film,
                             int32_t count, float* out_rays);
/* Reads `bytes` of device memory at `data` (16-byte aligned, a multiple of 16
 * bytes) `repeats` times through L2 (L1 skipped) with `blocks` blocks of 256
 * threads, writing at most 16 bytes to the device `sink`; asynchronous on
 * `stream`. Timed by the caller, it gives the L2 read bandwidth that the
 * traversal of a scene resident in L2 is measured against. No counterpart in
 * the reference. */
int albedo_probe_read_sweep(const void* data, int64_t bytes, int32_t repeats, int32_t blocks, void* sink,
                            void* stream);
/* Closest-hit (any = 0) or any-hit queries of given rays, traced as the
 * wavefront's persistent kernels trace them (persistent = 1: a turn descends
 * nodes then handles a leaf; 2: a turn is one step; 3: a turn is the whole
 * query, traced by the out-of-line traversal) or one query per thread
 * through the shared traversal (persistent = 0): raw hit flag, FP32 t
 * bits, object leaf position and triangle table position (0xFFFFFFFF if none),
 * so that tests can compare the two ways bit for bit. */
int albedo_probe_trace_modes(const albedo_scene* scene, const float* rays, int64_t count, float t_min, float t_max,
                             int32_t any, int32_t persistent, int32_t* out_hit, uint32_t* out_t_bits,
                             uint32_t* out_object_position, uint32_t* out_triangle_position);

#ifdef __cplusplus
}
#endif

#endif /* ALBEDO_B200_H */
