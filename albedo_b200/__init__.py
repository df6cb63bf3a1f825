"""albedo_b200: a B200-native (sm_100a) path tracer with albedo's render API.

The Python surface mirrors the reference's render entry points over the C ABI
of include/albedo_b200.h:

    read_scene / load_scene   readScene            (src/albedo/scene/scene_file.hpp:142-146)
    Scene builder methods     Scene::add*, setSky  (src/albedo/scene/scene.hpp:31-62)
    RenderJob                 RenderJob            (src/albedo/render/render_image.hpp:17-32)
    PixelBuffer               PixelBuffer          (src/albedo/image/pixel_buffer.hpp:17-65)
    render_image              renderImage          (src/albedo/render/render_image.hpp:36-49)
    resolve_srgb / write_ppm  encodeSrgb, toByte, writePpm (src/albedo/color/srgb.cpp:18-36,
                              src/albedo/image/ppm.cpp:22-85)
    Scene.intersect/occluded  Scene::intersect / occluded (src/albedo/scene/scene.hpp:69-88)

Errors raise the Python counterpart of the reference's exception: ValueError for
std::invalid_argument, SceneParseError for SceneParseError, OSError for
std::runtime_error (unreadable files), IndexError for std::out_of_range, and
DeviceError for CUDA failures. There is no CPU fallback: without the built
library, or without a CUDA device when one is needed, calls raise.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, byref, c_double, c_float, c_int32, c_uint32, c_void_p
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from ._lib import Accumulator, BasicMaterialC, CameraC, MaterialC, RenderJobC, SceneInfoC, TuningC, library

ACCUMULATOR_DTYPE = np.dtype([("r", "<f8"), ("g", "<f8"), ("b", "<f8"), ("count", "<i8")])

PATH, SCATTER_ONLY, NORMALS = 0, 1, 2
MEGAKERNEL, WAVEFRONT = 0, 1
ACCUMULATE_FP64, ACCUMULATE_KAHAN_FP32 = 0, 1


class SceneParseError(ValueError):
    """A scene file the reader rejects; the message names the line."""


class DeviceError(RuntimeError):
    """A CUDA call failed, or a kernel reported an error."""


class Unsupported(RuntimeError):
    """The scene exceeds a limit of the device layout."""


def _raise(status: int) -> None:
    if status == 0:
        return
    message = library().albedo_last_error().decode("utf-8", "replace")
    if status == 1:
        raise ValueError(message)
    if status == 2:
        raise SceneParseError(message)
    if status == 3:
        raise OSError(message)
    if status == 4:
        raise IndexError(message)
    if status == 6:
        raise MemoryError(message)
    if status == 7:
        raise Unsupported(message)
    raise DeviceError(message)


def _d3(values) -> ctypes.Array:
    return (c_double * 3)(*[float(v) for v in values])


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_float))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_int32))


@dataclass
class BasicMaterial:
    """BasicMaterial: kind "diffuse" (texture constant/checker/perlin), "conductor", "dielectric"."""

    kind: str = "diffuse"
    texture: str = "constant"
    a: tuple = (0.0, 0.0, 0.0)  # color / even / low, or conductor eta
    b: tuple = (0.0, 0.0, 0.0)  # odd / high, or conductor k
    frequency_or_scale: float = 1.0
    veins: float = 0.0
    ior: float = 1.5
    roughness: float = 0.0

    def to_c(self) -> BasicMaterialC:
        kinds = {"diffuse": 0, "conductor": 1, "dielectric": 2}
        textures = {"constant": 0, "checker": 1, "perlin": 2}
        c = BasicMaterialC()
        c.kind = kinds[self.kind]
        c.texture = textures[self.texture]
        c.a = (c_double * 3)(*self.a)
        c.b = (c_double * 3)(*self.b)
        c.frequency_or_scale = self.frequency_or_scale
        c.veins = self.veins
        c.ior = self.ior
        c.roughness = self.roughness
        return c


@dataclass
class RenderJob:
    """RenderJob without its camera and scene references; PathEstimator defaults."""

    width: int
    height: int
    samples_per_axis: int = 1
    seed: int = 0
    estimator: int = PATH
    max_depth: int = 64
    roulette_start: int = 3
    method: int = MEGAKERNEL
    accumulation: int = ACCUMULATE_FP64

    def to_c(self) -> RenderJobC:
        return RenderJobC(self.width, self.height, self.samples_per_axis, self.estimator, self.seed, self.max_depth,
                          self.roulette_start, self.method, self.accumulation)


@dataclass
class Camera:
    """CameraSettings (src/albedo/camera/perspective_camera.hpp:13-26) for one render."""

    look_from: tuple
    look_at: tuple
    up: tuple = (0.0, 1.0, 0.0)
    vertical_fov_degrees: float = 60.0

    def to_c(self) -> CameraC:
        c = CameraC()
        c.look_from[:] = [float(v) for v in self.look_from]
        c.look_at[:] = [float(v) for v in self.look_at]
        c.up[:] = [float(v) for v in self.up]
        c.vertical_fov_degrees = float(self.vertical_fov_degrees)
        return c


def _camera_ref(camera: Camera | None):
    return None if camera is None else byref(camera.to_c())


class PixelBuffer:
    """Per-pixel FP64 sums and sample counts, accumulated in place like PixelBuffer."""

    def __init__(self, width: int, height: int):
        if width <= 0 or height <= 0 or width * height > (1 << 28):
            raise ValueError(f"invalid image size {width}x{height}")
        self.width = width
        self.height = height
        self.pixels = np.zeros(width * height, dtype=ACCUMULATOR_DTYPE)

    def average(self) -> np.ndarray:
        """(H, W, 3) means; black where a pixel has no samples."""
        count = self.pixels["count"].astype(np.float64)
        rgb = np.stack([self.pixels["r"], self.pixels["g"], self.pixels["b"]], axis=-1)
        with np.errstate(invalid="ignore", divide="ignore"):
            avg = np.where(count[:, None] > 0, rgb / count[:, None], 0.0)
        return avg.reshape(self.height, self.width, 3)

    def write_ppm(self, path) -> None:
        """writePpm(path, image): resolved to sRGB bytes on the device."""
        _raise(library().albedo_save_ppm_host(str(path).encode(), self.pixels.ctypes.data_as(c_void_p),
                                              self.width, self.height))


class Scene:
    """A scene built on the host and, once committed, resident on the device."""

    def __init__(self, handle: int):
        self._handle = c_void_p(handle)

    @classmethod
    def create(cls) -> "Scene":
        handle = c_void_p()
        _raise(library().albedo_scene_create(byref(handle)))
        return cls(handle.value)

    @classmethod
    def read(cls, path) -> "Scene":
        """Parses a scene file and builds it on the host only (no device)."""
        handle = c_void_p()
        _raise(library().albedo_scene_read(str(path).encode(), byref(handle)))
        return cls(handle.value)

    @classmethod
    def load(cls, path) -> "Scene":
        """readScene and upload to the current CUDA device."""
        handle = c_void_p()
        _raise(library().albedo_scene_load(str(path).encode(), byref(handle)))
        return cls(handle.value)

    def close(self) -> None:
        if self._handle is not None and self._handle.value:
            library().albedo_scene_destroy(self._handle)
        self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> c_void_p:
        return self._handle

    # Scene building (mirrors Scene::add*, setSky and CameraSettings).
    def set_camera(self, look_from, look_at, up=(0.0, 1.0, 0.0), fov=60.0) -> None:
        _raise(library().albedo_scene_set_camera(self._handle, _d3(look_from), _d3(look_at), _d3(up), fov))

    def add_material(self, first: BasicMaterial, second: BasicMaterial | None = None, scale: float = 1.0,
                     veins: float = 0.0, threshold: float = 0.5) -> int:
        m = MaterialC()
        m.mix = 1 if second is not None else 0
        m.first = first.to_c()
        m.second = (second or first).to_c()
        m.scale, m.veins, m.threshold = scale, veins, threshold
        out = c_uint32()
        _raise(library().albedo_scene_add_material(self._handle, byref(m), byref(out)))
        return out.value

    def add_sphere(self, center, radius: float, material: int) -> int:
        out = c_uint32()
        _raise(library().albedo_scene_add_sphere(self._handle, _d3(center), radius, material, byref(out)))
        return out.value

    def add_area_light(self, center, radius: float, radiance, material: int) -> int:
        out = c_uint32()
        _raise(library().albedo_scene_add_area_light(self._handle, _d3(center), radius, _d3(radiance), material,
                                                     byref(out)))
        return out.value

    def add_point_light(self, position, intensity) -> None:
        _raise(library().albedo_scene_add_point_light(self._handle, _d3(position), _d3(intensity)))

    def set_sky(self, nadir, zenith=None) -> None:
        _raise(library().albedo_scene_set_sky(self._handle, _d3(nadir), _d3(zenith if zenith is not None else nadir)))

    def add_mesh(self, positions, faces, uvs=None, texture_faces=None, smooth=False) -> int:
        p = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        f = np.ascontiguousarray(faces, dtype=np.uint32).reshape(-1, 3)
        uv = np.ascontiguousarray(uvs if uvs is not None else np.zeros((0, 2)), dtype=np.float64).reshape(-1, 2)
        tf = np.ascontiguousarray(texture_faces if texture_faces is not None else np.zeros((0, 3)),
                                  dtype=np.uint32).reshape(-1, 3)
        out = c_uint32()
        _raise(library().albedo_scene_add_mesh(
            self._handle, p.ctypes.data_as(POINTER(c_double)), len(p), f.ctypes.data_as(POINTER(c_uint32)), len(f),
            uv.ctypes.data_as(POINTER(c_double)), len(uv), tf.ctypes.data_as(POINTER(c_uint32)), len(tf),
            1 if smooth else 0, byref(out)))
        return out.value

    def add_instance(self, mesh: int, to_world, to_object, material: int) -> int:
        w = (c_double * 12)(*np.asarray(to_world, dtype=np.float64).reshape(12))
        o = (c_double * 12)(*np.asarray(to_object, dtype=np.float64).reshape(12))
        out = c_uint32()
        _raise(library().albedo_scene_add_instance(self._handle, mesh, w, o, material, byref(out)))
        return out.value

    def add_triangles(self, positions, faces, material: int) -> None:
        p = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        f = np.ascontiguousarray(faces, dtype=np.uint32).reshape(-1, 3)
        _raise(library().albedo_scene_add_triangles(self._handle, p.ctypes.data_as(POINTER(c_double)), len(p),
                                                    f.ctypes.data_as(POINTER(c_uint32)), len(f), material))

    def prepare(self) -> None:
        _raise(library().albedo_scene_prepare(self._handle))

    def commit(self) -> None:
        _raise(library().albedo_scene_commit(self._handle))

    def info(self) -> dict:
        info = SceneInfoC()
        _raise(library().albedo_scene_get_info(self._handle, byref(info)))
        return {name: getattr(info, name) for name, _ in SceneInfoC._fields_}

    # Ray queries.
    def intersect(self, rays: np.ndarray, t_min: float = 0.0, t_max: float = float("inf"), geometry: bool = False):
        """Closest hits of (N, 6) float32 rays: dict of hit, t, object, triangle [, point, normal, ...]."""
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = len(rays)
        out = {"hit": np.zeros(n, np.int32), "t": np.zeros(n, np.float32), "object": np.full(n, -1, np.int32),
               "triangle": np.full(n, -1, np.int32)}
        extra = {}
        if geometry:
            extra = {"point": np.zeros((n, 3), np.float32), "normal": np.zeros((n, 3), np.float32),
                     "shading_normal": np.zeros((n, 3), np.float32), "front": np.zeros(n, np.int32)}
        _raise(library().albedo_trace_host(
            self._handle, _fptr(rays), n, t_min, t_max, _iptr(out["hit"]), _fptr(out["t"]), _iptr(out["object"]),
            _iptr(out["triangle"]), _fptr(extra["point"]) if geometry else None,
            _fptr(extra["normal"]) if geometry else None, _fptr(extra["shading_normal"]) if geometry else None,
            _iptr(extra["front"]) if geometry else None))
        out.update(extra)
        return out

    def occluded(self, rays: np.ndarray, t_max: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        t_max = np.ascontiguousarray(t_max, dtype=np.float32).reshape(-1)
        out = np.zeros(len(rays), np.int32)
        _raise(library().albedo_occluded_host(self._handle, _fptr(rays), _fptr(t_max), len(rays), _iptr(out)))
        return out

    def check(self) -> None:
        """Collects a kernel-reported error after asynchronous renders."""
        _raise(library().albedo_scene_check(self._handle))


def read_scene(path) -> Scene:
    """readScene(path), resident on the current CUDA device."""
    return Scene.load(path)


def render_image(scene: Scene, job: RenderJob, image: PixelBuffer) -> None:
    """renderImage: adds samples_per_axis^2 samples to every pixel of `image`."""
    if (image.width, image.height) != (job.width, job.height):
        raise ValueError("image size does not match the job")
    c = job.to_c()
    _raise(library().albedo_render_host(scene.handle, byref(c), image.pixels.ctypes.data_as(c_void_p)))


def render_image_ptr(scene: Scene, job: RenderJob, host_accumulators_ptr: int) -> None:
    """renderImage into a host array (pinned or pageable) of width*height accumulators."""
    c = job.to_c()
    _raise(library().albedo_render_host(scene.handle, byref(c), c_void_p(host_accumulators_ptr)))


def render_device(scene: Scene, job: RenderJob, accumulators_ptr: int, stream: int = 0,
                  camera: Camera | None = None) -> None:
    """Stream-ordered render into a device array of width*height accumulators,
    from `camera` instead of the scene's when given."""
    c = job.to_c()
    if camera is None:
        _raise(library().albedo_render(scene.handle, byref(c), c_void_p(accumulators_ptr), c_void_p(stream)))
    else:
        _raise(library().albedo_render_view(scene.handle, byref(c), _camera_ref(camera), c_void_p(accumulators_ptr),
                                            c_void_p(stream)))


def resolve_srgb(accumulators_ptr: int, width: int, height: int, out_ptr: int, stream: int = 0) -> None:
    """Stream-ordered resolve of width*height device accumulators into
    width*height*3 device bytes: the sRGB bytes writePpm writes for each pixel's
    average, rows from the top (image/ppm.cpp:22-33)."""
    _raise(library().albedo_resolve_srgb(c_void_p(accumulators_ptr), width, height, c_void_p(out_ptr),
                                         c_void_p(stream)))


SRGB_BUCKET_SHIFT, SRGB_BUCKET_BASE, SRGB_BUCKETS = 45, (1023 - 13) * 128, 13 * 128


def srgb_tables() -> tuple[np.ndarray, np.ndarray]:
    """The resolve's tables: lower[b] is the smallest positive double whose byte
    is at least b (b = 1..255; lower[0] is -inf), and start[k] the byte at the
    smallest double of bucket k (bits >> SRGB_BUCKET_SHIFT == SRGB_BUCKET_BASE + k)."""
    lower = np.empty(256, dtype=np.float64)
    start = np.empty(SRGB_BUCKETS, dtype=np.uint8)
    _raise(library().albedo_srgb_tables(lower.ctypes.data_as(POINTER(c_double)), start.ctypes.data_as(c_void_p)))
    return lower, start


def srgb_thresholds() -> np.ndarray:
    """lower of srgb_tables()."""
    return srgb_tables()[0]


def write_ppm(path, rgb: np.ndarray) -> None:
    """writePpm from host sRGB bytes of shape (height, width, 3)."""
    rgb = np.ascontiguousarray(rgb, dtype=np.uint8)
    if rgb.ndim != 3 or rgb.shape[2] != 3:
        raise ValueError("rgb must have shape (height, width, 3)")
    _raise(library().albedo_write_ppm(str(path).encode(), rgb.ctypes.data_as(c_void_p), rgb.shape[1], rgb.shape[0]))


def save_ppm(path, accumulators_ptr: int, width: int, height: int, stream: int = 0) -> None:
    """writePpm for device accumulators: resolved on `stream`, then written."""
    _raise(library().albedo_save_ppm(str(path).encode(), c_void_p(accumulators_ptr), width, height,
                                     c_void_p(stream)))


def _batch_array(items):
    from ._lib import BatchItemC

    array = (BatchItemC * len(items))()
    for i, (scene, job, ptr) in enumerate(items):
        array[i].scene = scene.handle.value
        array[i].job = job.to_c()
        array[i].accumulators = ptr
    return array


def render_batch(items, stream: int = 0) -> None:
    """Renders [(scene, job, device_accumulators_ptr), ...] in one wavefront run."""
    _raise(library().albedo_render_batch(_batch_array(items), len(items), c_void_p(stream)))


_TUNING_FIELDS = ["tile_width", "blocks_per_sm", "trace_blocks_per_sm", "fetch_batch", "iterations_per_graph",
                  "slot_count", "inline_traversal", "trace_loop", "ray_sort", "evaluations", "best_ms", "default_ms"]


def _tuning_dict(t: TuningC) -> dict:
    return {k: getattr(t, k) for k in _TUNING_FIELDS}


def autotune_megakernel(scene: Scene, job: RenderJob) -> dict:
    """Times every megakernel shape (tile width x register budget) on `job` at a
    quarter of its samples and keeps the fastest for `scene`."""
    out = TuningC()
    c = job.to_c()
    _raise(library().albedo_autotune_megakernel(scene.handle, byref(c), byref(out)))
    return _tuning_dict(out)


def autotune_batch(items) -> dict:
    """Tunes the wavefront engine's shape on [(scene, job, ptr), ...] (the
    accumulators are not touched) and keeps it for later batches and servers."""
    out = TuningC()
    _raise(library().albedo_autotune_batch(_batch_array(items), len(items), byref(out)))
    return _tuning_dict(out)


def set_tuning(scene: Scene | None = None, **shape) -> None:
    """Pins a launch shape: tile_width, blocks_per_sm and inline_traversal for a scene's megakernel,
    or (no scene) blocks_per_sm, trace_blocks_per_sm, fetch_batch, trace_loop, ray_sort,
    iterations_per_graph and slot_count for the wavefront engine."""
    t = TuningC()
    for k, v in shape.items():
        if k not in _TUNING_FIELDS[:9]:
            raise ValueError(f"unknown shape field {k}")
        setattr(t, k, int(v))
    _raise(library().albedo_tuning_set(None if scene is None else scene.handle, byref(t)))


def tuning(scene: Scene | None = None) -> dict:
    """The shape renders use now: the scene's megakernel shape, or (no scene) the wavefront engine's."""
    out = TuningC()
    _raise(library().albedo_tuning_get(None if scene is None else scene.handle, byref(out)))
    return _tuning_dict(out)


class Server:
    """Continuous-batching render server (albedo_server_* in the C ABI)."""

    def __init__(self, memory_budget_bytes: int = 150 << 30, slots: int = 1 << 20, express_pixels: int = 65536):
        """`express_pixels`: requests of at most this many pixels may be rendered by the
        megakernel beside a lightly loaded batch (0: every request joins the batch)."""
        handle = c_void_p()
        _raise(library().albedo_server_create(memory_budget_bytes, slots, byref(handle)))
        self._handle = handle
        _raise(library().albedo_server_set_express(self._handle, express_pixels))

    def submit(self, scene: Scene, job: RenderJob, accumulators_ptr: int, camera: Camera | None = None) -> int:
        c = job.to_c()
        ticket = ctypes.c_int64()
        _raise(library().albedo_server_submit_view(self._handle, scene.handle, byref(c), _camera_ref(camera),
                                                   c_void_p(accumulators_ptr), byref(ticket)))
        return ticket.value

    def step(self, capacity: int = 4096) -> list[int]:
        out = (ctypes.c_int64 * capacity)()
        count = c_int32()
        _raise(library().albedo_server_step(self._handle, out, capacity, byref(count)))
        return [out[i] for i in range(count.value)]

    def routes(self) -> tuple[int, int]:
        """Requests admitted so far (to the batch, to the express route)."""
        batched, express = ctypes.c_int64(), ctypes.c_int64()
        _raise(library().albedo_server_routes(self._handle, byref(batched), byref(express)))
        return batched.value, express.value

    def release_scene(self, scene: Scene) -> None:
        """Stops counting `scene` against the budget; it must have no requests left in the server."""
        _raise(library().albedo_server_release_scene(self._handle, scene.handle))

    def rays(self) -> int:
        """Ray queries the current batch has traced as of the last polled step."""
        out = ctypes.c_int64()
        _raise(library().albedo_server_rays(self._handle, byref(out)))
        return out.value

    def pending(self) -> tuple[int, int]:
        waiting, running = c_int32(), c_int32()
        _raise(library().albedo_server_pending(self._handle, byref(waiting), byref(running)))
        return waiting.value, running.value

    def close(self) -> None:
        if self._handle is not None and self._handle.value:
            library().albedo_server_destroy(self._handle)
        self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def wavefront_configure(slots: int = 1 << 20, blocks_per_sm: int = 8, iterations_per_graph: int = 4) -> None:
    """Shape of the wavefront engine: path slots, queue-kernel blocks per SM, iterations per graph."""
    _raise(library().albedo_wavefront_configure(slots, blocks_per_sm, iterations_per_graph))


def wavefront_last_iterations() -> int:
    out = ctypes.c_int64()
    _raise(library().albedo_wavefront_last_iterations(byref(out)))
    return out.value


def wavefront_last_rays() -> int:
    """Ray queries (closest hit plus shadow) the last wavefront run traced."""
    out = ctypes.c_int64()
    _raise(library().albedo_wavefront_last_rays(byref(out)))
    return out.value


_COUNT_NAMES = ["boxes", "triangles", "spheres", "instances", "rays", "reference_boxes"]


def work_counts(scene: Scene, job: RenderJob) -> dict:
    """Traversal work of one render of `job` (path estimator), counted on the device:
    child boxes the 4-wide traversal tested, triangles, spheres, instances entered,
    queries, and the boxes the reference's binary traversal tests for the same queries."""
    out = (ctypes.c_int64 * 6)()
    c = job.to_c()
    _raise(library().albedo_render_work_counts(scene.handle, byref(c), out))
    return dict(zip(_COUNT_NAMES, [int(v) for v in out]))


def trace_work_counts(scene: Scene, rays: np.ndarray, t_min: float = 0.0, t_max: float = float("inf")) -> dict:
    """The same counts for closest-hit queries of (N, 6) float32 rays."""
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
    out = (ctypes.c_int64 * 6)()
    _raise(library().albedo_trace_counts_host(scene.handle, _fptr(rays), len(rays), t_min, t_max, out))
    return dict(zip(_COUNT_NAMES, [int(v) for v in out]))


def algorithmic_bytes(counts: dict, boxes: str = "reference_boxes") -> int:
    """Bytes the reference's traversal must read for the counted work: 32 per box
    it tests (by default the boxes its binary traversal tests; `boxes="boxes"`
    counts the 4-wide traversal's child boxes instead), 48 per triangle, 32 per
    sphere (its 16-byte record and its object entry), 96 per instance entered
    (its two 3x4 FP32 transforms)."""
    return 32 * counts[boxes] + 48 * counts["triangles"] + 32 * counts["spheres"] + 96 * counts["instances"]


def read_sweep(data_ptr: int, nbytes: int, repeats: int, blocks: int, sink_ptr: int, stream: int = 0) -> None:
    """Reads `nbytes` of device memory `repeats` times through L2 (asynchronous;
    the caller times it): the L2 read bandwidth probe."""
    _raise(library().albedo_probe_read_sweep(c_void_p(data_ptr), nbytes, repeats, blocks, c_void_p(sink_ptr),
                                             c_void_p(stream)))


def render_pixels(scene: Scene, job: RenderJob, pixels: np.ndarray, with_squares: bool = False):
    """Renders only the listed (x, y) pixels; returns accumulators (and sums of squares)."""
    pixels = np.ascontiguousarray(pixels, dtype=np.int32).reshape(-1, 2)
    acc = np.zeros(len(pixels), dtype=ACCUMULATOR_DTYPE)
    squares = np.zeros((len(pixels), 3), np.float64) if with_squares else None
    c = job.to_c()
    _raise(library().albedo_render_pixels_host(
        scene.handle, byref(c), _iptr(pixels), len(pixels), acc.ctypes.data_as(c_void_p),
        squares.ctypes.data_as(POINTER(c_double)) if with_squares else None))
    return (acc, squares) if with_squares else acc


__all__ = [
    "ACCUMULATE_FP64", "ACCUMULATE_KAHAN_FP32", "ACCUMULATOR_DTYPE", "BasicMaterial", "Camera", "DeviceError",
    "MEGAKERNEL", "NORMALS", "PATH", "PixelBuffer", "RenderJob", "SCATTER_ONLY", "Scene", "SceneParseError",
    "Server", "Unsupported", "WAVEFRONT", "read_scene", "render_batch", "render_device", "render_image",
    "render_pixels", "Accumulator", "autotune_batch", "autotune_megakernel", "resolve_srgb", "save_ppm",
    "read_sweep", "set_tuning", "srgb_tables", "srgb_thresholds", "trace_work_counts", "tuning", "wavefront_last_rays", "write_ppm",
]
