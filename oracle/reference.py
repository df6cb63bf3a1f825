"""Test infrastructure: ctypes access to the reference renderer built from its own
sources (oracle/_ref/libalbedo_ref.so, see oracle/Makefile and ref_driver.cpp).

Only tests, the smoke check and bench.py's CPU-baseline legs use this module; the
product never imports it. The library is built in the development container
(where the reference checkout exists) and travels prebuilt to GPU machines.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_uint32, c_uint64, c_void_p
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
REF_LIBRARY = ORACLE_DIR / "_ref" / "libalbedo_ref.so"

_D = POINTER(c_double)
_I32 = POINTER(c_int32)
_I64 = POINTER(c_int64)

_PROTOTYPES = {
    "ref_last_error": (c_char_p, []),
    "ref_available_threads": (c_int, []),
    "ref_scene_load": (c_void_p, [c_char_p]),
    "ref_scene_free": (None, [c_void_p]),
    "ref_scene_create": (c_void_p, []),
    "ref_scene_add_triangles": (c_int, [c_void_p, _D, c_int64, _I64, c_int64]),
    "ref_scene_add_sphere": (c_int, [c_void_p, _D, c_double]),
    "ref_scene_object_count": (c_int64, [c_void_p]),
    "ref_render_image": (c_int, [c_void_p, c_int, c_int, c_int, c_uint64, c_int, c_int, c_int, _D]),
    "ref_render_pixels": (c_int, [c_void_p, c_int, c_int, c_int, c_uint64, c_int, c_int, c_int, c_int, _I32, c_int64,
                                  _D, _D]),
    "ref_intersect": (c_int, [c_void_p, _D, c_int64, c_double, c_double, c_int, _I32, _D, _I64, _D, _D, _D, _I32, _D]),
    "ref_occluded": (c_int, [c_void_p, _D, _D, c_int64, c_int, _I32]),
    "ref_camera_rays": (c_int, [c_void_p, c_int, c_int, _D, c_int64, _D]),
    "ref_pcg32": (None, [c_uint64, c_uint64, c_int64, POINTER(c_uint32)]),
    "ref_pixel_stream": (None, [c_uint64, c_int, c_int, c_int, c_int64, _D]),
    "ref_perlin_noise": (None, [_D, c_int64, _D, _D]),
    "ref_lobe_eval": (c_int, [c_int, _D, _D, c_int64, _D, _D]),
    "ref_lobe_sample": (c_int, [c_int, _D, _D, c_int64, _I32, _D, _D, _D, _I32]),
    "ref_fresnel_dielectric": (None, [_D, _D, c_int64, _D]),
    "ref_fresnel_conductor": (None, [_D, c_int64, _D, _D]),
    "ref_sphere_intersect": (None, [_D, _D, c_int64, c_double, c_double, _I32, _D]),
    "ref_triangle_intersect": (None, [_D, _D, c_int64, c_double, c_double, _I32, _D]),
    "ref_warps": (None, [_D, c_int64, _D, _D]),
    "ref_srgb_bytes": (None, [_D, c_int64, POINTER(ctypes.c_uint8)]),
    "ref_write_ppm": (c_int, [c_char_p, c_int, c_int, _D]),
}

_lib = None


def available() -> bool:
    return REF_LIBRARY.exists()


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not REF_LIBRARY.exists():
            raise RuntimeError(f"{REF_LIBRARY} is missing; build it with `make -C oracle ref`")
        l = ctypes.CDLL(str(REF_LIBRARY))
        for name, (restype, argtypes) in _PROTOTYPES.items():
            fn = getattr(l, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = l
    return _lib


def _d(a: np.ndarray):
    return a.ctypes.data_as(_D)


def _check(status: int) -> None:
    if status != 0:
        raise RuntimeError(lib().ref_last_error().decode())


def threads() -> int:
    return int(lib().ref_available_threads())


class RefScene:
    """A scene read by the reference's readScene."""

    def __init__(self, path):
        handle = lib().ref_scene_load(str(path).encode())
        if not handle:
            raise RuntimeError(lib().ref_last_error().decode())
        self.handle = c_void_p(handle)

    @classmethod
    def create(cls) -> "RefScene":
        """An empty Scene filled by add_triangles / add_sphere (Scene::add)."""
        scene = cls.__new__(cls)
        handle = lib().ref_scene_create()
        if not handle:
            raise RuntimeError(lib().ref_last_error().decode())
        scene.handle = c_void_p(handle)
        return scene

    def add_triangles(self, positions: np.ndarray, faces: np.ndarray) -> None:
        """Scene::add(TriangleMesh, material): every triangle its own object."""
        positions = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        faces = np.ascontiguousarray(faces, dtype=np.int64).reshape(-1, 3)
        _check(lib().ref_scene_add_triangles(self.handle, _d(positions), len(positions), faces.ctypes.data_as(_I64),
                                             len(faces)))

    def add_sphere(self, center, radius: float) -> None:
        c = np.ascontiguousarray(center, dtype=np.float64)
        _check(lib().ref_scene_add_sphere(self.handle, _d(c), float(radius)))

    def __del__(self):
        if getattr(self, "handle", None) is not None and lib is not None:
            lib().ref_scene_free(self.handle)
            self.handle = None

    def object_count(self) -> int:
        return int(lib().ref_scene_object_count(self.handle))

    def render_image(self, width, height, n, seed=0, max_depth=64, roulette_start=3, nthreads=None) -> np.ndarray:
        """renderImage: (H, W, 3) averages."""
        out = np.zeros((height, width, 3), np.float64)
        _check(lib().ref_render_image(self.handle, width, height, n, seed, max_depth, roulette_start,
                                      nthreads or threads(), _d(out)))
        return out

    def render_pixels(self, width, height, n, pixels, seed=0, estimator=0, max_depth=64, roulette_start=3,
                      nthreads=None):
        """Sums and sums of squares of n^2 samples for each listed (x, y) pixel."""
        pixels = np.ascontiguousarray(pixels, dtype=np.int32).reshape(-1, 2)
        sums = np.zeros((len(pixels), 3), np.float64)
        squares = np.zeros((len(pixels), 3), np.float64)
        _check(lib().ref_render_pixels(self.handle, width, height, n, seed, estimator, max_depth, roulette_start,
                                       nthreads or threads(), pixels.ctypes.data_as(_I32), len(pixels), _d(sums),
                                       _d(squares)))
        return sums, squares

    def intersect(self, rays: np.ndarray, t_min=0.0, t_max=float("inf"), nthreads=None) -> dict:
        rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 6)
        n = len(rays)
        out = {"hit": np.zeros(n, np.int32), "t": np.zeros(n), "object": np.full(n, -1, np.int64),
               "point": np.zeros((n, 3)), "normal": np.zeros((n, 3)), "shading_normal": np.zeros((n, 3)),
               "front": np.zeros(n, np.int32), "uv": np.zeros((n, 2))}
        _check(lib().ref_intersect(self.handle, _d(rays), n, t_min, t_max, nthreads or threads(),
                                   out["hit"].ctypes.data_as(_I32), _d(out["t"]), out["object"].ctypes.data_as(_I64),
                                   _d(out["point"]), _d(out["normal"]), _d(out["shading_normal"]),
                                   out["front"].ctypes.data_as(_I32), _d(out["uv"])))
        return out

    def occluded(self, rays: np.ndarray, t_max: np.ndarray, nthreads=None) -> np.ndarray:
        rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 6)
        t_max = np.ascontiguousarray(t_max, dtype=np.float64)
        out = np.zeros(len(rays), np.int32)
        _check(lib().ref_occluded(self.handle, _d(rays), _d(t_max), len(rays), nthreads or threads(),
                                  out.ctypes.data_as(_I32)))
        return out

    def camera_rays(self, width, height, film: np.ndarray) -> np.ndarray:
        film = np.ascontiguousarray(film, dtype=np.float64).reshape(-1, 2)
        out = np.zeros((len(film), 6))
        _check(lib().ref_camera_rays(self.handle, width, height, _d(film), len(film), _d(out)))
        return out


def pcg32(seed: int, stream: int, count: int) -> np.ndarray:
    out = np.zeros(count, np.uint32)
    lib().ref_pcg32(seed, stream, count, out.ctypes.data_as(POINTER(c_uint32)))
    return out


def pixel_stream(seed: int, x: int, y: int, width: int, count: int) -> np.ndarray:
    out = np.zeros(count, np.float64)
    lib().ref_pixel_stream(seed, x, y, width, count, _d(out))
    return out


def perlin(points: np.ndarray):
    points = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    noise = np.zeros(len(points))
    turb = np.zeros(len(points))
    lib().ref_perlin_noise(_d(points), len(points), _d(noise), _d(turb))
    return noise, turb


def lobe_eval(kind: int, params, wo_wi: np.ndarray):
    params = np.ascontiguousarray(params, dtype=np.float64)
    wo_wi = np.ascontiguousarray(wo_wi, dtype=np.float64).reshape(-1, 6)
    f = np.zeros((len(wo_wi), 3))
    pdf = np.zeros(len(wo_wi))
    _check(lib().ref_lobe_eval(kind, _d(params), _d(wo_wi), len(wo_wi), _d(f), _d(pdf)))
    return f, pdf


def lobe_sample(kind: int, params, inputs: np.ndarray):
    params = np.ascontiguousarray(params, dtype=np.float64)
    inputs = np.ascontiguousarray(inputs, dtype=np.float64).reshape(-1, 6)
    n = len(inputs)
    valid = np.zeros(n, np.int32)
    direction = np.zeros((n, 3))
    weight = np.zeros((n, 3))
    pdf = np.zeros(n)
    specular = np.zeros(n, np.int32)
    _check(lib().ref_lobe_sample(kind, _d(params), _d(inputs), n, valid.ctypes.data_as(_I32), _d(direction),
                                 _d(weight), _d(pdf), specular.ctypes.data_as(_I32)))
    return valid, direction, weight, pdf, specular


def srgb_bytes(linear: np.ndarray) -> np.ndarray:
    """The reference's toByte(encodeSrgb(x)) per value (color/srgb.cpp:18-36)."""
    linear = np.ascontiguousarray(linear, dtype=np.float64)
    out = np.empty(linear.shape, dtype=np.uint8)
    lib().ref_srgb_bytes(_d(linear), linear.size, out.ctypes.data_as(POINTER(ctypes.c_uint8)))
    return out


def write_ppm(path, averages: np.ndarray) -> None:
    """The reference's writePpm of an image whose pixel averages are `averages`
    (shape (H, W, 3)); raises RuntimeError with its message on failure."""
    averages = np.ascontiguousarray(averages, dtype=np.float64)
    h, w, _ = averages.shape
    _check(lib().ref_write_ppm(str(path).encode(), w, h, _d(averages)))
