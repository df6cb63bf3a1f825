"""Test infrastructure: ctypes access to the FP64 restatement of the reference's
ray-query path (trace_oracle.cpp), run over this repository's host scene tables."""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int, c_int32, c_int64, c_void_p
from pathlib import Path

import numpy as np

LIBRARY = Path(__file__).resolve().parent / "_build" / "libtrace_oracle.so"
_lib = None

_D = POINTER(c_double)
_I32 = POINTER(c_int32)
_I64 = POINTER(c_int64)


def available() -> bool:
    return LIBRARY.exists()


def lib():
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise RuntimeError(f"{LIBRARY} is missing; build it with `make -C oracle restatement`")
        l = ctypes.CDLL(str(LIBRARY))
        l.oracle_intersect.restype = None
        l.oracle_intersect.argtypes = [c_void_p, _D, c_int64, c_double, c_double, c_int, _I32, _D, _I64, _I64, _D, _D,
                                       _D, _I32, _I64]
        l.oracle_classify.restype = None
        l.oracle_classify.argtypes = [c_void_p, _D, c_int64, c_double, c_double, c_double, c_int, _I32, _I64, _I64,
                                      _I32, _D]
        _lib = l
    return _lib


def intersect(scene, rays: np.ndarray, t_min=0.0, t_max=float("inf"), threads: int = 8) -> dict:
    """Closest hits over an albedo_b200.Scene's host tables, with work counts per ray
    (boxes as the reference tests them, triangles, spheres, instances)."""
    from albedo_b200._lib import library

    view = library().albedo_scene_host_view(scene.handle)
    rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 6)
    n = len(rays)
    out = {"hit": np.zeros(n, np.int32), "t": np.zeros(n), "object": np.full(n, -1, np.int64),
           "triangle": np.full(n, -1, np.int64), "point": np.zeros((n, 3)), "normal": np.zeros((n, 3)),
           "shading_normal": np.zeros((n, 3)), "front": np.zeros(n, np.int32), "counts": np.zeros((n, 4), np.int64)}
    lib().oracle_intersect(view, rays.ctypes.data_as(_D), n, t_min, t_max, threads, out["hit"].ctypes.data_as(_I32),
                           out["t"].ctypes.data_as(_D), out["object"].ctypes.data_as(_I64),
                           out["triangle"].ctypes.data_as(_I64), out["point"].ctypes.data_as(_D),
                           out["normal"].ctypes.data_as(_D), out["shading_normal"].ctypes.data_as(_D),
                           out["front"].ctypes.data_as(_I32), out["counts"].ctypes.data_as(_I64))
    return out


# The FP32 error bound of the near-tie classification, in units of 2^-24 times
# the largest coordinate magnitude involved (see trace_oracle.cpp).
TIE_ULPS = 32.0


def classify(scene, rays: np.ndarray, device: dict, t_min=0.0, t_max=float("inf"), ulps=TIE_ULPS,
             threads: int = 8) -> dict:
    """Classifies device closest-hit answers (dict with hit, object, triangle) against
    the FP64 restatement: class 0 = the FP64 answer, 1 = a near-tie FP32 rounding
    explains, 2 = unexplained; `detail` as oracle_classify documents it."""
    from albedo_b200._lib import library

    view = library().albedo_scene_host_view(scene.handle)
    rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 6)
    n = len(rays)
    hit = np.ascontiguousarray(device["hit"], dtype=np.int32)
    obj = np.ascontiguousarray(device["object"], dtype=np.int64)
    tri = np.ascontiguousarray(device["triangle"], dtype=np.int64)
    out = np.zeros(n, np.int32)
    detail = np.zeros((n, 4))
    lib().oracle_classify(view, rays.ctypes.data_as(_D), n, t_min, t_max, ulps, threads, hit.ctypes.data_as(_I32),
                          obj.ctypes.data_as(_I64), tri.ctypes.data_as(_I64), out.ctypes.data_as(_I32),
                          detail.ctypes.data_as(_D))
    return {"class": out, "detail": detail}
