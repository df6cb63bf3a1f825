"""Test infrastructure: ctypes access to the C++ adapter harness
(tests/cpp/adapter_check.cpp, built by `make -C oracle adapter` into
oracle/_ref/libadapter_check.so against the reference's headers and library).
Only tests use it."""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_int, c_int64, c_uint64
from pathlib import Path

import numpy as np

LIBRARY = Path(__file__).resolve().parent / "_ref" / "libadapter_check.so"
_lib = None


def available() -> bool:
    return LIBRARY.exists()


def lib():
    global _lib
    if _lib is None:
        l = ctypes.CDLL(str(LIBRARY))
        l.adapter_message.restype = c_char_p
        l.adapter_camera.restype = c_int
        l.adapter_camera.argtypes = [c_char_p, c_int, c_int, POINTER(c_double)]
        l.adapter_render.restype = c_int
        l.adapter_render.argtypes = [c_char_p, c_int, c_int, c_int, c_int, c_int, c_int, c_uint64, c_int, c_int, c_int,
                                     c_int, POINTER(c_double), POINTER(c_int64), POINTER(c_int)]
        _lib = l
    return _lib


def camera(path, width: int, height: int) -> tuple[np.ndarray, np.ndarray]:
    """(recovered, file) camera settings: look_from, look_at, up, fov (10 values each)."""
    out = np.zeros(20)
    if lib().adapter_camera(str(path).encode(), width, height, out.ctypes.data_as(POINTER(c_double))) != 0:
        raise RuntimeError(lib().adapter_message().decode())
    return out[:10], out[10:]


def render(path, *, gpu: bool, width: int, height: int, samples_per_axis: int, seed: int = 0, estimator: int = 0,
           max_depth: int = 64, thread_count: int = 8, bind: bool = True, camera_width: int | None = None,
           prior_samples: int = 0):
    """renderImage through the adapter (gpu) or the reference: ("ok", (H, W, 3)
    averages) or ("error", kind, message) with kind 1 invalid_argument, 2
    runtime_error, 3 another exception."""
    out = np.zeros((height, width, 3))
    count = c_int64(0)
    kind = c_int(0)
    status = lib().adapter_render(str(path).encode(), int(gpu), int(bind), width, height,
                                  camera_width if camera_width is not None else width, samples_per_axis, seed,
                                  estimator, max_depth, thread_count, prior_samples,
                                  out.ctypes.data_as(POINTER(c_double)), ctypes.byref(count), ctypes.byref(kind))
    if status != 0:
        return "error", kind.value, lib().adapter_message().decode()
    return "ok", out
