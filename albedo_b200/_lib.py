"""Loads libalbedo_b200.so (built in-tree) and declares the C ABI of include/albedo_b200.h."""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_float, c_int32, c_int64, c_uint32, c_uint64, c_void_p
from pathlib import Path

LIBRARY_PATH = Path(__file__).resolve().parent / "libalbedo_b200.so"


class Accumulator(ctypes.Structure):
    _fields_ = [("r", c_double), ("g", c_double), ("b", c_double), ("count", c_int64)]


class RenderJobC(ctypes.Structure):
    _fields_ = [("width", c_int32), ("height", c_int32), ("samples_per_axis", c_int32), ("estimator", c_int32),
                ("seed", c_uint64), ("max_depth", c_int32), ("roulette_start", c_int32), ("method", c_int32),
                ("accumulation", c_int32)]


class CameraC(ctypes.Structure):
    _fields_ = [("look_from", c_double * 3), ("look_at", c_double * 3), ("up", c_double * 3),
                ("vertical_fov_degrees", c_double)]


class TuningC(ctypes.Structure):
    _fields_ = [("tile_width", c_int32), ("blocks_per_sm", c_int32), ("trace_blocks_per_sm", c_int32),
                ("fetch_batch", c_int32), ("iterations_per_graph", c_int32), ("slot_count", c_int32),
                ("evaluations", c_int32), ("inline_traversal", c_int32), ("trace_loop", c_int32),
                ("ray_sort", c_int32), ("best_ms", c_double), ("default_ms", c_double)]


class BatchItemC(ctypes.Structure):
    _fields_ = [("scene", c_void_p), ("job", RenderJobC), ("accumulators", c_void_p)]


class BasicMaterialC(ctypes.Structure):
    _fields_ = [("kind", c_int32), ("texture", c_int32), ("a", c_double * 3), ("b", c_double * 3),
                ("frequency_or_scale", c_double), ("veins", c_double), ("ior", c_double), ("roughness", c_double)]


class MaterialC(ctypes.Structure):
    _fields_ = [("mix", c_int32), ("reserved", c_int32), ("first", BasicMaterialC), ("second", BasicMaterialC),
                ("scale", c_double), ("veins", c_double), ("threshold", c_double)]


class SceneInfoC(ctypes.Structure):
    _fields_ = [("objects", c_int64), ("lights", c_int64), ("triangles", c_int64), ("nodes", c_int64),
                ("device_bytes", c_int64), ("stack_need", c_int32), ("stack_capacity", c_int32)]


_D3 = POINTER(c_double)
_F = POINTER(c_float)
_I = POINTER(c_int32)
_U = POINTER(c_uint32)

# name -> (restype, argtypes); every symbol include/albedo_b200.h declares.
PROTOTYPES: dict[str, tuple] = {
    "albedo_last_error": (c_char_p, []),
    "albedo_scene_load": (c_int32, [c_char_p, POINTER(c_void_p)]),
    "albedo_scene_read": (c_int32, [c_char_p, POINTER(c_void_p)]),
    "albedo_scene_create": (c_int32, [POINTER(c_void_p)]),
    "albedo_scene_destroy": (None, [c_void_p]),
    "albedo_scene_set_camera": (c_int32, [c_void_p, _D3, _D3, _D3, c_double]),
    "albedo_scene_add_material": (c_int32, [c_void_p, POINTER(MaterialC), _U]),
    "albedo_scene_add_sphere": (c_int32, [c_void_p, _D3, c_double, c_uint32, _U]),
    "albedo_scene_add_area_light": (c_int32, [c_void_p, _D3, c_double, _D3, c_uint32, _U]),
    "albedo_scene_add_point_light": (c_int32, [c_void_p, _D3, _D3]),
    "albedo_scene_set_sky": (c_int32, [c_void_p, _D3, _D3]),
    "albedo_scene_add_mesh": (c_int32, [c_void_p, _D3, c_int64, _U, c_int64, _D3, c_int64, _U, c_int64, c_int32, _U]),
    "albedo_scene_add_instance": (c_int32, [c_void_p, c_uint32, _D3, _D3, c_uint32, _U]),
    "albedo_scene_add_triangles": (c_int32, [c_void_p, _D3, c_int64, _U, c_int64, c_uint32]),
    "albedo_scene_prepare": (c_int32, [c_void_p]),
    "albedo_scene_commit": (c_int32, [c_void_p]),
    "albedo_scene_host_view": (c_void_p, [c_void_p]),
    "albedo_scene_get_info": (c_int32, [c_void_p, POINTER(SceneInfoC)]),
    "albedo_render": (c_int32, [c_void_p, POINTER(RenderJobC), c_void_p, c_void_p]),
    "albedo_render_host": (c_int32, [c_void_p, POINTER(RenderJobC), c_void_p]),
    "albedo_render_view": (c_int32, [c_void_p, POINTER(RenderJobC), POINTER(CameraC), c_void_p, c_void_p]),
    "albedo_probe_read_sweep": (c_int32, [c_void_p, c_int64, c_int32, c_int32, c_void_p, c_void_p]),
    "albedo_render_view_host": (c_int32, [c_void_p, POINTER(RenderJobC), POINTER(CameraC), c_void_p]),
    "albedo_render_pixels_host": (c_int32, [c_void_p, POINTER(RenderJobC), _I, c_int64, c_void_p, _D3]),
    "albedo_scene_check": (c_int32, [c_void_p]),
    "albedo_render_work_counts": (c_int32, [c_void_p, POINTER(RenderJobC), POINTER(c_int64)]),
    "albedo_trace_counts_host": (c_int32, [c_void_p, _F, c_int64, c_float, c_float, POINTER(c_int64)]),
    "albedo_render_batch": (c_int32, [c_void_p, c_int32, c_void_p]),
    "albedo_render_noalloc": (c_int32, [c_void_p, POINTER(RenderJobC), c_void_p, c_void_p]),
    "albedo_resolve_srgb": (c_int32, [c_void_p, c_int32, c_int32, c_void_p, c_void_p]),
    "albedo_srgb_tables": (c_int32, [_D3, c_void_p]),
    "albedo_write_ppm": (c_int32, [c_char_p, c_void_p, c_int32, c_int32]),
    "albedo_save_ppm": (c_int32, [c_char_p, c_void_p, c_int32, c_int32, c_void_p]),
    "albedo_save_ppm_host": (c_int32, [c_char_p, c_void_p, c_int32, c_int32]),
    "albedo_wavefront_configure": (c_int32, [c_int32, c_int32, c_int32]),
    "albedo_server_create": (c_int32, [c_int64, c_int32, POINTER(c_void_p)]),
    "albedo_server_submit": (c_int32, [c_void_p, c_void_p, POINTER(RenderJobC), c_void_p, POINTER(c_int64)]),
    "albedo_server_submit_view": (c_int32, [c_void_p, c_void_p, POINTER(RenderJobC), POINTER(CameraC), c_void_p,
                                            POINTER(c_int64)]),
    "albedo_server_step": (c_int32, [c_void_p, POINTER(c_int64), c_int32, POINTER(c_int32)]),
    "albedo_server_pending": (c_int32, [c_void_p, POINTER(c_int32), POINTER(c_int32)]),
    "albedo_server_release_scene": (c_int32, [c_void_p, c_void_p]),
    "albedo_server_set_express": (c_int32, [c_void_p, c_int64]),
    "albedo_server_routes": (c_int32, [c_void_p, POINTER(c_int64), POINTER(c_int64)]),
    "albedo_server_destroy": (None, [c_void_p]),
    "albedo_autotune_megakernel": (c_int32, [c_void_p, POINTER(RenderJobC), POINTER(TuningC)]),
    "albedo_autotune_batch": (c_int32, [c_void_p, c_int32, POINTER(TuningC)]),
    "albedo_tuning_get": (c_int32, [c_void_p, POINTER(TuningC)]),
    "albedo_tuning_set": (c_int32, [c_void_p, POINTER(TuningC)]),
    "albedo_wavefront_last_iterations": (c_int32, [POINTER(c_int64)]),
    "albedo_wavefront_last_rays": (c_int32, [POINTER(c_int64)]),
    "albedo_server_rays": (c_int32, [c_void_p, POINTER(c_int64)]),
    "albedo_trace_host": (c_int32, [c_void_p, _F, c_int64, c_float, c_float, _I, _F, _I, _I, _F, _F, _F, _I]),
    "albedo_occluded_host": (c_int32, [c_void_p, _F, _F, c_int64, _I]),
    "albedo_probe_pixel_stream": (c_int32, [c_uint64, c_int32, c_int32, c_int32, c_int32, _U, _F]),
    "albedo_probe_lobe_eval": (c_int32, [c_int32, _F, _F, c_int32, _F, _F]),
    "albedo_probe_lobe_sample": (c_int32, [c_int32, _F, _F, c_int32, _I, _F, _F, _F, _I]),
    "albedo_probe_perlin": (c_int32, [_F, c_int32, _F, _F]),
    "albedo_probe_camera_rays": (c_int32, [c_void_p, c_int32, c_int32, _F, c_int32, _F]),
    "albedo_probe_trace_modes": (c_int32, [c_void_p, _F, c_int64, c_float, c_float, c_int32, c_int32, _I, _U, _U,
                                           _U]),
}

_lib: ctypes.CDLL | None = None


def library() -> ctypes.CDLL:
    """The loaded library; raises if it has not been built (no fallback exists)."""
    global _lib
    if _lib is None:
        if not LIBRARY_PATH.exists():
            raise RuntimeError(
                f"{LIBRARY_PATH} is missing: build it with `python albedo_b200/build.py` "
                "(the CUDA path is the only implementation)")
        lib = ctypes.CDLL(str(LIBRARY_PATH))
        for name, (restype, argtypes) in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib
