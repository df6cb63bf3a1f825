"""The allocation-free render entry point (GPU).

albedo_render_noalloc is for callers that cannot allocate device memory (another
allocator owns it, or allocation would break a latency budget). It keeps its
path slots and queues in a static device array, one slot per pixel. This test
calls it through the C ABI twice in a row, on the same scene and job, and checks
each result against the existing wavefront entry point (albedo_render), with the
tolerance the wavefront tests use: identical sample counts, image sums within
1e-4 relative, and at most 0.5% of pixels differing by more than 1e-3 relative.
The second call must leave the device's free memory (cudaMemGetInfo) and the
torch allocator's counters exactly as they were: the first call on a device may
still load kernels, the second has nothing left to load or allocate.
It also checks that an image over the 65,536-pixel limit is refused. It is named
to be collected last, so a run that stops at its first failure has run every
other test before it.
"""

from ctypes import byref, c_void_p

import numpy as np
import pytest
import torch

import albedo_b200 as ab
from albedo_b200._lib import library

pytestmark = pytest.mark.gpu


def counts(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a[:, 3]).view(np.int64)


def assert_same_image(a: np.ndarray, b: np.ndarray):
    np.testing.assert_array_equal(counts(a), counts(b))
    ca, cb = a[:, :3], b[:, :3]
    assert np.abs(ca.sum() - cb.sum()) / cb.sum() < 1e-4
    rel = np.abs(ca - cb) / np.maximum(np.abs(cb), 1e-3)
    assert np.mean(rel.max(axis=1) > 1e-3) < 0.005


def noalloc_render(scene, job) -> np.ndarray:
    acc = torch.zeros((job.width * job.height, 4), dtype=torch.float64, device="cuda")
    c = job.to_c()
    status = library().albedo_render_noalloc(scene.handle, byref(c), c_void_p(acc.data_ptr()), c_void_p(0))
    assert status == 0, library().albedo_last_error().decode()
    torch.cuda.synchronize()
    scene.check()
    return acc.cpu().numpy()


def existing_render(scene, job) -> np.ndarray:
    acc = torch.zeros((job.width * job.height, 4), dtype=torch.float64, device="cuda")
    ab.render_device(scene, job, acc.data_ptr())
    torch.cuda.synchronize()
    scene.check()
    return acc.cpu().numpy()


def test_noalloc_matches_the_allocating_entry_point_twice(room_path):
    scene = ab.Scene.load(room_path)
    job = ab.RenderJob(160, 90, samples_per_axis=4, seed=3, max_depth=8, method=ab.WAVEFRONT)
    expected = existing_render(scene, job)
    assert np.all(counts(expected) == 16)
    first = noalloc_render(scene, job)
    acc = torch.zeros((job.width * job.height, 4), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    allocated_before = torch.cuda.memory_allocated()
    reserved_before = torch.cuda.memory_reserved()
    c = job.to_c()
    status = library().albedo_render_noalloc(scene.handle, byref(c), c_void_p(acc.data_ptr()), c_void_p(0))
    assert status == 0, library().albedo_last_error().decode()
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    assert torch.cuda.memory_allocated() == allocated_before
    assert torch.cuda.memory_reserved() == reserved_before
    scene.check()
    second = acc.cpu().numpy()
    assert_same_image(first, expected)
    assert_same_image(second, expected)


def test_noalloc_refuses_images_over_its_limit(room_path):
    scene = ab.Scene.load(room_path)
    job = ab.RenderJob(320, 240, samples_per_axis=1, method=ab.WAVEFRONT)  # 76,800 pixels
    c = job.to_c()
    status = library().albedo_render_noalloc(scene.handle, byref(c), c_void_p(0), c_void_p(0))
    assert status == 1  # ALBEDO_INVALID_ARGUMENT
    assert "at most 65536 pixels" in library().albedo_last_error().decode()
