"""The device path against the committed reference vectors (GPU).

The vectors (tests/golden/reference_vectors.npz, written by
tests/golden/make_golden.py from the reference renderer) travel with the tests,
so these checks need no reference build. Tolerances as in test_gpu_parity.py:
the per-pixel random stream bit-exact; ray queries with identical hits and
objects apart from near-ties (FP32 against FP64), t within 2 ulps on at least
99% of hits; sRGB bytes and the PPM file bit-exact; the rendered image, whose
paths follow the same random streams, equal to the reference's on most pixels
and in its mean.
"""

from ctypes import POINTER, c_float, c_uint32
from pathlib import Path

import numpy as np
import pytest

import albedo_b200 as ab

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_vectors.npz"


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as data:
        return {k: data[k] for k in data.files}


@pytest.fixture(scope="module")
def room(golden, tmp_path_factory):
    path = tmp_path_factory.mktemp("golden") / "room.scene"
    path.write_text(str(golden["room_scene_text"]))
    scene = ab.Scene.load(path)
    yield scene
    scene.close()


def test_pixel_stream_equals_the_vector(golden):
    u32 = np.zeros(64, np.uint32)
    real = np.zeros(64, np.float32)
    status = ab._lib.library().albedo_probe_pixel_stream(0, 3, 5, 320, 64, u32.ctypes.data_as(POINTER(c_uint32)),
                                                         real.ctypes.data_as(POINTER(c_float)))
    assert status == 0
    np.testing.assert_array_equal(u32.astype(np.float64) / 4294967296.0, golden["pixel_stream"])


def test_ray_queries_equal_the_vectors(golden, room):
    ours = room.intersect(golden["room_rays"].astype(np.float32))
    same = (ours["hit"] == golden["room_hit"]) & ((ours["hit"] == 0) | (ours["object"] == golden["room_object"]))
    assert (~same).sum() <= 1
    both = same & (ours["hit"] == 1)
    assert both.sum() > 200
    t_ref = golden["room_t"][both].astype(np.float32)
    ulps = np.abs(ours["t"][both].view(np.int32).astype(np.int64) - t_ref.view(np.int32).astype(np.int64))
    assert np.mean(ulps <= 2) >= 0.99 and ulps.max() <= 64, ulps.max()


def test_resolve_and_ppm_equal_the_reference_file(golden, tmp_path):
    import torch

    image = golden["room_image"]
    h, w, _ = image.shape
    acc = np.zeros(w * h, dtype=ab.ACCUMULATOR_DTYPE)
    flat = image.reshape(-1, 3)
    acc["r"], acc["g"], acc["b"], acc["count"] = flat[:, 0], flat[:, 1], flat[:, 2], 1
    device = torch.from_numpy(acc.view(np.float64).reshape(-1, 4).copy()).cuda()
    ab.save_ppm(tmp_path / "room.ppm", device.data_ptr(), w, h)
    assert (tmp_path / "room.ppm").read_bytes() == golden["room_ppm"].tobytes()


def test_rendered_image_follows_the_reference(golden, room):
    image = golden["room_image"]
    h, w, _ = image.shape
    pixels = ab.PixelBuffer(w, h)
    ab.render_image(room, ab.RenderJob(w, h, samples_per_axis=2, max_depth=8, seed=0), pixels)
    ours = pixels.average()
    close = np.all(np.abs(ours - image) <= 1e-3 * np.maximum(np.abs(image), 1e-3), axis=2)
    assert close.mean() >= 0.8, close.mean()
    assert abs(ours.mean() - image.mean()) <= 0.05 * image.mean()
