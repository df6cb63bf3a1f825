"""The device resolve to sRGB bytes and the PPM output, against the reference (GPU).

Bit-exact: every byte equals the reference's toByte(encodeSrgb(sum / count))
(color/srgb.cpp:18-36, image/pixel_buffer.cpp:37-45) on seeded accumulators
with empty pixels, NaN and infinite sums, negative and huge values, ragged
tails and unaligned buffers; at the largest image the reference accepts
(16384 x 16384 = 2^28 pixels) through a tiled pattern whose expected bytes tile
the same way. A rendered image saved by save_ppm is byte-identical to the file
the reference's writePpm writes for the same averages.
"""

from pathlib import Path

import numpy as np
import pytest

import albedo_b200 as ab
from albedo_b200 import scenes
from oracle import reference as ref

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="reference library not built")]


def seeded_accumulators(pixels: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    count = rng.integers(1, 4097, pixels).astype(np.int64)
    count[rng.random(pixels) < 0.05] = 0
    count[rng.random(pixels) < 0.01] = 1 << 40
    sums = rng.uniform(-0.1, 1.3, (pixels, 3)) * count[:, None]
    flat = sums.reshape(-1)
    flat[rng.random(flat.size) < 0.01] = np.nan
    flat[rng.random(flat.size) < 0.005] = np.inf
    flat[rng.random(flat.size) < 0.005] = -np.inf
    flat[rng.random(flat.size) < 0.02] = 0.0
    acc = np.zeros(pixels, dtype=ab.ACCUMULATOR_DTYPE)
    acc["r"], acc["g"], acc["b"], acc["count"] = sums[:, 0], sums[:, 1], sums[:, 2], count
    return acc


def expected_bytes(acc: np.ndarray) -> np.ndarray:
    count = acc["count"].astype(np.float64)
    rgb = np.stack([acc["r"], acc["g"], acc["b"]], axis=1)
    with np.errstate(invalid="ignore", divide="ignore"):
        avg = np.where(count[:, None] > 0, rgb / np.where(count > 0, count, 1.0)[:, None], 0.0)
    return ref.srgb_bytes(avg).reshape(-1)


def to_device(acc: np.ndarray, byte_offset: int = 0):
    import torch

    words = acc.view(np.float64).reshape(-1)
    extra = byte_offset // 8
    buf = torch.zeros(words.size + extra, dtype=torch.float64, device="cuda")
    buf[extra:] = torch.from_numpy(words.copy()).cuda()
    return buf, buf.data_ptr() + 8 * extra


@pytest.mark.parametrize("shape", [(1, 1), (1, 3), (5, 7), (13, 1), (270, 480), (1080, 1920)])
@pytest.mark.parametrize("offsets", [(0, 0), (32, 16), (16, 0), (0, 4), (8, 0), (0, 1), (8, 3)])
def test_resolve_is_bit_exact_with_the_reference(shape, offsets):
    import torch

    h, w = shape
    acc_offset, out_offset = offsets
    acc = seeded_accumulators(w * h, seed=w * 31 + h)
    buf, ptr = to_device(acc, acc_offset)
    out = torch.full((3 * w * h + out_offset + 16,), 77, dtype=torch.uint8, device="cuda")
    ab.resolve_srgb(ptr, w, h, out.data_ptr() + out_offset)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.array_equal(got[out_offset:out_offset + 3 * w * h], expected_bytes(acc))
    # Nothing outside the image is written.
    assert np.all(got[:out_offset] == 77) and np.all(got[out_offset + 3 * w * h:] == 77)


def test_averages_next_to_every_decision_resolve_exactly():
    # Averages within 6 ulps of every threshold and bucket edge, for counts that
    # are and are not powers of two (test_film_output.py builds them): a quotient
    # rounded the wrong way, or a table read from the wrong bucket, shows here.
    import sys
    import torch

    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from test_film_output import adversarial_accumulators, reference_average_bytes

    sums, counts = adversarial_accumulators()
    acc = np.zeros(len(sums), dtype=ab.ACCUMULATOR_DTYPE)
    acc["r"], acc["g"], acc["b"] = sums, np.roll(sums, 1), np.roll(sums, 2)
    acc["count"] = counts.astype(np.int64)
    device, ptr = to_device(acc)
    out = torch.empty(3 * len(sums), dtype=torch.uint8, device="cuda")
    ab.resolve_srgb(ptr, len(sums), 1, out.data_ptr())
    got = out.cpu().numpy().reshape(-1, 3)
    for channel, values in enumerate((acc["r"], acc["g"], acc["b"])):
        np.testing.assert_array_equal(got[:, channel], reference_average_bytes(values, counts))


def test_resolve_at_the_largest_image_size():
    import torch

    base_pixels = 1 << 16
    side = 1 << 14  # 16384 x 16384 = 2^28 pixels, PixelBuffer's limit
    acc = seeded_accumulators(base_pixels, seed=99)
    base, _ = to_device(acc)
    tiled = base.view(base_pixels, 4).repeat((side * side) // base_pixels, 1)
    out = torch.empty(3 * side * side, dtype=torch.uint8, device="cuda")
    ab.resolve_srgb(tiled.data_ptr(), side, side, out.data_ptr())
    expected = torch.from_numpy(expected_bytes(acc)).cuda()
    assert bool((out.view(-1, 3 * base_pixels) == expected[None, :]).all())
    del tiled, out
    with pytest.raises(ValueError, match="invalid image size"):
        ab.resolve_srgb(base.data_ptr(), side, side + 1, base.data_ptr())


def test_unaligned_accumulators_are_refused():
    import torch

    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    out = torch.zeros(64, dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError, match="8-byte aligned"):
        ab.resolve_srgb(buf.data_ptr() + 4, 2, 2, out.data_ptr())


def test_rendered_image_saves_like_the_reference_writer(tmp_path):
    import torch

    path = scenes.room_scene(tmp_path)
    scene = ab.Scene.load(path)
    w, h, n = 96, 54, 2
    acc = torch.zeros((w * h, 4), dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        ab.render_device(scene, ab.RenderJob(w, h, samples_per_axis=n, max_depth=8), acc.data_ptr(),
                         stream=stream.cuda_stream)
        ab.save_ppm(tmp_path / "ours.ppm", acc.data_ptr(), w, h, stream=stream.cuda_stream)
    scene.check()
    host = acc.cpu().numpy().copy().view(ab.ACCUMULATOR_DTYPE).reshape(-1)
    image = ab.PixelBuffer(w, h)
    image.pixels[:] = host
    ref.write_ppm(tmp_path / "theirs.ppm", image.average())
    assert (tmp_path / "ours.ppm").read_bytes() == (tmp_path / "theirs.ppm").read_bytes()
    # The host-buffer path (PixelBuffer.write_ppm) writes the same file.
    image.write_ppm(tmp_path / "host.ppm")
    assert (tmp_path / "host.ppm").read_bytes() == (tmp_path / "theirs.ppm").read_bytes()
    scene.close()
