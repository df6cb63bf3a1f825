"""The oracle pinned against the reference's known-answer tests (CPU only).

Known answers held by the reference's own tests:
  PCG32(seed 42, stream 54) first six outputs     tests/sampling/pcg32_test.cpp:12-28
  perlinNoise at three points, to 1e-12           tests/texture/perlin_noise_test.cpp:79-88
"""

import numpy as np
import pytest

from oracle import pcg32 as pcg
from oracle import reference as ref

PCG32_42_54 = [0xA15C02B7, 0x7B47F409, 0xBA1D3330, 0x83D2F293, 0xBFA4784B, 0xCBED606E]
PERLIN_POINTS = [((3.14, 42.0, 7.0), 0.13691995878400012), ((-0.3, -5.7, 2.25), 0.40750939192218755),
                 ((-300.6, 17.2, -0.45), -0.11245507194489657)]

pytestmark = pytest.mark.skipif(not ref.available(), reason="reference library not built")


def test_reference_pcg32_known_answer():
    assert list(ref.pcg32(42, 54, 6)) == PCG32_42_54


def test_restated_pcg32_known_answer():
    g = pcg.Pcg32Streams(np.array([42], np.uint64), np.array([54], np.uint64))
    assert [int(g.next_u32()[0]) for _ in range(6)] == PCG32_42_54


def test_restated_pixel_streams_match_reference():
    width = 960
    xs = np.array([0, 1, 959, 17, 480, 3])
    ys = np.array([0, 0, 539, 250, 270, 1])
    for seed in (0, 1, 12345678901234):
        streams = pcg.pixel_streams(seed, xs, ys, width)
        ours = np.stack([streams.next_real() for _ in range(64)], axis=1)
        for i, (x, y) in enumerate(zip(xs, ys)):
            theirs = ref.pixel_stream(seed, int(x), int(y), width, 64)
            np.testing.assert_array_equal(ours[i], theirs)


def test_reference_perlin_known_answers():
    points = np.array([p for p, _ in PERLIN_POINTS])
    noise, _ = ref.perlin(points)
    np.testing.assert_allclose(noise, [v for _, v in PERLIN_POINTS], rtol=0, atol=1e-12)


def test_restated_perlin_matches_reference():
    from albedo_b200.scenes import perlin_noise

    rng = np.random.default_rng(3)
    points = rng.uniform(-400, 400, size=(2000, 3))
    noise, _ = ref.perlin(points)
    np.testing.assert_allclose(perlin_noise(points), noise, rtol=0, atol=1e-12)
    known = perlin_noise(np.array([p for p, _ in PERLIN_POINTS]))
    np.testing.assert_allclose(known, [v for _, v in PERLIN_POINTS], rtol=0, atol=1e-12)
