"""The committed reference vectors (tests/golden/reference_vectors.npz), on the host.

They were written by tests/golden/make_golden.py from the reference renderer built
from its own sources. Here: the scene generator still writes the same room; the
oracle, rebuilt, reproduces every vector exactly (which pins the oracle build:
its compiler flags keep the reference's rounding); and the host parts of this
library that need no GPU (the sRGB tables, the PPM writer, the scene reader)
agree with the vectors.
"""

import sys
from pathlib import Path

import numpy as np
import pytest

import albedo_b200 as ab
from albedo_b200 import scenes
from oracle import reference as ref

GOLDEN = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLDEN))

import make_golden  # noqa: E402


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN / "reference_vectors.npz") as data:
        return {k: data[k] for k in data.files}


def test_the_room_generator_is_unchanged(golden, tmp_path):
    assert scenes.room_scene(tmp_path).read_text() == str(golden["room_scene_text"])


@pytest.mark.skipif(not ref.available(), reason="reference library not built")
def test_the_oracle_reproduces_every_vector(golden):
    fresh = make_golden.generate()
    assert set(fresh) == set(golden)
    for key, value in fresh.items():
        np.testing.assert_array_equal(value, golden[key], err_msg=key)


def test_srgb_tables_give_the_reference_bytes(golden):
    lower = ab.srgb_thresholds()[1:]
    values = golden["srgb_values"]
    ours = np.where(np.isnan(values), 0, np.searchsorted(lower, values, side="right")).astype(np.uint8)
    np.testing.assert_array_equal(ours, golden["srgb_bytes"])


def test_ppm_writer_writes_the_reference_file(golden, tmp_path):
    image = golden["room_image"]
    lower = ab.srgb_thresholds()[1:]
    rgb = np.where(np.isnan(image), 0, np.searchsorted(lower, image, side="right")).astype(np.uint8)
    ab.write_ppm(tmp_path / "room.ppm", rgb)
    assert (tmp_path / "room.ppm").read_bytes() == golden["room_ppm"].tobytes()


def test_scene_reader_reads_the_room(golden, tmp_path):
    path = tmp_path / "room.scene"
    path.write_text(str(golden["room_scene_text"]))
    # Four walls, five spheres and the area light's sphere.
    assert ab.Scene.read(path).info()["objects"] == 10
