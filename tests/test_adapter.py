"""The C++ adapter include/albedo_b200_adapter.hpp compiles against the
reference's own headers and links with the reference library (oracle/Makefile,
target `adapter`), and its host-side logic agrees with the reference (CPU only:
nothing here launches a kernel).

  camera    the settings recovered from a PerspectiveCamera's rays give the
            file's camera: the same position exactly, the view direction and
            the up direction's perpendicular part within 1e-12, the field of
            view within 1e-9 degrees
  errors    renderImage's argument checks raise std::invalid_argument with the
            reference's messages (render/render_image.cpp:60-67), before any
            GPU work; an unbound scene is refused the same way
"""

import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import adapter
from oracle import reference as ref

ORACLE = Path(__file__).resolve().parent.parent / "oracle"


@pytest.fixture(scope="module", autouse=True)
def built():
    root = subprocess.run(["make", "-s", "-C", str(ORACLE), "reference-root"], capture_output=True, text=True)
    if root.returncode == 0 and Path(root.stdout.strip(), "src").exists():
        subprocess.run(["make", "-C", str(ORACLE), "ref", "adapter"], check=True, capture_output=True)
    if not (adapter.available() and ref.available()):
        pytest.skip("adapter harness not built (needs the reference checkout)")


def _unit(v):
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("width, height", [(320, 180), (960, 540), (64, 64)])
def test_camera_settings_are_recovered_from_rays(room_path, trefoil_path, width, height):
    for path in (room_path, trefoil_path):
        mine, file = adapter.camera(path, width, height)
        np.testing.assert_array_equal(mine[:3], file[:3])
        forward = _unit(file[3:6] - file[:3])
        np.testing.assert_allclose(_unit(mine[3:6] - mine[:3]), forward, atol=1e-12)
        up = file[6:9] - np.dot(file[6:9], forward) * forward
        np.testing.assert_allclose(_unit(mine[6:9]), _unit(up), atol=1e-12)
        assert abs(mine[9] - file[9]) < 1e-9


@pytest.mark.parametrize("n, threads", [(0, 8), (-3, 8), (2, 0), (2, -1), (0, 0)])
def test_argument_checks_match_the_reference(room_path, n, threads):
    ours = adapter.render(room_path, gpu=True, bind=False, width=16, height=9, samples_per_axis=n, thread_count=threads)
    theirs = adapter.render(room_path, gpu=False, width=16, height=9, samples_per_axis=n, thread_count=threads)
    assert theirs[0] == "error" and ours == theirs, (ours, theirs)


def test_an_unbound_scene_is_refused(room_path):
    status, kind, message = adapter.render(room_path, gpu=True, bind=False, width=16, height=9, samples_per_axis=1)
    assert (status, kind) == ("error", 1)
    assert "bindScene" in message
