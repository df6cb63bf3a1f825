"""renderImage through the C++ adapter (include/albedo_b200_adapter.hpp) on the
GPU against the reference's own renderImage on the same RenderJob (GPU).

The adapter is built against the reference's headers and library (oracle/Makefile,
target `adapter`); the job is a reference RenderJob with a reference
PerspectiveCamera, and the image a reference PixelBuffer.

Tolerances: the same random streams give the same paths until FP32 rounding
splits one, so at least 90% of pixels agree within 1e-3 relative (or 1e-3
absolute for dark pixels) and the image means within 1%; the Normals estimator
agrees within 2e-5 on at least 99% of pixels; samples already in the buffer
stay, and the new ones add to them (pixel (0, 0) within the same tolerances).
"""

import numpy as np
import pytest

from oracle import adapter
from oracle import reference as ref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (adapter.available() and ref.available()), reason="adapter harness not built")]


def _close(ours, theirs):
    return np.abs(ours - theirs).max(axis=-1) <= 1e-3 * np.maximum(1.0, np.abs(theirs).max(axis=-1))


@pytest.mark.parametrize("which, width, height, n, depth", [("room", 160, 90, 2, 8), ("trefoil", 240, 135, 2, 10)])
def test_path_estimator_through_the_adapter_matches_render_image(which, width, height, n, depth, room_path,
                                                                  trefoil_path):
    path = room_path if which == "room" else trefoil_path
    status, ours = adapter.render(path, gpu=True, width=width, height=height, samples_per_axis=n, seed=4,
                                  max_depth=depth, prior_samples=5)
    assert status == "ok", ours
    status, theirs = adapter.render(path, gpu=False, width=width, height=height, samples_per_axis=n, seed=4,
                                    max_depth=depth, prior_samples=5)
    assert status == "ok"
    close = _close(ours, theirs)
    assert close.mean() >= 0.9, close.mean()
    assert abs(ours.mean() - theirs.mean()) / theirs.mean() < 0.01
    # Pixel (0, 0) held 5 samples of (1, 2, 3) before the render, and the render
    # added n^2 more: its average keeps the prior samples' 5 / (5 + n^2) share.
    prior = 5 / (5 + n * n) * np.array([1.0, 2.0, 3.0])
    assert np.all(ours[0, 0] >= prior - 1e-12), ours[0, 0]
    np.testing.assert_allclose(ours[0, 0], theirs[0, 0], rtol=0.05)


@pytest.mark.parametrize("which", ["room", "trefoil"])
def test_normals_through_the_adapter_match_render_image(which, room_path, trefoil_path):
    path = room_path if which == "room" else trefoil_path
    status, ours = adapter.render(path, gpu=True, width=192, height=108, samples_per_axis=2, estimator=2)
    assert status == "ok", ours
    _, theirs = adapter.render(path, gpu=False, width=192, height=108, samples_per_axis=2, estimator=2)
    err = np.abs(ours - theirs).max(axis=-1)
    assert np.mean(err <= 2e-5) >= 0.99, np.quantile(err, [0.5, 0.99, 1.0])


def test_a_camera_for_another_aspect_ratio_is_refused(room_path):
    status, kind, message = adapter.render(room_path, gpu=True, width=160, height=90, camera_width=120,
                                           samples_per_axis=1)
    assert (status, kind) == ("error", 1)
    assert "aspect ratio" in message
