"""The ScatterOnly and Normals estimators against the reference's own (GPU).

ScatterOnlyEstimator (estimator/scatter_only_estimator.cpp:14-48) is the
reference's independent check of next-event estimation and MIS
(tests/estimator/path_estimator_test.cpp:208-233): it only follows BSDF samples.
NormalsEstimator (estimator/normals_estimator.cpp:32-38) colours each sample by
the shading normal of its first hit, so it compares the device's shading
normals, smooth mesh normals included, with the reference's directly.

Tolerances:
  scatter only   per-pixel two-sample z-scores at equal spp (|z| > 4 on at most
                 0.5% of pixels), image means within 1%, as the path estimator's
                 image tests
  normals        per pixel within 2e-5 of the reference (FP32 normals against
                 FP64) on at least 99% of pixels; the rest are pixels where one
                 of the n^2 samples grazes a silhouette and the two sides hit
                 different surfaces (the ray-query tests classify such near-ties);
                 no pixel further off than one sample's whole share
"""

import numpy as np
import pytest

import albedo_b200 as ab
from oracle import reference as ref

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="reference library not built")]


def _pixels(width, height, count, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.integers(0, width, count), rng.integers(0, height, count)], axis=1).astype(np.int32)


@pytest.mark.parametrize("which, width, height, n, depth", [("room", 320, 180, 4, 8), ("trefoil", 960, 540, 4, 10)])
def test_scatter_only_matches_reference_at_equal_spp(which, width, height, n, depth, room_path, trefoil_path):
    path = room_path if which == "room" else trefoil_path
    scene = ab.Scene.load(path)
    pixels = _pixels(width, height, 2048, 31)
    job = ab.RenderJob(width, height, samples_per_axis=n, seed=5, estimator=ab.SCATTER_ONLY, max_depth=depth)
    acc, squares = ab.render_pixels(scene, job, pixels, with_squares=True)
    samples = n * n
    assert np.all(acc["count"] == samples)
    rsum, rsq = ref.RefScene(path).render_pixels(width, height, n, pixels, seed=5, estimator=1, max_depth=depth)
    ours = np.stack([acc["r"], acc["g"], acc["b"]], axis=1) / samples
    theirs = rsum / samples
    var_o = np.maximum(squares / samples - ours**2, 0)
    var_t = np.maximum(rsq / samples - theirs**2, 0)
    z = (ours - theirs) / np.sqrt((var_o + var_t) / samples + 1e-12)
    assert np.mean(np.abs(z) > 4) < 0.005, np.mean(np.abs(z) > 4)
    assert abs(ours.mean() - theirs.mean()) / theirs.mean() < 0.01


@pytest.mark.parametrize("which, width, height", [("room", 320, 180), ("trefoil", 480, 270)])
def test_normals_match_reference(which, width, height, room_path, trefoil_path):
    path = room_path if which == "room" else trefoil_path
    scene = ab.Scene.load(path)
    n = 2
    samples = n * n
    pixels = np.stack(np.meshgrid(np.arange(width), np.arange(height)), axis=-1).reshape(-1, 2).astype(np.int32)
    job = ab.RenderJob(width, height, samples_per_axis=n, seed=2, estimator=ab.NORMALS)
    acc = ab.render_pixels(scene, job, pixels)
    assert np.all(acc["count"] == samples)
    rsum, _ = ref.RefScene(path).render_pixels(width, height, n, pixels, seed=2, estimator=2)
    ours = np.stack([acc["r"], acc["g"], acc["b"]], axis=1) / samples
    theirs = rsum / samples
    err = np.abs(ours - theirs).max(axis=1)
    assert np.mean(err <= 2e-5) >= 0.99, (np.mean(err <= 2e-5), np.quantile(err, [0.5, 0.99, 1.0]))
    # A normal colour channel lies in [0, 1]: one sample's share is 1 / n^2.
    assert err.max() <= 1.0 / samples + 1e-5, err.max()
