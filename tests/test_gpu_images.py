"""Images against a 65,536-spp FP64 oracle (GPU).

The oracle is the reference renderer itself (FP64 throughout, built from its own
sources) at 256 x 256 = 65,536 samples per pixel, on a seeded subset of pixels,
with a seed of its own. Two statements are checked:

  matched RMSE   at equal spp and seed, the device image's relative RMSE against
                 the oracle equals the reference CPU image's within 3% over 512
                 pixels (the same random streams give the same paths until FP32
                 rounding sends one a different way; after that the two estimates
                 are independent draws, and the RMSE of 512 noisy pixels itself
                 varies by a few percent)
  bias           at 65,536 spp the device image's mean relative error against the
                 oracle is below 1%, and per-pixel differences are consistent with
                 Monte Carlo noise (|z| > 4 on at most 1% of pixels)
"""

import numpy as np
import pytest

import albedo_b200 as ab
from oracle import reference as ref

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="reference library not built")]

ORACLE_N = 256  # 65,536 spp
ORACLE_SEED = 1000003


def pixel_subset(width, height, count, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.integers(0, width, count), rng.integers(0, height, count)], axis=1).astype(np.int32)


def device_means(scene, width, height, n, pixels, seed, depth):
    acc, squares = ab.render_pixels(scene, ab.RenderJob(width, height, samples_per_axis=n, seed=seed,
                                                         max_depth=depth), pixels, with_squares=True)
    s = n * n
    mean = np.stack([acc["r"], acc["g"], acc["b"]], axis=1) / s
    var = np.maximum(squares / s - mean**2, 0) / s
    return mean, var


def relative_rmse(image, oracle):
    lum_o = oracle.mean(axis=1)
    keep = lum_o > 1e-3
    return np.sqrt(np.mean(((image - oracle)[keep] / lum_o[keep, None]) ** 2))


@pytest.mark.parametrize("which, width, height, depth", [("room", 320, 180, 8), ("trefoil", 960, 540, 10)])
def test_matched_rmse_and_bias_against_fp64_oracle(which, width, height, depth, room_path, trefoil_path):
    path = room_path if which == "room" else trefoil_path
    scene = ab.Scene.load(path)
    reference = ref.RefScene(path)
    pixels = pixel_subset(width, height, 512, 77)

    oracle_sum, oracle_sq = reference.render_pixels(width, height, ORACLE_N, pixels, seed=ORACLE_SEED, max_depth=depth)
    samples = ORACLE_N**2
    oracle = oracle_sum / samples
    oracle_var = np.maximum(oracle_sq / samples - oracle**2, 0) / samples

    # Matched RMSE at the configuration's own spp (n = 4).
    n = 4
    ours, _ = device_means(scene, width, height, n, pixels, 0, depth)
    theirs_sum, _ = reference.render_pixels(width, height, n, pixels, seed=0, max_depth=depth)
    theirs = theirs_sum / (n * n)
    rmse_ours = relative_rmse(ours, oracle)
    rmse_theirs = relative_rmse(theirs, oracle)
    assert abs(rmse_ours - rmse_theirs) / rmse_theirs < 0.03, (rmse_ours, rmse_theirs)

    # Bias: converged device image against the converged oracle.
    converged, converged_var = device_means(scene, width, height, ORACLE_N, pixels, 7, depth)
    lum = oracle.mean(axis=1)
    keep = lum > 1e-3
    mean_rel = np.mean(np.abs(converged - oracle)[keep] / lum[keep, None])
    assert mean_rel < 0.01, mean_rel
    z = (converged - oracle) / np.sqrt(converged_var + oracle_var + 1e-16)
    assert np.mean(np.abs(z) > 4) < 0.01, np.mean(np.abs(z) > 4)
