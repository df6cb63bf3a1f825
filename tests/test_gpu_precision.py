"""Precision form: the full-size large meshes against an FP64 oracle, both
render forms, FP64 and compensated FP32 accumulation (GPU).

Scenes at full size: a displaced icosphere (8 levels, 1,310,720 triangles;
seeded 3-octave Perlin displacement, amplitude 0.05) in rough glass (eta 1.5,
GGX alpha 0.1), and a soup of 1,000,000 random triangles (centers uniform in
the unit cube, edge lengths log-uniform in [1e-4, 1e-2]) in gold, rendered at
480 x 270 (bench.py renders the same scenes at 1920 x 1080).

The oracle is the reference renderer (FP64, accumulated in FP64) at 64 x 64 =
4,096 samples per pixel on 2,048 seeded pixels. On those pixels, for the
megakernel (both accumulation modes) and the wavefront:
  matched error  at 16 spp, the device image and the reference CPU renderer's
                 (same spp and seed) have the same mean squared relative error
                 against the oracle: the mean of the per-pixel differences of
                 squared errors is within 4 standard errors of zero (a paired
                 test; the oracle's own noise enters both sides alike, and rough
                 glass gives heavy-tailed per-pixel errors, which make a ratio of
                 two RMSEs over a few hundred pixels unstable)
  bias           at 4,096 spp the mean of the image over the pixels is within
                 1% of the oracle's (both carry noise: the per-pixel mean
                 absolute error, about 1.5% at this spp, measures noise, not
                 bias), and |z| > 4 on at most 1% of pixel channels
and the two accumulation modes agree within 1e-6 relative on every lit pixel.
"""

import numpy as np
import pytest
import torch

import albedo_b200 as ab
from albedo_b200 import scenes
from oracle import reference as ref

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="reference library not built")]

WIDTH, HEIGHT, DEPTH = 480, 270, 16
ORACLE_N = 64
ORACLE_SEED = 1000003
PIXELS = 2048


@pytest.fixture(scope="module")
def precision_scenes(tmp_path_factory):
    base = tmp_path_factory.mktemp("precision")
    return {"icosphere": scenes.icosphere_scene(base / "icosphere", levels=8),
            "soup": scenes.soup_scene(base / "soup", count=1_000_000)}


def pixel_subset(count, seed):
    rng = np.random.default_rng(seed)
    flat = rng.choice(WIDTH * HEIGHT, size=count, replace=False)
    return np.stack([flat % WIDTH, flat // WIDTH], axis=1).astype(np.int32)


def megakernel_means(scene, n, pixels, seed, accumulation):
    job = ab.RenderJob(WIDTH, HEIGHT, samples_per_axis=n, seed=seed, max_depth=DEPTH, accumulation=accumulation)
    acc, squares = ab.render_pixels(scene, job, pixels, with_squares=True)
    s = n * n
    mean = np.stack([acc["r"], acc["g"], acc["b"]], axis=1) / s
    var = np.maximum(squares / s - mean**2, 0) / s
    return mean, var


def wavefront_means(scene, n, pixels, seed):
    """The wavefront renders whole frames: the listed pixels of one."""
    job = ab.RenderJob(WIDTH, HEIGHT, samples_per_axis=n, seed=seed, max_depth=DEPTH, method=ab.WAVEFRONT)
    acc = torch.zeros((WIDTH * HEIGHT, 4), dtype=torch.float64, device="cuda")
    ab.render_device(scene, job, acc.data_ptr())
    torch.cuda.synchronize()
    scene.check()
    image = acc.cpu().numpy()
    picked = image[pixels[:, 1] * WIDTH + pixels[:, 0]]
    assert np.all(np.ascontiguousarray(picked[:, 3]).view(np.int64) == n * n)
    return picked[:, :3] / (n * n)


def squared_errors(image, oracle):
    """Per-pixel squared relative error against the oracle (pixels the oracle sees lit)."""
    lum = oracle.mean(axis=1)
    keep = lum > 1e-3
    return np.sum(((image - oracle)[keep] / lum[keep, None]) ** 2, axis=1)


def paired_t(ours, theirs, oracle):
    d = squared_errors(ours, oracle) - squared_errors(theirs, oracle)
    se = d.std(ddof=1) / np.sqrt(len(d))
    return 0.0 if se == 0 else d.mean() / se


def rel_rmse(image, oracle):
    return float(np.sqrt(squared_errors(image, oracle).mean() / 3))


@pytest.fixture(scope="module")
def oracles(precision_scenes):
    out = {}
    pixels = pixel_subset(PIXELS, 91)
    for which, path in precision_scenes.items():
        reference = ref.RefScene(path)
        oracle_sum, oracle_sq = reference.render_pixels(WIDTH, HEIGHT, ORACLE_N, pixels, seed=ORACLE_SEED,
                                                        max_depth=DEPTH)
        samples = ORACLE_N**2
        oracle = oracle_sum / samples
        oracle_var = np.maximum(oracle_sq / samples - oracle**2, 0) / samples
        theirs_sum, _ = reference.render_pixels(WIDTH, HEIGHT, 4, pixels, seed=0, max_depth=DEPTH)
        out[which] = {"pixels": pixels, "oracle": oracle, "oracle_var": oracle_var, "theirs": theirs_sum / 16}
    return out


@pytest.mark.parametrize("which", ["icosphere", "soup"])
def test_megakernel_against_the_fp64_oracle(which, precision_scenes, oracles):
    scene = ab.Scene.load(precision_scenes[which])
    o = oracles[which]
    pixels, oracle, theirs = o["pixels"], o["oracle"], o["theirs"]
    lum = oracle.mean(axis=1)
    keep = lum > 1e-3
    converged = {}
    for mode in (ab.ACCUMULATE_FP64, ab.ACCUMULATE_KAHAN_FP32):
        ours, _ = megakernel_means(scene, 4, pixels, 0, mode)
        t = paired_t(ours, theirs, oracle)
        assert abs(t) < 4, (mode, t, rel_rmse(ours, oracle), rel_rmse(theirs, oracle))
        mean, var = megakernel_means(scene, ORACLE_N, pixels, 7, mode)
        bias = abs(mean[keep].mean() - oracle[keep].mean()) / oracle[keep].mean()
        assert bias < 0.01, (mode, bias)
        z = (mean - oracle) / np.sqrt(var + o["oracle_var"] + 1e-16)
        assert np.mean(np.abs(z) > 4) < 0.01, (mode, np.mean(np.abs(z) > 4))
        converged[mode] = mean
    a, b = converged[ab.ACCUMULATE_KAHAN_FP32], converged[ab.ACCUMULATE_FP64]
    lit = np.abs(b) > 1e-9
    assert np.max(np.abs(a - b)[lit] / np.abs(b)[lit]) < 1e-6


@pytest.mark.parametrize("which", ["icosphere", "soup"])
def test_wavefront_against_the_fp64_oracle(which, precision_scenes, oracles):
    """The wavefront on the same pixels: the same matched-error and bias tests."""
    scene = ab.Scene.load(precision_scenes[which])
    o = oracles[which]
    pixels, oracle, theirs = o["pixels"], o["oracle"], o["theirs"]
    ours = wavefront_means(scene, 4, pixels, 0)
    t = paired_t(ours, theirs, oracle)
    assert abs(t) < 4, (t, rel_rmse(ours, oracle), rel_rmse(theirs, oracle))
    lum = oracle.mean(axis=1)
    keep = lum > 1e-3
    mean = wavefront_means(scene, ORACLE_N, pixels, 7)
    bias = abs(mean[keep].mean() - oracle[keep].mean()) / oracle[keep].mean()
    assert bias < 0.01, bias
    # The wavefront keeps no sums of squares: the megakernel's variance at the
    # same spp stands in for it (the two sample the same estimator).
    _, var = megakernel_means(scene, ORACLE_N, pixels, 7, ab.ACCUMULATE_FP64)
    z = (mean - oracle) / np.sqrt(var + o["oracle_var"] + 1e-16)
    assert np.mean(np.abs(z) > 4) < 0.01, np.mean(np.abs(z) > 4)
