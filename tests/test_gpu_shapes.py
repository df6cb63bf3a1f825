"""Every megakernel shape on a large mesh (GPU).

The autotuner picks, per scene, one of five megakernel variants: 3 or 4 blocks
per SM (the 4-blocks/SM kernels keep each path's state in shared memory and
4-byte stack entries), with the traversal out of line or inlined, or (3 blocks
per SM) with only the closest-hit query inlined. They compile the same source,
so on the displaced icosphere (81,920 triangles, an instanced mesh in rough
glass) each gives the default shape's image, with no traversal error, and the
persistent wavefront kernels give the megakernel's image the same way. Two
kernels may round a shading operation differently (the compiler contracts
multiply-adds per kernel), and in rough glass such a path then scatters
differently, so the images agree statistically: identical sample counts, image
sums within 2e-3 relative, at most 5% of pixels beyond 1e-3 relative. A kernel
that skipped work or lost hits would move the sum by far more.
"""

import numpy as np
import pytest
import torch

import albedo_b200 as ab
from albedo_b200 import scenes

pytestmark = pytest.mark.gpu

SHAPES = [(3, 0), (3, 1), (3, 2), (4, 0), (4, 1)]


@pytest.fixture(scope="module")
def icosphere(tmp_path_factory):
    return ab.Scene.load(scenes.icosphere_scene(tmp_path_factory.mktemp("shapes"), levels=6))


def render(scene, job):
    acc = torch.zeros((job.width * job.height, 4), dtype=torch.float64, device="cuda")
    ab.render_device(scene, job, acc.data_ptr())
    torch.cuda.synchronize()
    scene.check()
    return acc.cpu().numpy()


def assert_same_image(a, b):
    np.testing.assert_array_equal(a[:, 3], b[:, 3])
    ca, cb = a[:, :3], b[:, :3]
    assert abs(ca.sum() - cb.sum()) / cb.sum() < 2e-3, (ca.sum(), cb.sum())
    rel = np.abs(ca - cb) / np.maximum(np.abs(cb), 1e-3)
    assert np.mean(rel.max(axis=1) > 1e-3) < 0.05, np.mean(rel.max(axis=1) > 1e-3)


@pytest.mark.parametrize("blocks,inline", SHAPES)
def test_megakernel_shape_matches_the_default_on_a_large_mesh(icosphere, blocks, inline):
    job = ab.RenderJob(192, 108, samples_per_axis=4, seed=7, max_depth=16)
    ab.set_tuning(icosphere, tile_width=16, blocks_per_sm=3, inline_traversal=0)
    base = render(icosphere, job)
    ab.set_tuning(icosphere, tile_width=16, blocks_per_sm=blocks, inline_traversal=inline)
    assert_same_image(render(icosphere, job), base)
    ab.set_tuning(icosphere, tile_width=16, blocks_per_sm=3, inline_traversal=0)


def test_wavefront_matches_the_megakernel_on_a_large_mesh(icosphere):
    base = render(icosphere, ab.RenderJob(192, 108, samples_per_axis=4, seed=7, max_depth=16))
    wave = render(icosphere, ab.RenderJob(192, 108, samples_per_axis=4, seed=7, max_depth=16, method=ab.WAVEFRONT))
    assert_same_image(wave, base)
