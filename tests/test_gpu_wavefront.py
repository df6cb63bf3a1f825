"""The wavefront renderer and batches agree with the megakernel (GPU).

Both forms draw each pixel's random numbers in the same order, so a pixel's
paths are the same paths; only the order in which next-event contributions are
summed differs (FP32 rounding). Tolerance: mean relative difference of the image
below 1e-4, and at most 0.5% of pixels differing by more than 1e-3 relative
(rare branch flips on near-ties).
"""

import numpy as np
import pytest
import torch

import albedo_b200 as ab

pytestmark = pytest.mark.gpu


def render(scene, job):
    acc = torch.zeros((job.width * job.height, 4), dtype=torch.float64, device="cuda")
    ab.render_device(scene, job, acc.data_ptr())
    torch.cuda.synchronize()
    scene.check()
    return acc.cpu().numpy()


def counts(a: np.ndarray) -> np.ndarray:
    """The int64 sample counts stored in the accumulators' fourth field."""
    return np.ascontiguousarray(a[:, 3]).view(np.int64)


def compare(a: np.ndarray, b: np.ndarray):
    np.testing.assert_array_equal(counts(a), counts(b))
    ca, cb = a[:, :3], b[:, :3]
    scale = np.maximum(np.abs(cb), 1e-3)
    rel = np.abs(ca - cb) / scale
    assert np.abs(ca.sum() - cb.sum()) / cb.sum() < 1e-4
    assert np.mean(rel.max(axis=1) > 1e-3) < 0.005, np.mean(rel.max(axis=1) > 1e-3)


@pytest.mark.parametrize("which", ["room", "trefoil"])
def test_wavefront_matches_megakernel(which, room_path, trefoil_path):
    path = room_path if which == "room" else trefoil_path
    scene = ab.Scene.load(path)
    base = dict(width=160, height=90, samples_per_axis=4, max_depth=8)
    mega = render(scene, ab.RenderJob(**base, method=ab.MEGAKERNEL))
    wave = render(scene, ab.RenderJob(**base, method=ab.WAVEFRONT))
    assert np.all(counts(mega) == 16)
    compare(wave, mega)
    assert ab.wavefront_last_iterations() > 0


def test_batch_equals_jobs_rendered_alone(room_path, trefoil_path):
    room = ab.Scene.load(room_path)
    trefoil = ab.Scene.load(trefoil_path)
    jobs = [(room, ab.RenderJob(64, 36, samples_per_axis=3, seed=5, max_depth=6)),
            (trefoil, ab.RenderJob(96, 54, samples_per_axis=2, seed=9, max_depth=10)),
            (room, ab.RenderJob(40, 30, samples_per_axis=5, seed=1, max_depth=64))]
    accs = [torch.zeros((j.width * j.height, 4), dtype=torch.float64, device="cuda") for _, j in jobs]
    ab.render_batch([(s, j, a.data_ptr()) for (s, j), a in zip(jobs, accs)])
    torch.cuda.synchronize()
    for (scene, job), acc in zip(jobs, accs):
        alone = render(scene, ab.RenderJob(job.width, job.height, samples_per_axis=job.samples_per_axis,
                                           seed=job.seed, max_depth=job.max_depth, method=ab.MEGAKERNEL))
        compare(acc.cpu().numpy(), alone)


def test_wavefront_small_slot_pool_reuses_slots(room_path):
    scene = ab.Scene.load(room_path)
    ab.wavefront_configure(slots=1000, blocks_per_sm=2, iterations_per_graph=2)
    try:
        job = ab.RenderJob(64, 36, samples_per_axis=2, max_depth=5, method=ab.WAVEFRONT)
        wave = render(scene, job)
    finally:
        ab.wavefront_configure()
    mega = render(scene, ab.RenderJob(64, 36, samples_per_axis=2, max_depth=5))
    compare(wave, mega)


def test_wavefront_rejects_other_estimators(room_path):
    scene = ab.Scene.load(room_path)
    with pytest.raises(ab.Unsupported):
        render(scene, ab.RenderJob(16, 16, estimator=ab.NORMALS, method=ab.WAVEFRONT))


def test_ray_binning_leaves_batches_unchanged(room_path, trefoil_path):
    """Binning each bounce's rays by job, direction octant and origin cell before
    they are traced (ray_sort 1; 2 bins the shadow rays too) reorders the work,
    not its results: a batch of jobs on two scenes renders bit for bit the same
    with and without it."""
    room = ab.Scene.load(room_path)
    trefoil = ab.Scene.load(trefoil_path)
    jobs = [(room, ab.RenderJob(160, 90, samples_per_axis=3, seed=5, max_depth=8)),
            (trefoil, ab.RenderJob(192, 108, samples_per_axis=2, seed=9, max_depth=10)),
            (room, ab.RenderJob(64, 48, samples_per_axis=4, seed=1, max_depth=64))]
    images = []
    try:
        for ray_sort in (0, 1, 2):
            ab.set_tuning(blocks_per_sm=8, trace_blocks_per_sm=4, fetch_batch=32, iterations_per_graph=4,
                          slot_count=1 << 15, trace_loop=1, ray_sort=ray_sort)
            assert ab.tuning()["ray_sort"] == ray_sort
            accs = [torch.zeros((j.width * j.height, 4), dtype=torch.float64, device="cuda") for _, j in jobs]
            ab.render_batch([(s, j, a.data_ptr()) for (s, j), a in zip(jobs, accs)])
            torch.cuda.synchronize()
            room.check()
            trefoil.check()
            images.append([a.cpu().numpy() for a in accs])
    finally:
        ab.wavefront_configure()
    for variant in images[1:]:
        for unsorted, binned in zip(images[0], variant):
            np.testing.assert_array_equal(binned.view(np.int64), unsorted.view(np.int64))
