"""Autotuner, per-request cameras and compensated FP32 accumulation (GPU).

Tolerance where two launch shapes or two methods are compared: the wavefront
tests' (identical sample counts, image sums within 1e-4 relative, at most 0.5%
of pixels differing by more than 1e-3 relative).
"""

import numpy as np
import pytest
import torch

import albedo_b200 as ab
from albedo_b200 import scenes

pytestmark = pytest.mark.gpu


def render(scene, job, camera=None):
    acc = torch.zeros((job.width * job.height, 4), dtype=torch.float64, device="cuda")
    ab.render_device(scene, job, acc.data_ptr(), camera=camera)
    torch.cuda.synchronize()
    scene.check()
    return acc.cpu().numpy()


def counts(a):
    return np.ascontiguousarray(a[:, 3]).view(np.int64)


def assert_same_image(a, b):
    np.testing.assert_array_equal(counts(a), counts(b))
    ca, cb = a[:, :3], b[:, :3]
    assert np.abs(ca.sum() - cb.sum()) / cb.sum() < 1e-4
    rel = np.abs(ca - cb) / np.maximum(np.abs(cb), 1e-3)
    assert np.mean(rel.max(axis=1) > 1e-3) < 0.005


def scene_camera(path):
    return ab.Camera(*scenes.scene_camera(path))


def test_megakernel_tuning_keeps_a_valid_shape_and_the_image(room_path):
    scene = ab.Scene.load(room_path)
    job = ab.RenderJob(200, 120, samples_per_axis=4, max_depth=8)
    before = render(scene, job)
    assert ab.tuning(scene)["tile_width"] == 16 and ab.tuning(scene)["blocks_per_sm"] == 3
    t = ab.autotune_megakernel(scene, job)
    assert t["tile_width"] in (8, 16, 32) and t["blocks_per_sm"] in (3, 4) and t["inline_traversal"] in (0, 1, 2)
    assert t["inline_traversal"] != 2 or t["blocks_per_sm"] == 3
    assert t["evaluations"] == 15  # 3 tile widths x 5 kernel variants
    assert 0 < t["best_ms"] <= t["default_ms"]
    kept = ab.tuning(scene)
    assert all(kept[k] == t[k] for k in ("tile_width", "blocks_per_sm", "inline_traversal"))
    after = render(scene, job)
    assert_same_image(after, before)


def test_batch_tuning_leaves_accumulators_untouched_and_images_unchanged(room_path, trefoil_path):
    room, trefoil = ab.Scene.load(room_path), ab.Scene.load(trefoil_path)
    jobs = [(room, ab.RenderJob(64, 36, samples_per_axis=4, seed=5, max_depth=6, method=ab.WAVEFRONT)),
            (trefoil, ab.RenderJob(96, 54, samples_per_axis=2, seed=9, max_depth=10, method=ab.WAVEFRONT))]
    accs = [torch.zeros((j.width * j.height, 4), dtype=torch.float64, device="cuda") for _, j in jobs]
    ab.render_batch([(s, j, a.data_ptr()) for (s, j), a in zip(jobs, accs)])
    torch.cuda.synchronize()
    before = [a.cpu().numpy() for a in accs]
    untouched = [torch.zeros_like(a) for a in accs]
    shape = ab.autotune_batch([(s, j, a.data_ptr()) for (s, j), a in zip(jobs, untouched)])
    torch.cuda.synchronize()
    for a in untouched:
        assert torch.count_nonzero(a).item() == 0
    assert shape["trace_blocks_per_sm"] in (3, 4, 5)
    assert shape["fetch_batch"] in (16, 32, 64, 128)
    assert shape["blocks_per_sm"] in (4, 8, 16)
    assert shape["iterations_per_graph"] in (2, 4, 8)
    assert shape["slot_count"] in (1 << 17, 1 << 18, 1 << 19, 1 << 20, 1 << 21, 1 << 22)
    assert shape["trace_loop"] in (0, 1, 2)
    assert shape["evaluations"] >= 13 and shape["best_ms"] <= shape["default_ms"]
    kept = ab.tuning()
    assert all(kept[k] == shape[k] for k in ("trace_blocks_per_sm", "fetch_batch", "trace_loop", "blocks_per_sm",
                                             "iterations_per_graph", "slot_count"))
    for a in accs:
        a.zero_()
    ab.render_batch([(s, j, a.data_ptr()) for (s, j), a in zip(jobs, accs)])
    torch.cuda.synchronize()
    for a, b in zip(accs, before):
        assert_same_image(a.cpu().numpy(), b)
    ab.wavefront_configure()  # back to the default shape for the tests that follow


def test_camera_view_matches_the_scene_camera_and_methods_agree(room_path):
    scene = ab.Scene.load(room_path)
    job = ab.RenderJob(96, 54, samples_per_axis=3, max_depth=8)
    own = render(scene, job)
    same = scene_camera(room_path)
    np.testing.assert_array_equal(render(scene, job, same), own)
    f = same.look_from
    moved = ab.Camera((f[0] + 0.5, f[1] + 0.2, f[2]), same.look_at, same.up, same.vertical_fov_degrees * 0.8)
    mega = render(scene, job, moved)
    assert not np.allclose(mega[:, :3], own[:, :3])
    wave = render(scene, ab.RenderJob(96, 54, samples_per_axis=3, max_depth=8, method=ab.WAVEFRONT), moved)
    assert_same_image(wave, mega)
    with pytest.raises(ValueError):
        render(scene, job, ab.Camera(same.look_from, same.look_from, same.up, same.vertical_fov_degrees))


def test_server_renders_each_request_from_its_own_camera(room_path):
    scene = ab.Scene.load(room_path)
    own = scene_camera(room_path)
    f = own.look_from
    views = [ab.Camera((f[0] + dx, f[1], f[2]), own.look_at, own.up, own.vertical_fov_degrees)
             for dx in (-0.4, 0.0, 0.4)]
    job = ab.RenderJob(80, 45, samples_per_axis=2, max_depth=8, method=ab.WAVEFRONT)
    server = ab.Server(memory_budget_bytes=4 << 30, slots=1 << 16)
    accs = [torch.zeros((80 * 45, 4), dtype=torch.float64, device="cuda") for _ in views]
    for view, acc in zip(views, accs):
        server.submit(scene, job, acc.data_ptr(), camera=view)
    finished = []
    while len(finished) < len(views):
        finished += server.step()
    torch.cuda.synchronize()
    server.close()
    for view, acc in zip(views, accs):
        assert_same_image(acc.cpu().numpy(), render(scene, job, view))


def test_kahan_fp32_accumulation_matches_fp64(trefoil_path):
    scene = ab.Scene.load(trefoil_path)
    base = dict(width=96, height=54, samples_per_axis=16, max_depth=10)
    fp64 = render(scene, ab.RenderJob(**base))
    kahan = render(scene, ab.RenderJob(**base, accumulation=ab.ACCUMULATE_KAHAN_FP32))
    np.testing.assert_array_equal(counts(kahan), counts(fp64))
    # Sums of 256 FP32 samples with compensation: within a few FP32 ulps of FP64.
    rel = np.abs(kahan[:, :3] - fp64[:, :3]) / np.maximum(np.abs(fp64[:, :3]), 1e-30)
    assert np.max(rel[np.abs(fp64[:, :3]) > 1e-6]) < 1e-6
    with pytest.raises(ab.Unsupported):
        render(scene, ab.RenderJob(**base, method=ab.WAVEFRONT, accumulation=ab.ACCUMULATE_KAHAN_FP32))
