"""The render server: continuous batching (and the express route beside it)
gives each request the image it gets alone (GPU).

Requests are submitted while others are already running on the device; each
finished result is compared with the same job rendered alone by the wavefront.
A request the batch rendered must equal it bit for bit: the batch runs the same
kernels on the same per-pixel random streams, and a pixel's samples are summed
in the same order whichever slot renders them. A request the express route
rendered (the megakernel, compiled separately, so FP32 rounding can split a
path) gets the tolerance between the two forms: identical sample counts, image
sums within 1e-4 relative, at most 0.5% of pixels differing by more than 1e-3
relative. A second run uses a memory budget that admits one request at a time,
so later requests wait.
"""

import numpy as np
import pytest
import torch

import albedo_b200 as ab

pytestmark = pytest.mark.gpu


def counts(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a[:, 3]).view(np.int64)


def assert_same_image(a: np.ndarray, b: np.ndarray):
    np.testing.assert_array_equal(counts(a), counts(b))
    ca, cb = a[:, :3], b[:, :3]
    assert np.abs(ca.sum() - cb.sum()) / cb.sum() < 1e-4
    rel = np.abs(ca - cb) / np.maximum(np.abs(cb), 1e-3)
    assert np.mean(rel.max(axis=1) > 1e-3) < 0.005


def assert_identical(a: np.ndarray, b: np.ndarray):
    np.testing.assert_array_equal(a.view(np.int64), b.view(np.int64))


def alone(scene, job) -> np.ndarray:
    acc = torch.zeros((job.width * job.height, 4), dtype=torch.float64, device="cuda")
    ab.render_device(scene, job, acc.data_ptr())
    torch.cuda.synchronize()
    return acc.cpu().numpy()


def requests(room, trefoil):
    return [(room, ab.RenderJob(160, 90, samples_per_axis=4, seed=11, max_depth=8, method=ab.WAVEFRONT)),
            (trefoil, ab.RenderJob(96, 54, samples_per_axis=2, seed=12, max_depth=10, method=ab.WAVEFRONT)),
            (room, ab.RenderJob(64, 36, samples_per_axis=3, seed=13, max_depth=64, method=ab.WAVEFRONT)),
            (trefoil, ab.RenderJob(128, 72, samples_per_axis=3, seed=14, max_depth=6, method=ab.WAVEFRONT))]


def serve(server, items, stagger=True):
    accs = [torch.zeros((j.width * j.height, 4), dtype=torch.float64, device="cuda") for _, j in items]
    tickets = {}
    done = set()
    # The first request starts alone; the others arrive while it runs.
    tickets[server.submit(items[0][0], items[0][1], accs[0].data_ptr())] = 0
    steps = 0
    for k, (scene, job) in enumerate(items[1:], start=1):
        if stagger:
            done.update(server.step())
            steps += 1
        tickets[server.submit(scene, job, accs[k].data_ptr())] = k
    while len(done) < len(items):
        done.update(server.step())
        steps += 1
        assert steps < 100000
    torch.cuda.synchronize()
    assert set(tickets) == done
    return [a.cpu().numpy() for a in accs]


@pytest.mark.parametrize("express_pixels", [0, 65536])
def test_each_request_is_the_same_alone_and_in_the_mix(room_path, trefoil_path, express_pixels):
    """express_pixels 0: every request joins the batch on the device; 65536: small
    requests arriving while the batch is light take the megakernel route beside it."""
    room, trefoil = ab.Scene.load(room_path), ab.Scene.load(trefoil_path)
    items = requests(room, trefoil)
    server = ab.Server(memory_budget_bytes=8 << 30, slots=1 << 16, express_pixels=express_pixels)
    results = serve(server, items)
    assert server.pending() == (0, 0)
    batched, express = server.routes()
    assert batched + express == len(items) and (express == 0) == (express_pixels == 0)
    for (scene, job), result in zip(items, results):
        if express_pixels == 0:
            assert_identical(result, alone(scene, job))
        else:
            assert_same_image(result, alone(scene, job))
    server.close()


def test_requests_wait_for_memory_and_still_match(room_path, trefoil_path):
    room, trefoil = ab.Scene.load(room_path), ab.Scene.load(trefoil_path)
    items = requests(room, trefoil)
    slots = 1 << 14
    # Budget: the slot pool, both scenes and the largest request's accumulators,
    # so at most one or two requests fit at once and the rest wait.
    slot_bytes = slots * 264 + (1 << 20)
    scene_bytes = room.info()["device_bytes"] + trefoil.info()["device_bytes"]
    budget = slot_bytes + scene_bytes + 160 * 90 * 32 + 64 * 36 * 32 + (4 << 20)
    server = ab.Server(memory_budget_bytes=budget, slots=slots, express_pixels=0)
    accs = [torch.zeros((j.width * j.height, 4), dtype=torch.float64, device="cuda") for _, j in items]
    for (scene, job), acc in zip(items, accs):
        server.submit(scene, job, acc.data_ptr())
    waiting, running = server.pending()
    assert waiting >= 1 and running >= 1
    finished = []
    while len(finished) < len(items):
        finished += server.step()
    torch.cuda.synchronize()
    for (scene, job), acc in zip(items, accs):
        assert_identical(acc.cpu().numpy(), alone(scene, job))
    server.close()


def test_a_request_larger_than_the_budget_is_refused(room_path):
    room = ab.Scene.load(room_path)
    server = ab.Server(memory_budget_bytes=(1 << 14) * 264 + (8 << 20), slots=1 << 14)
    acc = torch.zeros((1024 * 576, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="exceeds the server's memory budget"):
        server.submit(room, ab.RenderJob(1024, 576, method=ab.WAVEFRONT), acc.data_ptr())
    server.close()


def test_releasing_a_scene_frees_its_share_of_the_budget(trefoil_path, tmp_path):
    from albedo_b200 import scenes

    first_scene = ab.Scene.load(trefoil_path)
    second_scene = ab.Scene.load(scenes.trefoil_scene(tmp_path / "other", seed=8))
    sizes = [first_scene.info()["device_bytes"], second_scene.info()["device_bytes"]]
    slots = 1 << 14
    # Budget: the slot pool and job table (264 B a slot, ray binning included,
    # plus about 1.2 MB), one scene and two small frames; the slack left is
    # smaller than either scene, so both scenes never fit at once.
    frame = 64 * 36 * 32
    budget = slots * 264 + (2 << 20) + max(sizes) + 2 * frame
    assert min(sizes) > (1 << 20) + 2 * frame
    server = ab.Server(memory_budget_bytes=budget, slots=slots, express_pixels=0)
    job = ab.RenderJob(64, 36, samples_per_axis=2, max_depth=8, method=ab.WAVEFRONT)
    a = torch.zeros((64 * 36, 4), dtype=torch.float64, device="cuda")
    b = torch.zeros((64 * 36, 4), dtype=torch.float64, device="cuda")
    first = server.submit(first_scene, job, a.data_ptr())
    with pytest.raises(ValueError, match="still has requests"):
        server.release_scene(first_scene)
    done = []
    while first not in done:
        done += server.step()
    second = server.submit(second_scene, job, b.data_ptr())
    assert server.pending() == (1, 0)  # the first scene's tables still count
    server.release_scene(first_scene)
    assert server.pending() == (0, 1)
    while second not in done:
        done += server.step()
    torch.cuda.synchronize()
    assert_identical(a.cpu().numpy(), alone(first_scene, job))
    assert_identical(b.cpu().numpy(), alone(second_scene, job))
    server.close()


def test_express_route_runs_beside_a_busy_batch(room_path, trefoil_path):
    """A large request fills the batch; a small one of the same scene that arrives
    then joins the batch (the batch is not light), and a small one needing a
    deeper traversal stack than the open batch takes the express route rather
    than wait for the batch to drain. Once the batch drains, a small request
    takes the express route. Every result equals its render alone."""
    room, trefoil = ab.Scene.load(room_path), ab.Scene.load(trefoil_path)
    assert trefoil.info()["stack_capacity"] > room.info()["stack_capacity"]
    big = ab.RenderJob(640, 480, samples_per_axis=2, seed=3, max_depth=8, method=ab.WAVEFRONT)  # 307,200 pixels
    small = ab.RenderJob(96, 54, samples_per_axis=3, seed=4, max_depth=10, method=ab.WAVEFRONT)
    server = ab.Server(memory_budget_bytes=8 << 30, slots=1 << 19, express_pixels=65536)
    jobs = [(room, big), (room, small), (trefoil, small), (room, small)]
    accs = [torch.zeros((j.width * j.height, 4), dtype=torch.float64, device="cuda") for _, j in jobs]
    tickets = [server.submit(room, big, accs[0].data_ptr()), server.submit(room, small, accs[1].data_ptr())]
    assert server.routes() == (2, 0)
    tickets.append(server.submit(trefoil, small, accs[2].data_ptr()))
    assert server.routes() == (2, 1)
    done = []
    while not all(t in done for t in tickets):
        done += server.step()
    tickets.append(server.submit(room, small, accs[3].data_ptr()))
    assert server.routes() == (2, 2)
    while tickets[-1] not in done:
        done += server.step()
    torch.cuda.synchronize()
    server.close()
    # The first two went to the batch, the last two took the express route.
    for k, ((scene, job), acc) in enumerate(zip(jobs, accs)):
        if k < 2:
            assert_identical(acc.cpu().numpy(), alone(scene, job))
        else:
            assert_same_image(acc.cpu().numpy(), alone(scene, job))
