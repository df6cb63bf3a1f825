#!/usr/bin/env python
"""Throughput of the path-tracing hot path on one or more B200s.

Workload (the instanced-mesh configuration): three instances of a seeded trefoil
tube (256 x 32 ring vertices, 16,384 smooth triangles, uniform scale 0.8-1.2,
seeded y-rotation) in gold, glass and copper on a 2-triangle checker floor inside
a room of radius-1e4 wall spheres, with an area light, a point light and a sky;
960 x 540 pixels, 8 x 8 = 64 stratified samples per pixel, PathEstimator
max_depth 10, roulette_start 3, seed 0. One step renders the full frame:
33,177,600 paths.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--method megakernel|wavefront]

Prints one JSON line. `value` is whole-job Mpaths/s with the scene and the
accumulators resident in HBM, timed with CUDA events per step and L2 flushed
(a 256 MiB write) between steps. `e2e` is the same metric through the C-ABI
call that takes host (pinned) accumulators: the host-to-device copy, the render
and the device-to-host copy of the frame's accumulators are inside each timed
step. `roofline` divides the algorithmic bytes of one launch (32 B per BVH box
tested, 48 B per triangle, 32 B per sphere, 96 B per instance entered, counted
on the device in an untimed counting launch) by the launch's measured time.
`cpu_baseline` is the reference renderer, built from its own sources, timed on
this machine's host cores over a band of rows of the same frame.

Under torchrun (N > 1) every rank renders its own replica of the frame (the path
does not shard across GPUs without changing per-pixel random streams, so the
runs are replicas); the time is the maximum over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WIDTH, HEIGHT, SAMPLES_PER_AXIS, MAX_DEPTH, ROULETTE_START, SEED = 960, 540, 8, 10, 3, 0
PATHS_PER_STEP = WIDTH * HEIGHT * SAMPLES_PER_AXIS * SAMPLES_PER_AXIS
METRIC = "Mpaths/s at matched RMSE vs plain GPU + host CPU; p50/p99 render latency"
WORKLOAD = "trefoil_x3_instanced_960x540_64spp_depth10"
L2_FLUSH_BYTES = 256 << 20


def parse_args():
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--method", choices=["megakernel", "wavefront"], default="megakernel")
    p.add_argument("--workload", choices=["trefoil", "batched", "served", "precision"], default="trefoil",
                   help="trefoil: the instanced-mesh frame (default); batched: 64 seeded jobs of uneven size; "
                        "served: Poisson request streams over 16 resident scenes; precision: 1.31M- and "
                        "1M-triangle meshes at 1920x1080, 256 spp, FP64 vs compensated FP32 sums")
    p.add_argument("--rates", default="10,50,100,200,500", help="served: arrival rates (requests/s) to sweep")
    p.add_argument("--requests", type=int, default=96, help="served: requests per rate")
    p.add_argument("--no-forms", action="store_true",
                   help="trefoil: skip the wavefront frame and the 64-job batched comparison in the line")
    return p.parse_args()


def wavefront_frame(scene, flush, steps: int = 3) -> dict:
    """The same frame rendered by the wavefront form (autotuned on it), timed
    with CUDA events per step, L2 flushed between steps."""
    import torch

    import albedo_b200 as ab

    job = ab.RenderJob(WIDTH, HEIGHT, samples_per_axis=SAMPLES_PER_AXIS, seed=SEED, max_depth=MAX_DEPTH,
                       roulette_start=ROULETTE_START, method=ab.WAVEFRONT)
    accum = torch.zeros((WIDTH * HEIGHT, 4), dtype=torch.float64, device="cuda")
    shape = ab.autotune_batch([(scene, job, accum.data_ptr())])
    ab.render_device(scene, job, accum.data_ptr())
    torch.cuda.synchronize()
    ms = []
    for i in range(steps):
        flush.fill_(i & 0xFF)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        ab.render_device(scene, job, accum.data_ptr())
        end.record()
        end.synchronize()
        ms.append(start.elapsed_time(end))
    scene.check()
    s = statistics.mean(ms) / 1e3
    return {"mpaths_per_s": PATHS_PER_STEP / s / 1e6, "mrays_per_s": ab.wavefront_last_rays() / s / 1e6,
            "ms_per_step": s * 1e3, "steps": steps, "iterations": ab.wavefront_last_iterations(), "autotune": shape}


RESOLVE_WIDTH, RESOLVE_HEIGHT = 3840, 2160
RESOLVE_BYTES_PER_PIXEL = 32 + 3  # one accumulator read, three sRGB bytes written


def film_resolve_figures(flush, launches: int = 20) -> dict:
    """The film's device resolve (accumulators to sRGB bytes, bit-exact with the
    reference's writePpm bytes) on a 3840 x 2160 frame: 265 MB of accumulators,
    more than L2. Between launches a 256 MB read evicts them from L2 and leaves
    it clean (a flush by writing would leave up to 126 MB of dirty lines for the
    timed launch to write back). Each launch is timed with CUDA events.
    Algorithmic bytes: 32 read and 3 written per pixel. Two sample counts: 64
    (the bench frame's; a power of two, so the average is one multiplication) and
    36 (an FP64 division per channel)."""
    import torch

    import albedo_b200 as ab

    pixels = RESOLVE_WIDTH * RESOLVE_HEIGHT
    out = torch.empty(3 * pixels, dtype=torch.uint8, device="cuda")
    peak = measured_peaks().get("hbm_gbs") or 6650.0
    figures = {}
    for count in (64, 36):
        generator = torch.Generator(device="cuda").manual_seed(5)
        acc = torch.rand((pixels, 4), dtype=torch.float64, device="cuda", generator=generator) * count
        acc.view(torch.int64)[:, 3] = count
        for _ in range(3):
            ab.resolve_srgb(acc.data_ptr(), RESOLVE_WIDTH, RESOLVE_HEIGHT, out.data_ptr())
        torch.cuda.synchronize()
        ms = []
        for _ in range(launches):
            flush.max()
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            ab.resolve_srgb(acc.data_ptr(), RESOLVE_WIDTH, RESOLVE_HEIGHT, out.data_ptr())
            end.record()
            end.synchronize()
            ms.append(start.elapsed_time(end))
        del acc
        launch_s = statistics.median(ms) / 1e3
        achieved = RESOLVE_BYTES_PER_PIXEL * pixels / launch_s / 1e9
        figures[f"samples_{count}"] = {
            "us_per_launch": launch_s * 1e6, "gpixels_per_s": pixels / launch_s / 1e9,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "algorithmic_bytes_per_launch": RESOLVE_BYTES_PER_PIXEL * pixels}}
    return {"workload": f"{RESOLVE_WIDTH}x{RESOLVE_HEIGHT} accumulators to sRGB bytes", "launches": launches,
            "l2": "256 MB read between launches (clean L2; inputs larger than L2)", **figures,
            "d2h_bytes_per_frame": {"accumulators": 32 * pixels, "srgb": 3 * pixels}}


def served_figures(rates: list[float], requests: int) -> list[dict]:
    """Poisson request streams (seeded) drawn from the batched-job distribution
    over 16 resident scenes, each request with its own seeded camera around its
    scene's, served under a 150 GB device budget: the continuous-batching server
    against the plain megakernel serving one request at a time in arrival order.
    Both use autotuned shapes (tuned before the streams start). Latency is
    completion minus arrival (wall clock); throughput is paths over the time from
    the first arrival to the last completion, where a request completes when its
    image is on the host as sRGB bytes (device resolve, then a copy of 3 bytes a
    pixel to pinned memory). The server's batch_mrays_per_s
    counts the rays its wavefront batch traced (not the express route's)."""
    import torch

    import albedo_b200 as ab
    from albedo_b200 import scenes

    tmp = tempfile.TemporaryDirectory()
    pool = scenes.batch_jobs(Path(tmp.name), count=16, scenes=16)
    loaded = [ab.Scene.load(j.scene) for j in pool]
    base_views = [scenes.scene_camera(j.scene) for j in pool]
    # Tuning (and warm-up): the megakernel per scene on its pool job, the
    # wavefront on the pool's jobs as one batch.
    tune_start = time.perf_counter()
    warm = [torch.zeros((j.width * j.height, 4), dtype=torch.float64, device="cuda") for j in pool]
    for scene, j in zip(loaded, pool):
        ab.autotune_megakernel(scene, ab.RenderJob(j.width, j.height, samples_per_axis=j.samples_per_axis,
                                                   max_depth=8))
    wave_shape = ab.autotune_batch([(scene, ab.RenderJob(j.width, j.height, samples_per_axis=j.samples_per_axis,
                                                         max_depth=8, method=ab.WAVEFRONT), a.data_ptr())
                                    for scene, j, a in zip(loaded, pool, warm)])
    tune_s = time.perf_counter() - tune_start
    del warm
    rng = np.random.default_rng(2024)
    results = []
    for rate in rates:
        gaps = rng.exponential(1.0 / rate, size=requests)
        arrivals = np.cumsum(gaps) - gaps[0]
        reqs = []
        for k in range(requests):
            w, h = scenes.RESOLUTIONS[int(rng.integers(0, 4))]
            n = int(np.clip(round(np.sqrt(np.exp(rng.uniform(np.log(4), np.log(64))))), 2, 8))
            sid = int(rng.integers(0, 16))
            view = ab.Camera(*scenes.request_view(base_views[sid], rng))
            reqs.append((sid, w, h, n, k, view))
        paths = sum(w * h * n * n for _, w, h, n, _, _ in reqs)
        accs = [torch.zeros((w * h, 4), dtype=torch.float64, device="cuda") for _, w, h, _, _, _ in reqs]
        srgb_dev = [torch.empty(3 * w * h, dtype=torch.uint8, device="cuda") for _, w, h, _, _, _ in reqs]
        srgb_host = [torch.empty(3 * w * h, dtype=torch.uint8).pin_memory() for _, w, h, _, _, _ in reqs]
        delivery = torch.cuda.Stream()

        def deliver(k):
            # The finished image reaches the host as sRGB bytes: resolved on the
            # device, 3 bytes a pixel copied instead of 32 of accumulators.
            _, w, h, _, _, _ = reqs[k]
            with torch.cuda.stream(delivery):
                ab.resolve_srgb(accs[k].data_ptr(), w, h, srgb_dev[k].data_ptr(), stream=delivery.cuda_stream)
                srgb_host[k].copy_(srgb_dev[k], non_blocking=True)
            delivery.synchronize()

        def job(r, method):
            _, w, h, n, seed, _ = r
            return ab.RenderJob(w, h, samples_per_axis=n, seed=seed, max_depth=8, method=method)

        # Continuous batching.
        server = ab.Server(memory_budget_bytes=150 << 30, slots=1 << 20)
        done_at = {}
        ticket_of = {}
        submitted = 0
        rays = 0
        last_rays = 0
        torch.cuda.synchronize()
        start = time.perf_counter()
        while len(done_at) < len(reqs):
            now = time.perf_counter() - start
            while submitted < len(reqs) and arrivals[submitted] <= now:
                r = reqs[submitted]
                ticket = server.submit(loaded[r[0]], job(r, ab.WAVEFRONT), accs[submitted].data_ptr(), camera=r[5])
                ticket_of[ticket] = submitted
                submitted += 1
            finished = server.step()
            now = time.perf_counter() - start
            for t in finished:
                deliver(ticket_of[t])
                done_at[ticket_of[t]] = time.perf_counter() - start
            count = server.rays()
            rays += count - last_rays if count >= last_rays else count
            last_rays = count
            waiting, running = server.pending()
            if waiting == 0 and running == 0 and submitted < len(reqs):
                time.sleep(max(0.0, arrivals[submitted] - (time.perf_counter() - start)))
        routes = server.routes()
        server.close()
        lat_server = np.array([done_at[k] - arrivals[k] for k in range(len(reqs))])
        span_server = max(done_at.values()) - arrivals[0]

        # One request at a time, megakernel.
        torch.cuda.synchronize()
        start = time.perf_counter()
        finish = []
        for k, r in enumerate(reqs):
            now = time.perf_counter() - start
            if now < arrivals[k]:
                time.sleep(arrivals[k] - now)
            ab.render_device(loaded[r[0]], job(r, ab.MEGAKERNEL), accs[k].data_ptr(), camera=r[5])
            torch.cuda.synchronize()
            deliver(k)
            finish.append(time.perf_counter() - start)
        lat_mega = np.array(finish) - arrivals
        span_mega = finish[-1] - arrivals[0]
        results.append({
            "rate_per_s": rate, "requests": len(reqs), "paths": paths,
            "server": {"mpaths_per_s": paths / span_server / 1e6, "batch_mrays_per_s": rays / span_server / 1e6,
                       "routed_batch": routes[0], "routed_express": routes[1],
                       "p50_ms": float(np.percentile(lat_server, 50) * 1e3),
                       "p99_ms": float(np.percentile(lat_server, 99) * 1e3)},
            "megakernel_one_at_a_time": {"mpaths_per_s": paths / span_mega / 1e6,
                                         "p50_ms": float(np.percentile(lat_mega, 50) * 1e3),
                                         "p99_ms": float(np.percentile(lat_mega, 99) * 1e3)},
            "speedup_over_megakernel": span_mega / span_server})
    for s in loaded:
        s.check()
    return [{"autotune": {"seconds": tune_s, "wavefront": wave_shape}}] + results


def run_served(args) -> None:
    """The served form as its own bench line: value is the server's best Mpaths/s
    over the swept arrival rates (see served_figures)."""
    with ClockSampler(0) as clocks:
        figures = served_figures([float(r) for r in args.rates.split(",")], args.requests)
    tuning, results = figures[0], figures[1:]
    best = max(r["server"]["mpaths_per_s"] for r in results)
    line = {"metric": METRIC, "value": best, "unit": "Mpaths/s", "n_gpus": 1, "steps": len(results), "warmup": 0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene files, seeded Poisson arrivals and cameras)",
            "config": {"workload": "served_poisson_16_scenes", "budget_bytes": 150 << 30, "slots": 1 << 20,
                       "max_depth": 8, "timing": "wall clock from arrival to observed completion"},
            "autotune": tuning["autotune"], "sweep": results, "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)


def run_precision(args) -> None:
    """The precision form at full size: a displaced icosphere of 8 levels
    (1,310,720 triangles) in rough glass and a 1,000,000-triangle random soup,
    1920 x 1080 at 16 x 16 = 256 spp, PathEstimator max_depth 16. For each scene:
    megakernel frames with FP64 and with Kahan-compensated FP32 per-pixel sums
    (the same autotuned shape for both, CUDA events, L2 flushed between steps)
    and a wavefront frame; the error of every image against the FP64 oracle (the
    reference renderer at 65,536 spp on 256 seeded pixels, host cores) next to
    the reference renderer's own error at 256 spp on the same pixels; and the
    largest relative difference between the two accumulation modes."""
    import torch

    import albedo_b200 as ab
    from albedo_b200 import scenes
    from oracle import reference as ref

    width, height, n, depth = 1920, 1080, 16, 16
    paths = width * height * n * n
    rng = np.random.default_rng(91)
    pixels = np.stack([rng.integers(0, width, 256), rng.integers(0, height, 256)], axis=1).astype(np.int32)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    tmp = tempfile.TemporaryDirectory()
    results = []
    with ClockSampler(0) as clocks:
        for name, make in (("icosphere_8_levels", scenes.icosphere_scene), ("soup_1M", scenes.soup_scene)):
            path = make(Path(tmp.name) / name)
            t0 = time.perf_counter()
            scene = ab.Scene.load(path)
            load_s = time.perf_counter() - t0
            info = scene.info()
            frames = {}
            images = {}
            for label, method, accumulation in (("megakernel_fp64", ab.MEGAKERNEL, ab.ACCUMULATE_FP64),
                                                ("megakernel_kahan_fp32", ab.MEGAKERNEL, ab.ACCUMULATE_KAHAN_FP32),
                                                ("wavefront_fp64", ab.WAVEFRONT, ab.ACCUMULATE_FP64)):
                job = ab.RenderJob(width, height, samples_per_axis=n, seed=0, max_depth=depth, method=method,
                                   accumulation=accumulation)
                acc = torch.zeros((width * height, 4), dtype=torch.float64, device="cuda")
                if label == "megakernel_fp64":
                    # Both accumulation modes run the shape tuned here.
                    ab.autotune_megakernel(scene, job)
                elif method == ab.WAVEFRONT:
                    ab.autotune_batch([(scene, job, acc.data_ptr())])
                steps = args.steps if method == ab.MEGAKERNEL else 1
                ms = []
                for i in range(steps):
                    acc.zero_()
                    flush.fill_(i & 0xFF)
                    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    start.record()
                    ab.render_device(scene, job, acc.data_ptr())
                    end.record()
                    end.synchronize()
                    ms.append(start.elapsed_time(end))
                scene.check()
                frames[label] = {"mpaths_per_s": paths / (statistics.mean(ms) / 1e3) / 1e6,
                                 "ms_per_frame": statistics.mean(ms), "steps": steps}
                images[label] = acc.cpu().numpy()
            reference = ref.RefScene(path)
            t0 = time.perf_counter()
            oracle_sum, _ = reference.render_pixels(width, height, 256, pixels, seed=1000003, max_depth=depth)
            oracle_s = time.perf_counter() - t0
            oracle = oracle_sum / 65536.0
            theirs_sum, _ = reference.render_pixels(width, height, n, pixels, seed=0, max_depth=depth)
            lum = oracle.mean(axis=1)
            keep = lum > 1e-3

            def errors(rgb):
                err = (rgb - oracle)[keep] / lum[keep, None]
                return {"rel_rmse": float(np.sqrt(np.mean(err ** 2))), "mean_rel": float(np.mean(np.abs(err)))}

            index = pixels[:, 1] * width + pixels[:, 0]
            err = {label: errors(img[index, :3] / (n * n)) for label, img in images.items()}
            err["reference_cpu_256spp"] = errors(theirs_sum / (n * n))
            fp64, kahan = images["megakernel_fp64"][:, :3], images["megakernel_kahan_fp32"][:, :3]
            lit = np.abs(fp64) > 1e-9
            results.append({"scene": name, "triangles": info["triangles"], "bvh_nodes": info["nodes"],
                            "device_bytes": info["device_bytes"], "load_s": load_s, "frames": frames,
                            "error_vs_fp64_oracle": err,
                            "oracle": {"pixels": 256, "spp": 65536, "seconds": oracle_s},
                            "kahan_vs_fp64_max_rel": float(np.max(np.abs(kahan - fp64)[lit] / np.abs(fp64)[lit])),
                            "tuned_megakernel": {k: ab.tuning(scene)[k]
                                                 for k in ("tile_width", "blocks_per_sm", "inline_traversal")}})
            scene.close()
    value = statistics.mean(r["frames"]["megakernel_fp64"]["mpaths_per_s"] for r in results)
    line = {"metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": 1, "steps": args.steps, "warmup": 0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded meshes written as OBJ)",
            "config": {"workload": "precision_large_meshes_1920x1080_256spp", "max_depth": depth,
                       "value": "mean over the two scenes of the FP64-accumulation megakernel"},
            "scenes": results, "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)


def batched_figures(steps: int, warmup: int, count: int = 64) -> dict:
    """`count` seeded jobs of uneven size (displaced icospheres of 1k-500k
    triangles, 0-8 spheres, mixed materials, 128x72..1024x576, 4-64 spp), one
    scene each: one batched wavefront run of all of them against the plain
    megakernel serving them one at a time (a synchronize after each). Both forms
    run with the shapes the autotuner picked (per scene for the megakernel, for
    the batch for the wavefront); tuning is outside the timed region."""
    import torch

    import albedo_b200 as ab
    from albedo_b200 import scenes

    tmp = tempfile.TemporaryDirectory()
    jobs = scenes.batch_jobs(Path(tmp.name), count=count)
    loaded = {j.scene: ab.Scene.load(j.scene) for j in jobs}
    paths = sum(j.width * j.height * j.samples_per_axis ** 2 for j in jobs)
    accs = [torch.zeros((j.width * j.height, 4), dtype=torch.float64, device="cuda") for j in jobs]

    def rjob(j, method):
        return ab.RenderJob(j.width, j.height, samples_per_axis=j.samples_per_axis, seed=j.seed, max_depth=8,
                            method=method)

    items = [(loaded[j.scene], rjob(j, ab.WAVEFRONT), a.data_ptr()) for j, a in zip(jobs, accs)]
    tune_start = time.perf_counter()
    mega_shapes = [ab.autotune_megakernel(loaded[j.scene], rjob(j, ab.MEGAKERNEL)) for j in jobs]
    wave_shape = ab.autotune_batch(items)
    tune_s = time.perf_counter() - tune_start
    counts = [ab.work_counts(loaded[j.scene], rjob(j, ab.MEGAKERNEL)) for j in jobs]
    alg_bytes = sum(ab.algorithmic_bytes(c) for c in counts)

    def one_at_a_time():
        for j, a in zip(jobs, accs):
            ab.render_device(loaded[j.scene], rjob(j, ab.MEGAKERNEL), a.data_ptr())
            torch.cuda.synchronize()

    def batched():
        ab.render_batch(items)
        torch.cuda.synchronize()

    def timed(fn):
        for _ in range(warmup):
            fn()
        ms = []
        for _ in range(steps):
            torch.cuda.synchronize()
            start = time.perf_counter()
            fn()
            ms.append((time.perf_counter() - start) * 1e3)
        return ms

    with ClockSampler(0) as clocks:
        batch_ms = timed(batched)
        rays = ab.wavefront_last_rays()
        mega_ms = timed(one_at_a_time)
    for s in loaded.values():
        s.check()
    batch_s = statistics.mean(batch_ms) / 1e3
    mega_s = statistics.mean(mega_ms) / 1e3
    peak = measured_peaks().get("hbm_gbs") or 6650.0
    tiles = {}
    for shape in mega_shapes:
        key = (f"{shape['tile_width']}x{128 // shape['tile_width']}/{shape['blocks_per_sm']}"
               + ("/inline" if shape["inline_traversal"] else ""))
        tiles[key] = tiles.get(key, 0) + 1
    return {
        "jobs": len(jobs), "paths_per_step": paths,
        "wavefront": {"mpaths_per_s": paths / batch_s / 1e6, "mrays_per_s": rays / batch_s / 1e6,
                      "ms_per_step": batch_s * 1e3, "rays_per_step": rays,
                      "traversal_gbs": alg_bytes / batch_s / 1e9, "traversal_frac_of_hbm": alg_bytes / batch_s / 1e9 / peak,
                      "iterations": ab.wavefront_last_iterations()},
        "megakernel_one_at_a_time": {"mpaths_per_s": paths / mega_s / 1e6, "ms_per_step": mega_s * 1e3},
        "speedup_over_megakernel": mega_s / batch_s,
        "autotune": {"seconds": tune_s, "wavefront": wave_shape, "megakernel_shapes": tiles},
        "algorithmic_bytes_per_step": alg_bytes,
        "timing": "wall clock around each step, device synchronized on both sides",
        "clocks": clocks.summary(),
        "jobs_detail": [[j.width, j.height, j.samples_per_axis ** 2] for j in jobs],
    }


def run_batched(args) -> None:
    """The batched form as its own bench line: value is the batched wavefront's
    Mpaths/s over 64 seeded jobs (see batched_figures)."""
    fig = batched_figures(args.steps, args.warmup)
    line = {"metric": METRIC, "value": fig["wavefront"]["mpaths_per_s"], "unit": "Mpaths/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": fig["wavefront"]["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene files)",
            "config": {"workload": "batched_64_jobs_mixed", "max_depth": 8,
                       "method": "wavefront batch (one run for all jobs), autotuned"},
            "batched": fig, "clocks": fig["clocks"]}
    print(json.dumps(line), flush=True)


def config(method: str, n_gpus: int) -> dict:
    return {"workload": WORKLOAD, "resolution": [WIDTH, HEIGHT], "samples_per_axis": SAMPLES_PER_AXIS,
            "spp": SAMPLES_PER_AXIS ** 2, "max_depth": MAX_DEPTH, "roulette_start": ROULETTE_START, "seed": SEED,
            "paths_per_step": PATHS_PER_STEP, "method": method,
            "parallelism": "replicas" if n_gpus > 1 else "single",
            "l2": "flushed between steps (256 MiB write)"}


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu_index = gpu_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu_index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self) -> dict | None:
        rows = []
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append({"sm": float(parts[1]), "max": float(parts[2]), "power": float(parts[3]),
                             "hw_slowdown": parts[5], "hw_thermal": parts[6], "sw_thermal": parts[7],
                             "sw_power_cap": parts[8]})
            except ValueError:
                continue
        if not rows:
            return None
        reasons = set()
        for r in rows:
            for key, name in (("hw_slowdown", "hw_slowdown"), ("hw_thermal", "hw_thermal_slowdown"),
                              ("sw_thermal", "sw_thermal_slowdown"), ("sw_power_cap", "sw_power_cap")):
                if r[key].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in rows), "sm_max_mhz": max(r["max"] for r in rows),
                "power_w_max": max(r["power"] for r in rows), "samples": len(rows), "reasons": sorted(reasons)}


def measured_peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        return json.loads(path.read_text())
    return {}


def profiled_traffic() -> tuple[float | None, str | None]:
    """DRAM bytes per launch of the megakernel from the committed ncu summary."""
    path = ROOT / "profiles" / "megakernel_trefoil_960x540.txt"
    if not path.exists():
        return None, None
    for line in path.read_text().splitlines():
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":", 1)[1].split()[0]), path.name
    return None, None


def cpu_baseline_sample(scene_path: Path, target_seconds: float = 12.0) -> dict:
    """The reference renderer on all host cores over a band of full-spp rows."""
    from oracle import reference as ref

    scene = ref.RefScene(scene_path)
    threads = ref.threads()

    def run(rows: int) -> float:
        y0 = HEIGHT // 2 - rows // 2
        xs, ys = np.meshgrid(np.arange(WIDTH), np.arange(y0, y0 + rows))
        pixels = np.stack([xs.ravel(), ys.ravel()], axis=1)
        start = time.perf_counter()
        scene.render_pixels(WIDTH, HEIGHT, SAMPLES_PER_AXIS, pixels, seed=SEED, max_depth=MAX_DEPTH,
                            roulette_start=ROULETTE_START, nthreads=threads)
        return time.perf_counter() - start

    probe_rows = 2
    probe = run(probe_rows)
    rows = int(np.clip(probe_rows * target_seconds / max(probe, 1e-3), probe_rows, HEIGHT))
    seconds = run(rows)
    paths = rows * WIDTH * SAMPLES_PER_AXIS ** 2
    return {"value": paths / seconds / 1e6, "unit": "Mpaths/s", "cores": threads, "kind": "reference",
            "sample": f"{rows} full rows x {WIDTH} px x {SAMPLES_PER_AXIS ** 2} spp through the middle of the frame "
                      f"({paths} paths, {seconds:.1f} s), reference renderImage pixel loop on {threads} threads"}


def run_reference(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    from albedo_b200 import scenes

    with tempfile.TemporaryDirectory() as tmp:
        scene_path = scenes.trefoil_scene(Path(tmp))
        for _ in range(args.warmup):
            cpu_baseline_sample(scene_path, target_seconds=2.0)
        values = []
        samples = []
        for _ in range(args.steps):
            s = cpu_baseline_sample(scene_path, target_seconds=6.0)
            values.append(s["value"])
            samples.append(s)
        value = statistics.median(values)
        base = samples[-1]
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": PATHS_PER_STEP / value / 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded scene files)", "config": config("reference CPU renderer", 1),
                "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": base["cores"], "kind": "reference",
                                 "sample": "each step: " + base["sample"]},
                "e2e": {"value": value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    from albedo_b200.replicas import max_over_ranks, ranks_from_env, whole_job_throughput

    ranks = ranks_from_env()
    rank, world, local_rank = ranks.rank, ranks.world, ranks.local_rank
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "batched":
        if rank == 0:
            run_batched(args)
        return
    if args.workload == "served":
        if rank == 0:
            run_served(args)
        return
    if args.workload == "precision":
        if rank == 0:
            run_precision(args)
        return

    import torch

    import albedo_b200 as ab
    from albedo_b200 import scenes

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod

    def barrier():
        if dist is not None:
            dist.barrier()

    method = ab.WAVEFRONT if args.method == "wavefront" else ab.MEGAKERNEL
    tmp = tempfile.TemporaryDirectory()
    scene_path = scenes.trefoil_scene(Path(tmp.name))
    scene = ab.Scene.load(scene_path)
    job = ab.RenderJob(WIDTH, HEIGHT, samples_per_axis=SAMPLES_PER_AXIS, seed=SEED, max_depth=MAX_DEPTH,
                       roulette_start=ROULETTE_START, method=method)
    accum = torch.zeros((WIDTH * HEIGHT, 4), dtype=torch.float64, device="cuda")
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    # Launch shape from the autotuner (untimed; renders into scratch accumulators).
    if method == ab.MEGAKERNEL:
        tuned = ab.autotune_megakernel(scene, job)
    else:
        tuned = ab.autotune_batch([(scene, job, accum.data_ptr())])

    for _ in range(args.warmup):
        ab.render_device(scene, job, accum.data_ptr())
    torch.cuda.synchronize()
    scene.check()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        for i in range(args.steps):
            flush.fill_(i & 0xFF)
            starts[i].record()
            ab.render_device(scene, job, accum.data_ptr())
            ends[i].record()
        torch.cuda.synchronize()
    barrier()
    scene.check()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_s = max_over_ranks(sum(step_ms), dist, "cuda") / 1e3
    value = whole_job_throughput(PATHS_PER_STEP / 1e6, args.steps, world, total_s)

    # End to end through the host-buffer entry point, pinned accumulators.
    host_accum = torch.zeros((WIDTH * HEIGHT, 4), dtype=torch.float64).pin_memory()
    ab.render_image_ptr(scene, job, host_accum.data_ptr())
    e2e_ms = []
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as e2e_clocks:
        for i in range(args.steps):
            flush.fill_(i & 0xFF)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            ab.render_image_ptr(scene, job, host_accum.data_ptr())
            e.record()
            e.synchronize()
            e2e_ms.append(s.elapsed_time(e))
    barrier()
    e2e_value = whole_job_throughput(PATHS_PER_STEP / 1e6, args.steps, world,
                                     max_over_ranks(sum(e2e_ms), dist, "cuda") / 1e3)
    frame_bytes = WIDTH * HEIGHT * 32

    if rank == 0:
        counts = ab.work_counts(scene, job)
        alg_bytes = ab.algorithmic_bytes(counts)
        launch_s = statistics.mean(step_ms) / 1e3
        peaks = measured_peaks()
        peak = peaks.get("hbm_gbs")
        peak_source = "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)" if peak else "fallback 6650 GB/s"
        peak = peak or 6650.0
        achieved = alg_bytes / launch_s / 1e9
        traffic, traffic_source = profiled_traffic()
        line = {
            "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene files in the reference's formats)",
            "config": config(args.method, world),
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99))},
            "steps_ms": step_ms,
            "mrays_per_s": world * counts["rays"] * args.steps / total_s / 1e6,
            "gpu_launches": args.steps,
            "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": frame_bytes,
                    "d2h_bytes_per_step": frame_bytes, "ms_per_step": statistics.mean(e2e_ms), "steps_ms": e2e_ms,
                    "clocks": e2e_clocks.summary()},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": f"megakernel<{scene.info()['stack_capacity']}, path>",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "work_per_launch": counts, "peak_source": peak_source,
                         "traffic_source": traffic_source},
            "clocks": clocks.summary(),
            "autotune": tuned,
        }
        if world == 1:
            line["cpu_baseline"] = cpu_baseline_sample(scene_path)
            if not args.no_forms:
                line["forms"] = {"wavefront_frame": wavefront_frame(scene, flush),
                                 "batched_64_jobs": batched_figures(1, 1),
                                 "film_resolve": film_resolve_figures(flush)}
        print(json.dumps(line), flush=True)
    scene.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
