#!/usr/bin/env python
"""Throughput of the path-tracing hot path on one or more B200s.

Workload (the large-mesh configuration, the largest that fits one GPU): an
icosphere subdivided 8 levels (1,310,720 triangles) displaced radially by seeded
3-octave Perlin noise (amplitude 0.05), in rough glass (ior 1.5, GGX alpha 0.1),
instanced on a checker floor under an area light, a point light and a sky;
1920 x 1080 pixels, 16 x 16 = 256 stratified samples per pixel, PathEstimator
max_depth 16, roulette_start 3, seed 0. One step renders the full frame:
530,841,600 paths. The plain form (the per-pixel megakernel) renders it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--method megakernel|wavefront] [--no-forms]

Prints one JSON line. `value` is whole-job Mpaths/s with the scene and the
accumulators resident in HBM, timed with CUDA events per step and L2 flushed
(a 256 MiB write) between steps; the scene's tables (about 250 MB) exceed L2
anyway. `e2e` is the same metric through the C-ABI call that takes host
(pinned) accumulators: the host-to-device copy, the render and the
device-to-host copy of the frame's accumulators are inside each timed step.
`roofline` divides the algorithmic bytes of one launch (32 B per BVH box the
reference's traversal tests, 48 B per triangle, 32 B per sphere, 96 B per
instance entered, counted on the device in an untimed counting launch) by the
launch's measured time, against the measured HBM copy peak and, beside it, the
L2 read peak measured in the same run by a read sweep of this library.
`cpu_baseline` is the reference renderer, built from its own sources, timed on
this machine's host cores rendering the same frame through its own renderImage
at 36 samples per pixel. `precision` holds every form's error on this frame
against the FP64 oracle (the reference at 65,536 spp on 2,048 seeded pixels).

`forms` (1 GPU, unless --no-forms) adds the other configurations: the 1M-triangle
random soup at the same frame; the instanced trefoil frame (960x540, 64 spp),
whose scene fits L2, by both forms against the L2 peak; 64 batched jobs of
uneven size in one wavefront run against the megakernel one job at a time; the
served request stream (Poisson arrivals over 16 resident scenes, 1,000 requests
per rate) with p50/p99 latency; and the film resolve to sRGB bytes.

Under torchrun (N > 1) every rank renders its own replica of the frame (the path
does not shard across GPUs without changing per-pixel random streams, so the
runs are replicas); the time is the maximum over ranks.
"""

from __future__ import annotations

import argparse
import json
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from dataclasses import dataclass
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mpaths/s at matched RMSE vs plain GPU + host CPU; p50/p99 render latency"
L2_FLUSH_BYTES = 256 << 20
ROULETTE_START, SEED = 3, 0


@dataclass(frozen=True)
class Frame:
    workload: str
    width: int
    height: int
    samples_per_axis: int
    max_depth: int

    @property
    def paths(self) -> int:
        return self.width * self.height * self.samples_per_axis ** 2


LARGE = Frame("icosphere_8_levels_1310720_tris_rough_glass_1920x1080_256spp_depth16", 1920, 1080, 16, 16)
SOUP = Frame("soup_1000000_tris_1920x1080_256spp_depth16", 1920, 1080, 16, 16)
TREFOIL = Frame("trefoil_x3_instanced_960x540_64spp_depth10", 960, 540, 8, 10)
# The reference renders the large frame at 4 x 4 samples per pixel per step of
# the reference arm (about 4 s on 16 host threads) and at 6 x 6 for the CPU
# baseline in our line (about 10 s): bounded samples of its own renderImage
# call on the same frame (a path's cost does not depend on the pixel's spp).
REFERENCE_SAMPLES_PER_AXIS = 4
BASELINE_SAMPLES_PER_AXIS = 6


def parse_args():
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--method", choices=["megakernel", "wavefront"], default="megakernel")
    p.add_argument("--workload", choices=["large", "batched", "served"], default="large",
                   help="large: the 1.31M-triangle frame and all forms (default); batched: 64 seeded jobs of "
                        "uneven size alone; served: the Poisson request streams alone")
    p.add_argument("--rates", default="100,500", help="served: arrival rates (requests/s) to sweep")
    p.add_argument("--requests", type=int, default=1000, help="served: requests per rate")
    p.add_argument("--e2e-steps", type=int, default=5, help="steps of the end-to-end (host buffer) measurement")
    p.add_argument("--no-forms", action="store_true", help="the headline frame only")
    return p.parse_args()


def render_job(frame: Frame, method: int, accumulation: int = 0):
    import albedo_b200 as ab

    return ab.RenderJob(frame.width, frame.height, samples_per_axis=frame.samples_per_axis, seed=SEED,
                        max_depth=frame.max_depth, roulette_start=ROULETTE_START, method=method,
                        accumulation=accumulation)


def timed_frames(scene, job, accum, flush, steps: int) -> list[float]:
    """Per-step CUDA-event times (ms) of renders of `job`, L2 flushed before each."""
    import torch

    import albedo_b200 as ab

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
    return ms


# ------------------------------------------------------------------ peaks


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


def hbm_peak() -> tuple[float, str]:
    peak = measured_peaks().get("hbm_gbs")
    if peak:
        return float(peak), "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)"
    return 6650.0, "fallback 6650 GB/s"


def l2_read_peak(launches: int = 20) -> dict:
    """The L2 read bandwidth of this GPU, measured: a 32 MiB buffer (a quarter of
    L2) read 16 times per launch through L2 only (albedo_probe_read_sweep), best
    of `launches` CUDA-event-timed launches after warm-up, grid of 8 blocks of
    256 threads per SM."""
    import torch

    import albedo_b200 as ab

    nbytes = 32 << 20
    repeats = 16
    data = torch.randint(0, 2**31 - 1, (nbytes // 4,), dtype=torch.int32, device="cuda")
    sink = torch.zeros(4, dtype=torch.int32, device="cuda")
    blocks = 8 * torch.cuda.get_device_properties(0).multi_processor_count
    for _ in range(3):
        ab.read_sweep(data.data_ptr(), nbytes, repeats, blocks, sink.data_ptr())
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(launches):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        ab.read_sweep(data.data_ptr(), nbytes, repeats, blocks, sink.data_ptr())
        end.record()
        end.synchronize()
        best = min(best, start.elapsed_time(end) / 1e3)
    return {"gbs": nbytes * repeats / best / 1e9, "buffer_bytes": nbytes, "repeats": repeats, "blocks": blocks,
            "launches": launches, "method": "best of the launches, CUDA events, ld.global.cg 16-byte loads"}


def roofline(counts: dict, launch_s: float, l2: dict | None, kernel: str) -> dict:
    """The dominant kernel's algorithmic bytes per launch over its launch time,
    against the HBM copy peak (and, beside it, the measured L2 read peak)."""
    import albedo_b200 as ab

    alg_bytes = ab.algorithmic_bytes(counts)
    achieved = alg_bytes / launch_s / 1e9
    peak, source = hbm_peak()
    out = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
           "traffic": None, "kernel": kernel, "algorithmic_bytes_per_launch": alg_bytes, "work_per_launch": counts,
           "peak_source": source}
    if l2 is not None:
        out["l2"] = {"achieved": achieved, "peak": l2["gbs"], "frac": achieved / l2["gbs"],
                     "peak_source": "measured in this run (l2_read_peak)"}
    return out


def profiled_traffic(name: str, paths: int) -> tuple[float | None, str | None]:
    """DRAM bytes per launch of a frame of `paths` paths from a committed ncu
    summary (`dram_bytes_per_path: X` scaled by the paths one launch renders)."""
    path = ROOT / "profiles" / name
    if not path.exists():
        return None, None
    for line in path.read_text().splitlines():
        if line.startswith("dram_bytes_per_path:"):
            return float(line.split(":", 1)[1].split()[0]) * paths, path.name
    return None, None


# ------------------------------------------------------------------ the reference on the host


def reference_frame_sample(scene_path: Path, frame: Frame, samples_per_axis: int = REFERENCE_SAMPLES_PER_AXIS,
                           scene=None) -> dict:
    """The reference's own renderImage on the full frame of `frame` at
    samples_per_axis^2 samples per pixel, on all host threads."""
    from oracle import reference as ref

    scene = scene or ref.RefScene(scene_path)
    threads = ref.threads()
    start = time.perf_counter()
    scene.render_image(frame.width, frame.height, samples_per_axis, seed=SEED, max_depth=frame.max_depth,
                       roulette_start=ROULETTE_START, nthreads=threads)
    seconds = time.perf_counter() - start
    paths = frame.width * frame.height * samples_per_axis ** 2
    return {"value": paths / seconds / 1e6, "unit": "Mpaths/s", "cores": threads, "kind": "reference",
            "seconds": seconds,
            "sample": f"the full {frame.width}x{frame.height} frame at {samples_per_axis ** 2} spp ({paths} paths, "
                      f"{seconds:.1f} s) through the reference's renderImage (PixelBuffer, PathEstimator "
                      f"max_depth {frame.max_depth}) on {threads} threads"}


def run_reference(args, rank: int) -> None:
    """The reference arm: the reference renderer built from its own sources,
    rendering the headline frame through renderImage on the host's cores; each
    step is the full frame at 16 spp."""
    if rank != 0:
        return
    from albedo_b200 import scenes
    from oracle import reference as ref

    with tempfile.TemporaryDirectory() as tmp:
        scene_path = scenes.icosphere_scene(Path(tmp) / "large")
        scene = ref.RefScene(scene_path)
        for _ in range(args.warmup):
            reference_frame_sample(scene_path, LARGE, scene=scene)
        samples = [reference_frame_sample(scene_path, LARGE, scene=scene) for _ in range(args.steps)]
        total_paths = sum(LARGE.width * LARGE.height * REFERENCE_SAMPLES_PER_AXIS ** 2 for _ in samples)
        total_s = sum(s["seconds"] for s in samples)
        value = total_paths / total_s / 1e6
        base = samples[-1]
        cfg = config(LARGE, "reference CPU renderer (renderImage)", 1)
        # The same frame and scene; each timed step renders it at 16 spp (Mpaths/s
        # hardly depends on the sample count), which these fields state.
        cfg["timed_samples_per_axis"] = REFERENCE_SAMPLES_PER_AXIS
        cfg["timed_paths_per_step"] = LARGE.width * LARGE.height * REFERENCE_SAMPLES_PER_AXIS ** 2
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_s * 1e3 / len(samples),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded scene files in the reference's formats)",
                "config": cfg,
                "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": base["cores"], "kind": "reference",
                                 "sample": "each step: " + base["sample"]},
                "e2e": {"value": value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ forms


def precision_errors(scene_path: Path, frame: Frame, images: dict, pixel_count: int = 2048) -> dict:
    """Every image's error against the FP64 oracle (the reference renderer at
    65,536 spp, accumulated in FP64, on `pixel_count` seeded pixels, host cores)
    next to the reference renderer's own error at the frame's spp on the same
    pixels: relative RMSE and mean relative error over pixels whose oracle
    luminance exceeds 1e-3, and the paired statistic of each image's per-pixel
    squared errors against the reference's (mean difference over its standard
    error: |t| < 4 is matched RMSE)."""
    from oracle import reference as ref

    rng = np.random.default_rng(91)
    pixels = np.stack([rng.integers(0, frame.width, pixel_count), rng.integers(0, frame.height, pixel_count)],
                      axis=1).astype(np.int32)
    reference = ref.RefScene(scene_path)
    t0 = time.perf_counter()
    oracle_sum, _ = reference.render_pixels(frame.width, frame.height, 256, pixels, seed=1000003,
                                            max_depth=frame.max_depth)
    oracle_s = time.perf_counter() - t0
    oracle = oracle_sum / 65536.0
    spp = frame.samples_per_axis ** 2
    theirs_sum, _ = reference.render_pixels(frame.width, frame.height, frame.samples_per_axis, pixels, seed=SEED,
                                            max_depth=frame.max_depth)
    lum = oracle.mean(axis=1)
    keep = lum > 1e-3

    def squared(rgb):
        return np.sum(((rgb - oracle)[keep] / lum[keep, None]) ** 2, axis=1)

    def errors(rgb):
        err = (rgb - oracle)[keep] / lum[keep, None]
        return {"rel_rmse": float(np.sqrt(np.mean(err ** 2))), "mean_rel": float(np.mean(np.abs(err)))}

    theirs = theirs_sum / spp
    index = pixels[:, 1] * frame.width + pixels[:, 0]
    out = {}
    for label, img in images.items():
        ours = img[index, :3] / spp
        d = squared(ours) - squared(theirs)
        se = d.std(ddof=1) / np.sqrt(len(d))
        out[label] = {**errors(ours), "paired_t_vs_reference": float(d.mean() / se) if se > 0 else 0.0}
    out["reference_cpu_equal_spp"] = errors(theirs)
    out["oracle"] = {"pixels": pixel_count, "spp": 65536, "seconds": oracle_s, "pixels_lit": int(keep.sum())}
    return out


def large_forms(scene, scene_path: Path, frame: Frame, flush, fp64_image, steps: int = 1) -> dict:
    """The headline frame by the other forms (Kahan-compensated FP32 sums in the
    megakernel, the wavefront), and every image's error against the FP64
    oracle."""
    import torch

    import albedo_b200 as ab

    frames = {}
    images = {"megakernel_fp64": fp64_image}
    for label, method, accumulation in (("megakernel_kahan_fp32", ab.MEGAKERNEL, ab.ACCUMULATE_KAHAN_FP32),
                                        ("wavefront_fp64", ab.WAVEFRONT, ab.ACCUMULATE_FP64)):
        job = render_job(frame, method, accumulation)
        acc = torch.zeros((frame.width * frame.height, 4), dtype=torch.float64, device="cuda")
        if method == ab.WAVEFRONT:
            frames[label + "_autotune"] = ab.autotune_batch([(scene, job, acc.data_ptr())])
        acc.zero_()
        ms = timed_frames(scene, job, acc, flush, steps)
        if steps != 1:
            acc.zero_()
            ab.render_device(scene, job, acc.data_ptr())
            torch.cuda.synchronize()
            scene.check()
        frames[label] = {"mpaths_per_s": frame.paths / (statistics.mean(ms) / 1e3) / 1e6,
                         "ms_per_frame": statistics.mean(ms), "steps": steps}
        if method == ab.WAVEFRONT:
            frames[label]["mrays_per_s"] = ab.wavefront_last_rays() / (statistics.mean(ms) / 1e3) / 1e6
            frames[label]["iterations"] = ab.wavefront_last_iterations()
        images[label] = acc.cpu().numpy()
    fp64, kahan = images["megakernel_fp64"][:, :3], images["megakernel_kahan_fp32"][:, :3]
    lit = np.abs(fp64) > 1e-9
    frames["kahan_vs_fp64_max_rel"] = float(np.max(np.abs(kahan - fp64)[lit] / np.abs(fp64)[lit]))
    frames["error_vs_fp64_oracle"] = precision_errors(scene_path, frame, images)
    return frames


def soup_form(tmp: Path, flush) -> dict:
    """The 1M-triangle random soup at the large frame: megakernel and wavefront,
    each tuned on the frame, one step each, and their errors against the FP64
    oracle."""
    import torch

    import albedo_b200 as ab
    from albedo_b200 import scenes

    path = scenes.soup_scene(tmp / "soup")
    t0 = time.perf_counter()
    scene = ab.Scene.load(path)
    load_s = time.perf_counter() - t0
    images = {}
    out = {"workload": SOUP.workload, "load_s": load_s, "triangles": scene.info()["triangles"]}
    for label, method in (("megakernel_fp64", ab.MEGAKERNEL), ("wavefront_fp64", ab.WAVEFRONT)):
        job = render_job(SOUP, method)
        acc = torch.zeros((SOUP.width * SOUP.height, 4), dtype=torch.float64, device="cuda")
        if method == ab.MEGAKERNEL:
            # Tuned on the frame itself (the tuner renders it at a quarter of its samples).
            out["megakernel_autotune"] = ab.autotune_megakernel(scene, job)
        else:
            # Tuned on the frame itself, as the megakernel.
            out["wavefront_autotune"] = ab.autotune_batch([(scene, job, acc.data_ptr())])
        ms = timed_frames(scene, job, acc, flush, 1)
        out[label] = {"mpaths_per_s": SOUP.paths / (ms[0] / 1e3) / 1e6, "ms_per_frame": ms[0]}
        images[label] = acc.cpu().numpy()
    scene.check()
    out["error_vs_fp64_oracle"] = precision_errors(path, SOUP, images, pixel_count=512)
    scene.close()
    return out


def trefoil_form(tmp: Path, flush, l2: dict, steps: int = 3) -> dict:
    """The instanced trefoil frame, whose scene (a few MB) is L2-resident: the
    megakernel and the wavefront (each autotuned), CUDA events per step, L2
    flushed between steps, with the traversal's algorithmic bytes against the L2
    and HBM peaks."""
    import torch

    import albedo_b200 as ab
    from albedo_b200 import scenes

    scene = ab.Scene.load(scenes.trefoil_scene(tmp / "trefoil"))
    accum = torch.zeros((TREFOIL.width * TREFOIL.height, 4), dtype=torch.float64, device="cuda")
    out = {"workload": TREFOIL.workload, "paths_per_step": TREFOIL.paths}
    counts = None
    for label, method in (("megakernel", ab.MEGAKERNEL), ("wavefront", ab.WAVEFRONT)):
        job = render_job(TREFOIL, method)
        if method == ab.MEGAKERNEL:
            shape = ab.autotune_megakernel(scene, job)
            counts = ab.work_counts(scene, job)
        else:
            shape = ab.autotune_batch([(scene, job, accum.data_ptr())])
        ab.render_device(scene, job, accum.data_ptr())
        torch.cuda.synchronize()
        ms = timed_frames(scene, job, accum, flush, steps)
        launch_s = statistics.mean(ms) / 1e3
        out[label] = {"mpaths_per_s": TREFOIL.paths / launch_s / 1e6, "ms_per_step": launch_s * 1e3,
                      "steps": steps, "autotune": shape,
                      "roofline": roofline(counts, launch_s, l2, label)}
        if method == ab.WAVEFRONT:
            out[label]["mrays_per_s"] = ab.wavefront_last_rays() / launch_s / 1e6
            out[label]["iterations"] = ab.wavefront_last_iterations()
        else:
            out[label]["mrays_per_s"] = counts["rays"] / launch_s / 1e6
    out["wavefront_speedup_over_megakernel"] = out["megakernel"]["ms_per_step"] / out["wavefront"]["ms_per_step"]
    scene.close()
    return out


RESOLVE_WIDTH, RESOLVE_HEIGHT = 3840, 2160
RESOLVE_BYTES_PER_PIXEL = 32 + 3  # one accumulator read, three sRGB bytes written


def film_resolve_figures(flush, launches: int = 20) -> dict:
    """The film's device resolve (accumulators to sRGB bytes, bit-exact with the
    reference's writePpm bytes) on a 3840 x 2160 frame: 265 MB of accumulators,
    more than L2. Between launches a 256 MB read evicts them from L2 and leaves
    it clean (a flush by writing would leave up to 126 MB of dirty lines for the
    timed launch to write back). Each launch is timed with CUDA events.
    Algorithmic bytes: 32 read and 3 written per pixel. Two sample counts: 64
    (a power of two, so the average is one multiplication) and 36 (an FP64
    division per channel)."""
    import torch

    import albedo_b200 as ab

    pixels = RESOLVE_WIDTH * RESOLVE_HEIGHT
    out = torch.empty(3 * pixels, dtype=torch.uint8, device="cuda")
    peak, _ = hbm_peak()
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


def served_figures(rates: list[float], requests: int, l2: dict | None = None) -> list[dict]:
    """Poisson request streams (seeded) drawn from the batched-job distribution
    over 16 resident scenes, each request with its own seeded camera around its
    scene's, served under a 150 GB device budget: the continuous-batching server
    against the plain megakernel serving one request at a time in arrival order.
    Both use autotuned shapes (tuned before the streams start). Latency is
    completion minus arrival (wall clock); throughput is paths over the time from
    the first arrival to the last completion, where a request completes when its
    image is on the host as sRGB bytes (device resolve, then a copy of 3 bytes a
    pixel to pinned memory). The server's batch_mrays_per_s counts the rays its
    wavefront batch traced (not the express route's); its traversal GB/s is
    those rays times the pool's algorithmic bytes per ray (counted on each
    pool scene's own job), against the HBM and L2 peaks."""
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
    pool_bytes = pool_rays = 0
    for scene, j in zip(loaded, pool):
        pool_job = ab.RenderJob(j.width, j.height, samples_per_axis=j.samples_per_axis, max_depth=8)
        ab.autotune_megakernel(scene, pool_job)
        counts = ab.work_counts(scene, pool_job)
        pool_bytes += ab.algorithmic_bytes(counts)
        pool_rays += counts["rays"]
    bytes_per_ray = pool_bytes / max(pool_rays, 1)
    wave_shape = ab.autotune_batch([(scene, ab.RenderJob(j.width, j.height, samples_per_axis=j.samples_per_axis,
                                                         max_depth=8, method=ab.WAVEFRONT), a.data_ptr())
                                    for scene, j, a in zip(loaded, pool, warm)])
    tune_s = time.perf_counter() - tune_start
    del warm
    hbm, _ = hbm_peak()
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
        traversal_gbs = rays * bytes_per_ray / span_server / 1e9
        server_fig = {"mpaths_per_s": paths / span_server / 1e6, "batch_mrays_per_s": rays / span_server / 1e6,
                      "routed_batch": routes[0], "routed_express": routes[1],
                      "p50_ms": float(np.percentile(lat_server, 50) * 1e3),
                      "p99_ms": float(np.percentile(lat_server, 99) * 1e3),
                      "traversal_gbs": traversal_gbs, "traversal_frac_of_hbm": traversal_gbs / hbm}
        if l2 is not None:
            server_fig["traversal_frac_of_l2"] = traversal_gbs / l2["gbs"]
        results.append({
            "rate_per_s": rate, "requests": len(reqs), "paths": paths, "server": server_fig,
            "megakernel_one_at_a_time": {"mpaths_per_s": paths / span_mega / 1e6,
                                         "p50_ms": float(np.percentile(lat_mega, 50) * 1e3),
                                         "p99_ms": float(np.percentile(lat_mega, 99) * 1e3)},
            "speedup_over_megakernel": span_mega / span_server})
        del accs, srgb_dev, srgb_host
    for s in loaded:
        s.check()
    return [{"autotune": {"seconds": tune_s, "wavefront": wave_shape},
             "pool_algorithmic_bytes_per_ray": bytes_per_ray}] + results


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


def batched_figures(steps: int, warmup: int, count: int = 64, l2: dict | None = None) -> dict:
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
    iterations = ab.wavefront_last_iterations()
    # The tuned shape with each ray-binning setting (0 none, 1 the extension rays,
    # 2 the shadow rays too), one timed batch each.
    ray_sort_ms = {}
    for ray_sort in (0, 1, 2):
        ab.set_tuning(**{k: wave_shape[k] for k in ("blocks_per_sm", "trace_blocks_per_sm", "fetch_batch",
                                                     "iterations_per_graph", "slot_count", "trace_loop")},
                      ray_sort=ray_sort)
        ray_sort_ms[ray_sort] = statistics.mean(timed(batched)) if steps > 0 else None
    ab.set_tuning(**{k: wave_shape[k] for k in ("blocks_per_sm", "trace_blocks_per_sm", "fetch_batch",
                                                 "iterations_per_graph", "slot_count", "trace_loop", "ray_sort")})
    # The fixed cost of one iteration (its graph's launches, the queue kernels on
    # nearly empty queues, the host's completion polling): two 4 x 4-pixel jobs
    # whose iterations do almost no work, at 1 and at 8 x 8 samples per pixel (a
    # pixel's samples run one after another, so the second takes about 64 times
    # the iterations); the difference of their times over the difference of
    # their iteration counts leaves out the per-call costs. Times the batch's
    # iteration count, it bounds what one persistent launch for the whole batch
    # could save.
    tiny_acc = torch.zeros((16, 4), dtype=torch.float64, device="cuda")
    tiny_scene = loaded[jobs[0].scene]

    def tiny_run(n):
        tiny = [(tiny_scene, ab.RenderJob(4, 4, samples_per_axis=n, max_depth=8, method=ab.WAVEFRONT),
                 tiny_acc.data_ptr())]
        ab.render_batch(tiny)
        torch.cuda.synchronize()
        runs = []
        for _ in range(3):
            start = time.perf_counter()
            ab.render_batch(tiny)
            torch.cuda.synchronize()
            runs.append(((time.perf_counter() - start) * 1e3, ab.wavefront_last_iterations()))
        return min(runs)

    short_ms, short_iterations = tiny_run(1)
    long_ms, long_iterations = tiny_run(8)
    per_iteration_ms = (long_ms - short_ms) / max(long_iterations - short_iterations, 1)
    for s in loaded.values():
        s.check()
    batch_s = statistics.mean(batch_ms) / 1e3
    mega_s = statistics.mean(mega_ms) / 1e3
    peak, _ = hbm_peak()
    tiles = {}
    for shape in mega_shapes:
        key = (f"{shape['tile_width']}x{128 // shape['tile_width']}/{shape['blocks_per_sm']}"
               + {0: "", 1: "/inline", 2: "/inline-closest"}[shape["inline_traversal"]])
        tiles[key] = tiles.get(key, 0) + 1
    wave = {"mpaths_per_s": paths / batch_s / 1e6, "mrays_per_s": rays / batch_s / 1e6,
            "ms_per_step": batch_s * 1e3, "rays_per_step": rays,
            "traversal_gbs": alg_bytes / batch_s / 1e9, "traversal_frac_of_hbm": alg_bytes / batch_s / 1e9 / peak,
            "iterations": iterations, "empty_iteration_ms": per_iteration_ms,
            "fixed_cost_share": per_iteration_ms * iterations / (batch_s * 1e3),
            "ray_sort_ms": {str(k): v for k, v in ray_sort_ms.items()}}
    if l2 is not None:
        wave["traversal_frac_of_l2"] = alg_bytes / batch_s / 1e9 / l2["gbs"]
    return {
        "jobs": len(jobs), "paths_per_step": paths, "wavefront": wave,
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


def config(frame: Frame, method: str, n_gpus: int) -> dict:
    return {"workload": frame.workload, "resolution": [frame.width, frame.height],
            "samples_per_axis": frame.samples_per_axis, "spp": frame.samples_per_axis ** 2,
            "max_depth": frame.max_depth, "roulette_start": ROULETTE_START, "seed": SEED,
            "paths_per_step": frame.paths, "method": method,
            "parallelism": "replicas" if n_gpus > 1 else "single",
            "l2": "flushed between steps (256 MiB write); the scene's tables exceed L2"}


# ------------------------------------------------------------------ the headline frame


def main():
    args = parse_args()
    from albedo_b200.replicas import max_over_ranks, ranks_from_env, whole_job_throughput

    ranks = ranks_from_env()
    rank, world, local_rank = ranks.rank, ranks.world, ranks.local_rank
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "batched":
        if rank == 0:
            run_batched(args)
        return
    if args.workload == "served":
        if rank == 0:
            run_served(args)
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

    frame = LARGE
    method = ab.WAVEFRONT if args.method == "wavefront" else ab.MEGAKERNEL
    tmp = tempfile.TemporaryDirectory()
    scene_path = scenes.icosphere_scene(Path(tmp.name) / "large")
    load_start = time.perf_counter()
    scene = ab.Scene.load(scene_path)
    load_s = time.perf_counter() - load_start
    job = render_job(frame, method)
    accum = torch.zeros((frame.width * frame.height, 4), dtype=torch.float64, device="cuda")
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
    value = whole_job_throughput(frame.paths / 1e6, args.steps, world, total_s)

    # End to end through the host-buffer entry point, pinned accumulators.
    e2e_steps = max(1, min(args.e2e_steps, args.steps))
    host_accum = torch.zeros((frame.width * frame.height, 4), dtype=torch.float64).pin_memory()
    ab.render_image_ptr(scene, job, host_accum.data_ptr())
    e2e_ms = []
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as e2e_clocks:
        for i in range(e2e_steps):
            flush.fill_(i & 0xFF)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            ab.render_image_ptr(scene, job, host_accum.data_ptr())
            e.record()
            e.synchronize()
            e2e_ms.append(s.elapsed_time(e))
    barrier()
    e2e_value = whole_job_throughput(frame.paths / 1e6, e2e_steps, world,
                                     max_over_ranks(sum(e2e_ms), dist, "cuda") / 1e3)
    frame_bytes = frame.width * frame.height * 32

    if rank == 0:
        counts = ab.work_counts(scene, job)
        launch_s = statistics.mean(step_ms) / 1e3
        l2 = l2_read_peak()
        kernel = (f"megakernel<{scene.info()['stack_capacity']}, path>" if method == ab.MEGAKERNEL
                  else "wavefront (extend + shadow + shade iterations)")
        roof = roofline(counts, launch_s, l2, kernel)
        traffic, traffic_source = profiled_traffic("megakernel_icosphere8_1920x1080.txt", frame.paths)
        roof["traffic"] = traffic
        roof["traffic_source"] = traffic_source
        line = {
            "metric": METRIC, "value": value, "unit": "Mpaths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene files in the reference's formats)",
            "config": config(frame, args.method, world),
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99))},
            "steps_ms": step_ms,
            "mrays_per_s": world * counts["rays"] * args.steps / total_s / 1e6,
            "gpu_launches": args.steps,
            "scene": {"triangles": scene.info()["triangles"], "bvh_nodes": scene.info()["nodes"],
                      "device_bytes": scene.info()["device_bytes"], "load_s": load_s},
            "e2e": {"value": e2e_value, "unit": "Mpaths/s", "h2d_bytes_per_step": frame_bytes,
                    "d2h_bytes_per_step": frame_bytes, "steps": e2e_steps, "ms_per_step": statistics.mean(e2e_ms),
                    "steps_ms": e2e_ms, "clocks": e2e_clocks.summary()},
            "roofline": roof,
            "l2_read_peak": l2,
            "clocks": clocks.summary(),
            "autotune": tuned,
        }
        if world == 1:
            line["cpu_baseline"] = reference_frame_sample(scene_path, frame, BASELINE_SAMPLES_PER_AXIS)
            if not args.no_forms and method == ab.MEGAKERNEL:
                accum.zero_()
                ab.render_device(scene, job, accum.data_ptr())
                torch.cuda.synchronize()
                fp64_image = accum.cpu().numpy()
                line["precision"] = large_forms(scene, scene_path, frame, flush, fp64_image)
                forms_tmp = Path(tmp.name)
                line["forms"] = {"soup": soup_form(forms_tmp, flush),
                                 "instanced_trefoil": trefoil_form(forms_tmp, flush, l2),
                                 "batched_64_jobs": batched_figures(1, 1, l2=l2),
                                 "film_resolve": film_resolve_figures(flush)}
                served = served_figures([float(r) for r in args.rates.split(",")], args.requests, l2)
                line["forms"]["served"] = {"autotune": served[0], "sweep": served[1:]}
        print(json.dumps(line), flush=True)
    scene.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
