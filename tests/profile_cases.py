"""Fixed render cases for profiling under ncu: one render, nothing else.

    python tests/profile_cases.py megakernel --width 480 --height 270 --spp 64 [--autotune]
                                   [--accumulation fp64|kahan] [--mega-shape TILE,BLOCKS,INLINE]
    python tests/profile_cases.py wavefront --width 480 --height 270 --spp 16 [--autotune]
    python tests/profile_cases.py resolve --width 3840 --height 2160

Both use the instanced trefoil scene (albedo_b200.scenes.trefoil_scene) unless
--scene icosphere6 or icosphere8 (displaced icospheres of 6 and 8 levels, 81,920 and
1,310,720 triangles), max depth 10 (16 for icosphere8, as the bench frame), seed 0. --trace-loop pins the wavefront traversal's turn shape (0:
nodes then leaf, 1: one step, 2: whole query out of line), --ray-sort its ray binning. With --autotune the launch shape is tuned first (as bench.py
does); a warm-up render precedes the profiled one unless --no-warmup. The case
prints how many launches of the render kernels come before the profiled render,
for ncu's `-s` (pass `-k regex:<kernel>` to pick the kernel). `resolve` resolves
seeded accumulators (64 samples a pixel) of the given size to sRGB bytes: one
warm-up launch, then the profiled one.
"""

from __future__ import annotations

import argparse
import math
import sys
import tempfile
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))

# Megakernel launches one tuning pass makes: every shape (3 tile widths x 5
# kernel variants) once untimed and twice timed.
MEGAKERNEL_TUNING_LAUNCHES = 15 * 3


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("method", choices=["megakernel", "wavefront", "resolve"])
    parser.add_argument("--width", type=int, default=480)
    parser.add_argument("--height", type=int, default=270)
    parser.add_argument("--spp", type=int, default=16)
    parser.add_argument("--no-warmup", action="store_true")
    parser.add_argument("--autotune", action="store_true")
    parser.add_argument("--scene", choices=["trefoil", "icosphere6", "icosphere8"], default="trefoil")
    parser.add_argument("--depth", type=int, default=None, help="max depth (default 10; 16 for icosphere8)")
    parser.add_argument("--trace-loop", type=int, choices=[0, 1, 2], default=None)
    parser.add_argument("--ray-sort", type=int, choices=[0, 1, 2], default=None,
                        help="wavefront: pin ray binning (0 none, 1 extension rays, 2 shadow rays too)")
    parser.add_argument("--mega-shape", default=None,
                        help="megakernel: pin TILE,BLOCKS,INLINE (tile width, blocks per SM, traversal placement)")
    parser.add_argument("--accumulation", choices=["fp64", "kahan"], default="fp64",
                        help="megakernel per-pixel sums: FP64 or Kahan-compensated FP32")
    args = parser.parse_args()

    import torch

    import albedo_b200 as ab
    from albedo_b200 import scenes

    if args.method == "resolve":
        resolve_case(args.width, args.height, warmups=0 if args.no_warmup else 1)
        return
    n = int(round(math.sqrt(args.spp)))
    with tempfile.TemporaryDirectory() as tmp:
        if args.scene.startswith("icosphere"):
            scene = ab.Scene.load(scenes.icosphere_scene(Path(tmp), levels=int(args.scene[-1])))
        else:
            scene = ab.Scene.load(scenes.trefoil_scene(Path(tmp)))
        if args.trace_loop is not None or args.ray_sort is not None:
            shape = ab.tuning()
            ab.set_tuning(blocks_per_sm=shape["blocks_per_sm"], trace_blocks_per_sm=5,
                          fetch_batch=shape["fetch_batch"], iterations_per_graph=shape["iterations_per_graph"],
                          slot_count=shape["slot_count"],
                          trace_loop=args.trace_loop if args.trace_loop is not None else shape["trace_loop"],
                          ray_sort=args.ray_sort if args.ray_sort is not None else shape["ray_sort"])
        method = ab.WAVEFRONT if args.method == "wavefront" else ab.MEGAKERNEL
        accumulation = ab.ACCUMULATE_KAHAN_FP32 if args.accumulation == "kahan" else ab.ACCUMULATE_FP64
        depth = args.depth if args.depth is not None else (16 if args.scene == "icosphere8" else 10)
        job = ab.RenderJob(args.width, args.height, samples_per_axis=n, max_depth=depth, method=method,
                           accumulation=accumulation)
        acc = torch.zeros((args.width * args.height, 4), dtype=torch.float64, device="cuda")
        before = 0
        shape = None
        if args.mega_shape is not None and method == ab.MEGAKERNEL:
            tile, blocks, inline = (int(v) for v in args.mega_shape.split(","))
            ab.set_tuning(scene, tile_width=tile, blocks_per_sm=blocks, inline_traversal=inline)
        if args.autotune:
            if method == ab.MEGAKERNEL:
                shape = ab.autotune_megakernel(scene, job)
                before += MEGAKERNEL_TUNING_LAUNCHES
            else:
                shape = ab.autotune_batch([(scene, job, acc.data_ptr())])
        warmups = 0 if args.no_warmup else 1
        for _ in range(warmups + 1):
            ab.render_device(scene, job, acc.data_ptr())
        torch.cuda.synchronize()
        scene.check()
        if method == ab.MEGAKERNEL:
            before += warmups
            counts = ab.work_counts(scene, job)
            print(f"rendered {args.width}x{args.height} at {n * n} spp (megakernel); megakernel launches before the "
                  f"profiled render: {before}; shape {ab.tuning(scene)}; work {counts}")
        else:
            print(f"rendered {args.width}x{args.height} at {n * n} spp (wavefront, {ab.wavefront_last_iterations()} "
                  f"iterations, {ab.wavefront_last_rays()} rays per render); tuned shape {shape or ab.tuning()}")
        scene.close()


def resolve_case(width: int, height: int, warmups: int) -> None:
    import torch

    import albedo_b200 as ab

    generator = torch.Generator(device="cuda").manual_seed(5)
    acc = torch.rand((width * height, 4), dtype=torch.float64, device="cuda", generator=generator) * 64.0
    acc.view(torch.int64)[:, 3] = 64
    out = torch.empty(3 * width * height, dtype=torch.uint8, device="cuda")
    for _ in range(warmups + 1):
        ab.resolve_srgb(acc.data_ptr(), width, height, out.data_ptr())
    torch.cuda.synchronize()
    print(f"resolved {width}x{height} accumulators to sRGB; resolve launches before the profiled one: {warmups}")


if __name__ == "__main__":
    main()
