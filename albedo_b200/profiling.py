"""Fixed render cases for profiling under ncu: one render, nothing else.

    python -m albedo_b200.profiling megakernel --width 480 --height 270 --spp 64
    python -m albedo_b200.profiling wavefront --width 480 --height 270 --spp 16

Both use the instanced trefoil scene (albedo_b200.scenes.trefoil_scene), max
depth 10, seed 0. A warm-up render precedes the profiled one unless --no-warmup;
pass `-k regex:<kernel> -s <skip>` to ncu to pick the launch.
"""

from __future__ import annotations

import argparse
import math
import tempfile
from pathlib import Path


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("method", choices=["megakernel", "wavefront"])
    parser.add_argument("--width", type=int, default=480)
    parser.add_argument("--height", type=int, default=270)
    parser.add_argument("--spp", type=int, default=16)
    parser.add_argument("--no-warmup", action="store_true")
    args = parser.parse_args()

    import torch

    import albedo_b200 as ab
    from albedo_b200 import scenes

    n = int(round(math.sqrt(args.spp)))
    with tempfile.TemporaryDirectory() as tmp:
        scene = ab.Scene.load(scenes.trefoil_scene(Path(tmp)))
        method = ab.WAVEFRONT if args.method == "wavefront" else ab.MEGAKERNEL
        job = ab.RenderJob(args.width, args.height, samples_per_axis=n, max_depth=10, method=method)
        acc = torch.zeros((args.width * args.height, 4), dtype=torch.float64, device="cuda")
        for _ in range(1 if args.no_warmup else 2):
            ab.render_device(scene, job, acc.data_ptr())
        torch.cuda.synchronize()
        scene.check()
        counts = ab.work_counts(scene, job) if method == ab.MEGAKERNEL else None
        print(f"rendered {args.width}x{args.height} at {n * n} spp ({args.method})", counts or "")
        scene.close()


if __name__ == "__main__":
    main()
