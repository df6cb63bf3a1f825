"""Writes tests/golden/reference_vectors.npz: outputs of the reference renderer,
built from its own sources (oracle/Makefile), on seeded inputs.

    python tests/golden/make_golden.py

The fixtures pin the oracle build (tests/test_golden.py regenerates them and
expects the same values) and let device tests check the path against the
reference where the reference library is not built (tests/test_gpu_golden.py).
Contents:
  pcg32               PCG32(seed 42, stream 54), 32 outputs (sampling/pcg32.hpp)
  pixel_stream        the per-pixel stream of pixel (3, 5) of a 320-wide image,
                      seed 0: 64 doubles (render/render_image.cpp:27-44)
  srgb_values/bytes   toByte(encodeSrgb(x)) (color/srgb.cpp:18-36) on 4,096
                      seeded values and on 0, -0, 1, NaN and the infinities
  room_scene_text     the room scene file (albedo_b200.scenes.room_scene)
  room_rays / _hit / _object / _t
                      Scene::intersect on 512 seeded rays in the room
  room_image          renderImage averages, 32 x 18, 2 x 2 spp, depth 8, seed 0
  room_ppm            writePpm of room_image
"""

import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from albedo_b200 import scenes  # noqa: E402
from oracle import reference as ref  # noqa: E402

IMAGE = dict(width=32, height=18, n=2, max_depth=8, seed=0)


def room_rays(count: int = 512, seed: int = 17) -> np.ndarray:
    rng = np.random.default_rng(seed)
    origin = rng.uniform([-2.8, 0.05, -3.5], [2.8, 4.5, 3.0], size=(count, 3))
    direction = rng.normal(size=(count, 3))
    direction /= np.linalg.norm(direction, axis=1, keepdims=True)
    return np.concatenate([origin, direction], axis=1).astype(np.float32).astype(np.float64)


def srgb_values(seed: int = 3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.uniform(-0.1, 1.2, 2048), np.exp(rng.uniform(np.log(1e-6), np.log(2.0), 2048)),
                           [0.0, -0.0, 1.0, np.nan, np.inf, -np.inf]])


def generate() -> dict:
    with tempfile.TemporaryDirectory() as tmp:
        path = scenes.room_scene(Path(tmp))
        scene = ref.RefScene(path)
        rays = room_rays()
        hits = scene.intersect(rays)
        image = scene.render_image(IMAGE["width"], IMAGE["height"], IMAGE["n"], seed=IMAGE["seed"],
                                   max_depth=IMAGE["max_depth"])
        ppm = Path(tmp) / "room.ppm"
        ref.write_ppm(ppm, image)
        text = path.read_text()
        ppm_bytes = np.frombuffer(ppm.read_bytes(), dtype=np.uint8).copy()
    values = srgb_values()
    return {
        "pcg32": ref.pcg32(42, 54, 32),
        "pixel_stream": ref.pixel_stream(0, 3, 5, 320, 64),
        "srgb_values": values,
        "srgb_bytes": ref.srgb_bytes(values),
        "room_scene_text": np.array(text),
        "room_rays": rays,
        "room_hit": hits["hit"],
        "room_object": hits["object"],
        "room_t": hits["t"],
        "room_image": image,
        "room_ppm": ppm_bytes,
    }


if __name__ == "__main__":
    if not ref.available():
        sys.exit("build the reference first: make -C oracle ref")
    np.savez_compressed(HERE / "reference_vectors.npz", **generate())
    print("wrote", HERE / "reference_vectors.npz")
