"""Seeded synthetic scenes for the benchmark configurations, written in the
reference's own scene-file and OBJ formats so the same files drive both the
reference renderer and this one.

Every number written is a float32 value printed exactly (17 significant digits),
so the FP64 reference and the FP32 device see the same geometry.

    room_scene        analytic-sphere room: 4 walls of radius 1e4, five r=0.8 spheres
                      (smooth glass, rough glass alpha 0.2, silver mirror, gold
                      roughness 0.25, blue diffuse), area + point light + sky
    trefoil_scene     a trefoil-knot tube (256 segments x 32 ring vertices, 16384
                      triangles, smooth) instanced 3x (uniform scale 0.8-1.2, seeded
                      y-rotation) in gold, glass and copper on a 2-triangle checker floor
    icosphere_scene   an 8-level icosphere (1,310,720 triangles) displaced by 3 octaves
                      of Perlin noise (amplitude 0.05), rough dielectric alpha 0.1
    soup_scene        1,000,000 random triangles in the unit cube, edges log-uniform
                      in [1e-4, 1e-2]
    batch_jobs        64 seeded render jobs of uneven size (displaced icospheres of
                      1k-500k triangles, 0-8 spheres, mixed materials)
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np


def f32(x: float) -> float:
    return float(np.float32(x))


def num(x: float) -> str:
    return repr(f32(x))


def vec(*xs) -> str:
    return " ".join(num(x) for x in xs)


class Pcg32:
    """PCG32 (XSH-RR), as the renderer seeds per-pixel streams; used here to draw
    scene parameters reproducibly."""

    MASK = (1 << 64) - 1

    def __init__(self, seed: int, stream: int = 54):
        self.state = 0
        self.inc = ((stream << 1) | 1) & self.MASK
        self.next_u32()
        self.state = (self.state + seed) & self.MASK
        self.next_u32()

    def next_u32(self) -> int:
        old = self.state
        self.state = (old * 6364136223846793005 + self.inc) & self.MASK
        xorshifted = (((old >> 18) ^ old) >> 27) & 0xFFFFFFFF
        rot = old >> 59
        return ((xorshifted >> rot) | (xorshifted << ((32 - rot) & 31))) & 0xFFFFFFFF

    def uniform(self, low: float = 0.0, high: float = 1.0) -> float:
        return low + (high - low) * self.next_u32() / 4294967296.0


MATERIALS = """\
material gold    conductor eta 0.156 0.424 1.383  k 3.602 2.472 1.915  roughness 0.25
material silver  conductor eta 0.155 0.117 0.138  k 4.83 3.12 2.15  roughness 0
material copper  conductor eta 0.238 1.007 1.240  k 3.626 2.582 2.393  roughness 0.3
material glass   dielectric ior 1.5  roughness 0
material rough_glass dielectric ior 1.5  roughness 0.44721359549995793
material white   diffuse color 0.73 0.73 0.73
material red     diffuse color 0.63 0.07 0.05
material green   diffuse color 0.12 0.45 0.15
material blue    diffuse color 0.15 0.3 0.7
material tiles   checker even 0.73 0.73 0.73  odd 0.3 0.3 0.3  frequency 1.25
"""

LIGHTS = """\
area_light 0 5.5999999046325684 -1.2000000476837158  radius 1.1000000238418579  radiance 9 7.5999999046325684 5.8000001907348633
point_light 0.80000001192092896 4.1999998092651367 3.2000000476837158  intensity 1.2000000476837158 2 3.5999999046325684
sky 0.05000000074505806 0.059999998658895493 0.079999998211860657
"""

CAMERA = "camera from 0 2.4000000953674316 7.8000001907348633  at 0 1.8999999761581421 -0.5  up 0 1 0  fov 38\n"


def room_scene(directory: Path) -> Path:
    """The plain-method room: 320x180 at 16 spp, max depth 8 in its configuration."""
    directory.mkdir(parents=True, exist_ok=True)
    lines = ["# Analytic-sphere room (seedless; all values float32-exact).", CAMERA, MATERIALS,
             f"sphere {vec(0, -10000, 0)}  radius 10000  material white",
             f"sphere {vec(0, 0, -10004)}  radius 10000  material white",
             f"sphere {vec(-10003, 0, 0)}  radius 10000  material red",
             f"sphere {vec(10003, 0, 0)}  radius 10000  material green"]
    r = 0.8
    for (x, z), material in zip([(-2.2, -1.2), (-1.1, 0.6), (0.0, -1.6), (1.1, 0.6), (2.2, -1.2)],
                                ["glass", "rough_glass", "silver", "gold", "blue"]):
        lines.append(f"sphere {vec(x, r, z)}  radius {num(r)}  material {material}")
    lines.append(LIGHTS)
    path = directory / "room.scene"
    path.write_text("\n".join(lines) + "\n")
    return path


def trefoil_mesh(segments: int = 256, sides: int = 32, tube_radius: float = 0.45):
    """Tube around the trefoil (sin t + 2 sin 2t, cos t - 2 cos 2t, -sin 3t) along its
    Frenet frame; quads wound counter-clockwise seen from outside, split in two."""
    t = 2 * np.pi * np.arange(segments) / segments
    c = np.stack([np.sin(t) + 2 * np.sin(2 * t), np.cos(t) - 2 * np.cos(2 * t), -np.sin(3 * t)], axis=1)
    d1 = np.stack([np.cos(t) + 4 * np.cos(2 * t), -np.sin(t) + 4 * np.sin(2 * t), -3 * np.cos(3 * t)], axis=1)
    d2 = np.stack([-np.sin(t) - 8 * np.sin(2 * t), -np.cos(t) + 8 * np.cos(2 * t), 9 * np.sin(3 * t)], axis=1)
    tangent = d1 / np.linalg.norm(d1, axis=1, keepdims=True)
    binormal = np.cross(d1, d2)
    binormal /= np.linalg.norm(binormal, axis=1, keepdims=True)
    normal = np.cross(binormal, tangent)
    a = 2 * np.pi * np.arange(sides) / sides
    ring = (np.cos(a)[None, :, None] * normal[:, None, :] + np.sin(a)[None, :, None] * binormal[:, None, :])
    points = (c[:, None, :] + tube_radius * ring).reshape(-1, 3).astype(np.float32)
    seg = np.arange(segments)[:, None]
    side = np.arange(sides)[None, :]

    def index(s, k):
        return (s % segments) * sides + (k % sides)

    q0, q1, q2, q3 = index(seg, side), index(seg, side + 1), index(seg + 1, side + 1), index(seg + 1, side)
    quads = np.stack([q0, q1, q2, q3], axis=-1).reshape(-1, 4)
    return points, quads


def write_obj(path: Path, points: np.ndarray, faces: np.ndarray, uvs: np.ndarray | None = None) -> None:
    lines = [f"v {repr(float(x))} {repr(float(y))} {repr(float(z))}" for x, y, z in points.astype(np.float32)]
    if uvs is not None:
        lines += [f"vt {repr(float(u))} {repr(float(v))}" for u, v in uvs.astype(np.float32)]
        lines += ["f " + " ".join(f"{i + 1}/{i + 1}" for i in face) for face in faces]
    else:
        lines += ["f " + " ".join(str(i + 1) for i in face) for face in faces]
    path.write_text("\n".join(lines) + "\n")


def write_floor(path: Path) -> None:
    points = np.array([[-3.5, 0, 12], [3.5, 0, 12], [3.5, 0, -4.5], [-3.5, 0, -4.5]], np.float32)
    write_obj(path, points, np.array([[0, 1, 2, 3]]), uvs=points[:, [0, 2]])


def trefoil_scene(directory: Path, seed: int = 7) -> Path:
    """The instanced-mesh configuration: 960x540 at 64 spp, max depth 10."""
    directory.mkdir(parents=True, exist_ok=True)
    points, quads = trefoil_mesh()
    write_obj(directory / "trefoil.obj", points, quads)
    write_floor(directory / "floor.obj")
    rng = Pcg32(seed)
    lines = ["# Trefoil tube instanced three times on a checker floor.", CAMERA, MATERIALS,
             "mesh floor floor.obj", "mesh knot trefoil.obj smooth", "instance floor material tiles",
             f"sphere {vec(0, 10005, 0)}  radius 10000  material white",
             f"sphere {vec(0, 0, -10004)}  radius 10000  material white",
             f"sphere {vec(-10003, 0, 0)}  radius 10000  material red",
             f"sphere {vec(10003, 0, 0)}  radius 10000  material green"]
    for material, (x, z) in zip(["gold", "glass", "copper"], [(-1.7, -1.4), (0.0, 0.4), (1.7, -1.4)]):
        s = f32(rng.uniform(0.8, 1.2))
        angle = f32(rng.uniform(0.0, 360.0))
        lines.append(f"instance knot material {material}  fit 1.6000000238418579  scale {num(s)}  "
                     f"rotate 0 1 0 {num(angle)}  ground  translate {vec(x, 0, z)}")
    lines.append(LIGHTS)
    path = directory / "trefoil.scene"
    path.write_text("\n".join(lines) + "\n")
    return path


# ---------------------------------------------------------------- Perlin noise (for displacement)

_PERM = np.array([
    151, 160, 137, 91, 90, 15, 131, 13, 201, 95, 96, 53, 194, 233, 7, 225, 140, 36, 103, 30, 69, 142, 8, 99, 37,
    240, 21, 10, 23, 190, 6, 148, 247, 120, 234, 75, 0, 26, 197, 62, 94, 252, 219, 203, 117, 35, 11, 32, 57, 177,
    33, 88, 237, 149, 56, 87, 174, 20, 125, 136, 171, 168, 68, 175, 74, 165, 71, 134, 139, 48, 27, 166, 77, 146,
    158, 231, 83, 111, 229, 122, 60, 211, 133, 230, 220, 105, 92, 41, 55, 46, 245, 40, 244, 102, 143, 54, 65, 25,
    63, 161, 1, 216, 80, 73, 209, 76, 132, 187, 208, 89, 18, 169, 200, 196, 135, 130, 116, 188, 159, 86, 164, 100,
    109, 198, 173, 186, 3, 64, 52, 217, 226, 250, 124, 123, 5, 202, 38, 147, 118, 126, 255, 82, 85, 212, 207, 206,
    59, 227, 47, 16, 58, 17, 182, 189, 28, 42, 223, 183, 170, 213, 119, 248, 152, 2, 44, 154, 163, 70, 221, 153,
    101, 155, 167, 43, 172, 9, 129, 22, 39, 253, 19, 98, 108, 110, 79, 113, 224, 232, 178, 185, 112, 104, 218, 246,
    97, 228, 251, 34, 242, 193, 238, 210, 144, 12, 191, 179, 162, 241, 81, 51, 145, 235, 249, 14, 239, 107, 49, 192,
    214, 31, 181, 199, 106, 157, 184, 84, 204, 176, 115, 121, 50, 45, 127, 4, 150, 254, 138, 236, 205, 93, 222, 114,
    67, 29, 24, 72, 243, 141, 128, 195, 78, 66, 215, 61, 156, 180], dtype=np.int64)


def perlin_noise(p: np.ndarray) -> np.ndarray:
    """Perlin's improved noise (2002) at (N, 3) points, vectorized in FP64."""
    f = np.floor(p)
    cell = np.mod(f, 256.0).astype(np.int64)
    x, y, z = (p - f).T
    xi, yi, zi = cell.T

    def fade(t):
        return t * t * t * (t * (t * 6 - 15) + 10)

    def grad(h, gx, gy, gz):
        h = h & 15
        u = np.where(h < 8, gx, gy)
        v = np.where(h < 4, gy, np.where((h == 12) | (h == 14), gx, gz))
        return np.where((h & 1) == 0, u, -u) + np.where((h & 2) == 0, v, -v)

    def hashed(i):
        return _PERM[i % 256]

    u, v, w = fade(x), fade(y), fade(z)
    a = hashed(xi) + yi
    aa = hashed(a) + zi
    ab = hashed(a + 1) + zi
    b = hashed(xi + 1) + yi
    ba = hashed(b) + zi
    bb = hashed(b + 1) + zi

    def lerp(t, lo, hi):
        return lo + t * (hi - lo)

    return lerp(w,
                lerp(v, lerp(u, grad(hashed(aa), x, y, z), grad(hashed(ba), x - 1, y, z)),
                     lerp(u, grad(hashed(ab), x, y - 1, z), grad(hashed(bb), x - 1, y - 1, z))),
                lerp(v, lerp(u, grad(hashed(aa + 1), x, y, z - 1), grad(hashed(ba + 1), x - 1, y, z - 1)),
                     lerp(u, grad(hashed(ab + 1), x, y - 1, z - 1), grad(hashed(bb + 1), x - 1, y - 1, z - 1))))


def icosphere(levels: int):
    """Unit icosphere: 20 * 4^levels triangles, counter-clockwise seen from outside."""
    t = (1 + 5 ** 0.5) / 2
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                      [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                      [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    points = np.array(verts, dtype=np.float64)
    points /= np.linalg.norm(points, axis=1, keepdims=True)
    for _ in range(levels):
        edges = np.concatenate([faces[:, [0, 1]], faces[:, [1, 2]], faces[:, [2, 0]]])
        key = np.sort(edges, axis=1)
        uniq, inverse = np.unique(key, axis=0, return_inverse=True)
        mid = points[uniq[:, 0]] + points[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(points)
        points = np.concatenate([points, mid])
        m = inverse.reshape(3, -1).T + base
        a, b, c = faces[:, 0], faces[:, 1], faces[:, 2]
        ab, bc, ca = m[:, 0], m[:, 1], m[:, 2]
        faces = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                                np.stack([ab, bc, ca], 1)])
    return points, faces


def displaced_icosphere(levels: int, seed: int, amplitude: float = 0.05):
    points, faces = icosphere(levels)
    rng = np.random.default_rng(seed)
    offset = rng.uniform(0, 256, size=3)
    height = sum((0.5 ** k) * perlin_noise((2.0 ** k) * (points * 2.0) + offset) for k in range(3))
    points = points * (1.0 + amplitude * height)[:, None]
    return points.astype(np.float32), faces


def icosphere_scene(directory: Path, levels: int = 8, seed: int = 11) -> Path:
    directory.mkdir(parents=True, exist_ok=True)
    points, faces = displaced_icosphere(levels, seed)
    write_obj(directory / "icosphere.obj", points, faces)
    write_floor(directory / "floor.obj")
    lines = ["# Displaced icosphere in rough glass.", CAMERA, MATERIALS,
             "material frosted dielectric ior 1.5 roughness 0.31622776601683794",
             "mesh floor floor.obj", "mesh ball icosphere.obj smooth", "instance floor material tiles",
             "instance ball material frosted  fit 2.5999999046325684  ground  translate 0 0 -0.5", LIGHTS]
    path = directory / "icosphere.scene"
    path.write_text("\n".join(lines) + "\n")
    return path


def soup_scene(directory: Path, count: int = 1_000_000, seed: int = 13) -> Path:
    directory.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(seed)
    centers = rng.uniform(0, 1, size=(count, 3))
    dirs = rng.normal(size=(count, 2, 3))
    dirs /= np.linalg.norm(dirs, axis=2, keepdims=True)
    lengths = np.exp(rng.uniform(np.log(1e-4), np.log(1e-2), size=(count, 2)))
    e1 = dirs[:, 0] * lengths[:, :1]
    e2 = dirs[:, 1] * lengths[:, 1:]
    v0 = centers - (e1 + e2) / 3
    pts = np.stack([v0, v0 + e1, v0 + e2], axis=1).reshape(-1, 3).astype(np.float32)
    faces = np.arange(3 * count).reshape(-1, 3)
    write_obj(directory / "soup.obj", pts, faces)
    write_floor(directory / "floor.obj")
    lines = ["# Random triangle soup in the unit cube.", CAMERA, MATERIALS,
             "mesh floor floor.obj", "mesh soup soup.obj", "instance floor material tiles",
             "instance soup material gold  fit 3  ground  translate 0 0 -0.5", LIGHTS]
    path = directory / "soup.scene"
    path.write_text("\n".join(lines) + "\n")
    return path


@dataclass
class BatchJob:
    scene: Path
    width: int
    height: int
    samples_per_axis: int
    seed: int


RESOLUTIONS = [(128, 72), (320, 180), (640, 360), (1024, 576)]


def batch_jobs(directory: Path, count: int = 64, seed: int = 17, scenes: int | None = None) -> list[BatchJob]:
    """Seeded jobs of uneven size: displaced icospheres whose triangle count is
    log-uniform in [1k, 500k] (subdivision level matching it), 0-8 analytic spheres,
    materials uniform over diffuse / conductor / dielectric / mix, resolutions from
    RESOLUTIONS and spp log-uniform in [4, 64] rounded to n^2 with n in 2..8."""
    directory.mkdir(parents=True, exist_ok=True)
    rng = Pcg32(seed)
    material_lines = MATERIALS + (
        "material marble_a diffuse color 0.8 0.78 0.75\n"
        "material mixed mix first gold second marble_a scale 2 veins 6 threshold 0.5\n")
    kinds = ["white", "gold", "frosted_glass", "mixed"]
    jobs: list[BatchJob] = []
    scene_count = scenes if scenes is not None else count
    scene_paths: list[Path] = []
    level_cache: dict[int, Path] = {}
    for s in range(scene_count):
        tris = math.exp(rng.uniform(math.log(1e3), math.log(5e5)))
        level = int(np.clip(round(math.log(tris / 20.0, 4)), 2, 7))
        if level not in level_cache:
            pts, faces = displaced_icosphere(level, seed + level)
            obj = directory / f"ico{level}.obj"
            write_obj(obj, pts, faces)
            level_cache[level] = obj
        write_floor(directory / "floor.obj")
        spheres = int(rng.uniform(0, 9))
        material = kinds[int(rng.uniform(0, 4))]
        lines = [f"# Batch scene {s}", CAMERA, material_lines,
                 "material frosted_glass dielectric ior 1.5 roughness 0.3",
                 "mesh floor floor.obj", f"mesh ball {level_cache[level].name} smooth",
                 "instance floor material tiles",
                 f"instance ball material {material}  fit 2  ground  translate 0 0 -0.8"]
        for k in range(spheres):
            r = f32(rng.uniform(0.2, 0.5))
            x = f32(rng.uniform(-2.5, 2.5))
            z = f32(rng.uniform(-2.5, 1.5))
            m = kinds[int(rng.uniform(0, 4))]
            lines.append(f"sphere {vec(x, r, z)} radius {num(r)} material {m}")
        lines.append(LIGHTS)
        path = directory / f"batch{s:02d}.scene"
        path.write_text("\n".join(lines) + "\n")
        scene_paths.append(path)
    for j in range(count):
        w, h = RESOLUTIONS[int(rng.uniform(0, 4))]
        spp = math.exp(rng.uniform(math.log(4), math.log(64)))
        n = int(np.clip(round(math.sqrt(spp)), 2, 8))
        jobs.append(BatchJob(scene_paths[j % scene_count], w, h, n, j))
    return jobs


def scene_camera(path: Path) -> tuple:
    """(look_from, look_at, up, fov) of a scene file's `camera from .. at .. up .. fov ..` line."""
    words = next(line for line in Path(path).read_text().splitlines() if line.startswith("camera")).split()
    values: dict[str, list[float]] = {}
    key = None
    for w in words[1:]:
        if w in ("from", "at", "up", "fov"):
            key = w
            values[key] = []
        else:
            values[key].append(float(w))
    return (tuple(values["from"]), tuple(values["at"]), tuple(values.get("up", (0.0, 1.0, 0.0))),
            values.get("fov", [60.0])[0])


def request_view(base: tuple, rng: np.random.Generator) -> tuple:
    """A seeded per-request camera around a scene's own: the eye moves up to 1.5
    units sideways, 0.5 down / 1 up and 1 forward or back; the target up to 0.5
    sideways and 0.3 vertically; up and field of view stay."""
    eye, target, up, fov = base
    eye = (eye[0] + rng.uniform(-1.5, 1.5), eye[1] + rng.uniform(-0.5, 1.0), eye[2] + rng.uniform(-1.0, 1.0))
    target = (target[0] + rng.uniform(-0.5, 0.5), target[1] + rng.uniform(-0.3, 0.3),
              target[2] + rng.uniform(-0.5, 0.5))
    return eye, target, up, fov


def flattened_parts(seed: int = 29) -> list[tuple]:
    """A scene of meshes added flattened, every triangle its own object
    (Scene::add(const TriangleMesh&, ...), scene/scene.cpp:33-61), between
    spheres, in this add order: a trefoil tube placed by a seeded rotation and
    scale, a sphere, a displaced level-5 icosphere (20,480 triangles), two
    spheres. Positions, centres and radii are FP32 values, so both renderers
    hold the same geometry. Parts are ("triangles", positions, faces) or ("sphere", centre,
    radius)."""
    rng = Pcg32(seed)
    points, quads = trefoil_mesh(128, 16)
    faces = np.concatenate([quads[:, [0, 1, 2]], quads[:, [0, 2, 3]]])
    angle = rng.uniform(0, 2 * np.pi)
    scale = rng.uniform(0.7, 0.9)
    rot = np.array([[np.cos(angle), 0, np.sin(angle)], [0, 1, 0], [-np.sin(angle), 0, np.cos(angle)]])
    knot = (points.astype(np.float64) @ rot.T) * scale * 0.5 + np.array([-0.8, 1.4, -0.6])
    ball_points, ball_faces = displaced_icosphere(5, seed)
    ball = ball_points.astype(np.float64) * 0.9 + np.array([1.1, 1.0, 0.2])
    return [("triangles", knot.astype(np.float32).astype(np.float64), faces),
            ("sphere", (0.0, 0.375, 1.375), 0.375),
            ("triangles", ball.astype(np.float32).astype(np.float64), ball_faces),
            ("sphere", (-1.625, 0.5, 1.25), 0.5),
            ("sphere", (0.0, -1000.0, 0.0), 1000.0)]
