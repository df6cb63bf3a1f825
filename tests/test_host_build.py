"""The host scene build reproduces the reference exactly (CPU only).

The FP64 restatement of the query path (oracle/trace_oracle.cpp) runs over this
repository's host tables: its BVHs (built by albedo_b200/csrc/host/bvh_build.cpp),
transforms, triangles and smooth normals. Its answers must equal the reference's
Scene::intersect bit for bit on every ray, which holds only if the hierarchy,
the instance transforms and the geometry are the reference's own.
"""

from pathlib import Path

import numpy as np
import pytest

import albedo_b200 as ab
from oracle import reference as ref
from oracle import restatement

pytestmark = pytest.mark.skipif(not (ref.available() and restatement.available()), reason="oracle not built")


def _assets() -> Path | None:
    from oracle import reference_root

    root = reference_root()
    return root / "assets" if root is not None else None


def random_rays(count, seed, low, high):
    rng = np.random.default_rng(seed)
    origin = rng.uniform(low, high, size=(count, 3))
    direction = rng.normal(size=(count, 3))
    direction /= np.linalg.norm(direction, axis=1, keepdims=True)
    return np.concatenate([origin, direction], axis=1).astype(np.float32).astype(np.float64)


def scene_paths(room_path, trefoil_path):
    paths = [room_path, trefoil_path]
    assets = _assets()
    if assets is not None and (assets / "meshes.scene").exists():
        paths.append(assets / "meshes.scene")
    return paths


@pytest.mark.parametrize("index", [0, 1, 2])
def test_restatement_equals_reference_bit_for_bit(index, room_path, trefoil_path):
    paths = scene_paths(room_path, trefoil_path)
    if index >= len(paths):
        pytest.skip("reference assets absent")
    path = paths[index]
    scene = ab.Scene.read(path)
    rays = random_rays(20_000, 21 + index, [-2.8, 0.05, -3.5], [2.8, 4.5, 3.0])
    ours = restatement.intersect(scene, rays)
    theirs = ref.RefScene(path).intersect(rays)
    np.testing.assert_array_equal(ours["hit"], theirs["hit"])
    hit = ours["hit"] == 1
    assert hit.mean() > 0.5
    np.testing.assert_array_equal(ours["object"][hit], theirs["object"][hit])
    np.testing.assert_array_equal(ours["t"][hit], theirs["t"][hit])
    np.testing.assert_array_equal(ours["point"][hit], theirs["point"][hit])
    np.testing.assert_array_equal(ours["normal"][hit], theirs["normal"][hit])
    np.testing.assert_array_equal(ours["shading_normal"][hit], theirs["shading_normal"][hit])
    np.testing.assert_array_equal(ours["front"][hit], theirs["front"][hit])


def test_restatement_reports_triangles_inside_instances(trefoil_path):
    scene = ab.Scene.read(trefoil_path)
    rays = random_rays(20_000, 5, [-2.8, 0.05, -3.5], [2.8, 4.5, 3.0])
    ours = restatement.intersect(scene, rays)
    hit = ours["hit"] == 1
    info = scene.info()
    assert info["objects"] == 9
    # Objects 0 (floor) and 5..7 (knots) are instances; 1..4 and 8 are spheres.
    instanced = np.isin(ours["object"], [0, 5, 6, 7]) & hit
    assert instanced.sum() > 1000
    assert np.all(ours["triangle"][instanced] >= 0)
    assert np.all(ours["triangle"][hit & ~instanced] == -1)
    assert (ours["counts"][hit][:, 0] > 0).all()


def build_flattened(parts):
    """The same scene on both sides: ours through albedo_scene_add_triangles /
    add_sphere, the reference's through Scene::add (TriangleMesh and Sphere)."""
    ours = ab.Scene.create()
    ours.set_camera((0, 2, 6), (0, 1, 0))
    material = ours.add_material(ab.BasicMaterial("diffuse", a=(0.5, 0.5, 0.5)))
    theirs = ref.RefScene.create()
    for part in parts:
        if part[0] == "triangles":
            ours.add_triangles(part[1], part[2], material)
            theirs.add_triangles(part[1], part[2])
        else:
            ours.add_sphere(part[1], part[2], material)
            theirs.add_sphere(part[1], part[2])
    return ours, theirs


def test_flattened_meshes_give_the_reference_object_ids():
    """Meshes added flattened make every triangle its own object, in add order,
    under one TLAS: object ids, t and points equal the reference's bit for bit."""
    from albedo_b200 import scenes

    ours, theirs = build_flattened(scenes.flattened_parts())
    ours.prepare()
    assert ours.info()["objects"] == theirs.object_count() == 4096 + 20480 + 3
    rays = random_rays(50_000, 33, [-2.8, 0.05, -3.5], [2.8, 4.5, 3.0])
    mine = restatement.intersect(ours, rays)
    their = theirs.intersect(rays)
    np.testing.assert_array_equal(mine["hit"], their["hit"])
    hit = mine["hit"] == 1
    assert hit.mean() > 0.3
    np.testing.assert_array_equal(mine["object"][hit], their["object"][hit])
    np.testing.assert_array_equal(mine["t"][hit], their["t"][hit])
    np.testing.assert_array_equal(mine["point"][hit], their["point"][hit])


@pytest.mark.parametrize("which", ["room", "trefoil"])
def test_near_tie_classifier_flags_planted_mistakes(which, room_path, trefoil_path):
    """The FP64 restatement's near-tie classifier (oracle_classify), which the GPU
    ray-id tests rely on: the restatement's own answers are all class 0; answers
    with a wrong object or a wrong miss planted in them are class 2 (unexplained)."""
    scene = ab.Scene.read(room_path if which == "room" else trefoil_path)
    rays = random_rays(20_000, 41, [-2.8, 0.05, -3.5], [2.8, 4.5, 3.0])
    mine = restatement.intersect(scene, rays)
    exact = restatement.classify(scene, rays, mine)["class"]
    assert np.all(exact == 0)
    planted = np.flatnonzero(mine["hit"])[:50]
    wrong_object = {k: mine[k].copy() for k in ("hit", "object", "triangle")}
    wrong_object["object"][planted] = (wrong_object["object"][planted] + 1) % scene.info()["objects"]
    wrong_object["triangle"][planted] = -1
    klass = restatement.classify(scene, rays, wrong_object)["class"]
    assert np.all(klass[planted] == 2) and np.count_nonzero(klass) == len(planted)
    wrong_miss = {k: mine[k].copy() for k in ("hit", "object", "triangle")}
    wrong_miss["hit"][planted] = 0
    klass = restatement.classify(scene, rays, wrong_miss)["class"]
    assert np.all(klass[planted] == 2) and np.count_nonzero(klass) == len(planted)
