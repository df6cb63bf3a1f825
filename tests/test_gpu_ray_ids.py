"""Ray-query identity: hit flags, object ids and triangle ids of 10^6 seeded
random rays against the reference and its FP64 restatement (GPU).

Every disagreement must be a near-tie that FP32 rounding explains; none may be
left unexplained. The FP64 restatement (oracle/trace_oracle.cpp, equal to the
reference's Scene::intersect bit for bit, tests/test_host_build.py) classifies
each disagreement with an error bound of 32 FP32 ulps of the largest coordinate
involved (oracle/restatement.py TIE_ULPS): the device's primitive must be
within that bound of being hit, and no farther along the ray than the nearest
primitive that is surely hit, plus both bounds; a device miss must have no
primitive surely hit. Ties are counted and bounded (at most 2 in 10^4 rays).

  ids        the reference's object ids (HitRecord::object, add order) for the
             room and the instanced trefoil; triangle ids inside instanced meshes
             (which the reference's API does not expose) against the
             restatement, for the trefoil and the 1.31M-triangle icosphere; and
             per-triangle object ids for meshes added flattened through
             albedo_scene_add_triangles on our side and Scene::add(TriangleMesh)
             on the reference's (scene/scene.cpp:33-61)
  t          within 2 FP32 ulps of the reference's FP64 t, rounded, where the
             ids agree
  geometry   front-face flags equal; the geometric and shading normals' dot
             products with the reference's above 1 - 1e-5
"""

import numpy as np
import pytest

import albedo_b200 as ab
from albedo_b200 import scenes
from oracle import reference as ref
from oracle import restatement

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (ref.available() and restatement.available()), reason="oracle not built")]

MAX_TIES = 200  # per 10^6 rays


def unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def random_rays(count, seed, low, high):
    rng = np.random.default_rng(seed)
    origin = rng.uniform(low, high, size=(count, 3))
    direction = unit(rng.normal(size=(count, 3)))
    return np.concatenate([origin, direction], axis=1).astype(np.float32)


def ulp_distance(ours_f32, reference_f64):
    """Distance in FP32 ulps between a device float and the reference double rounded to FP32."""
    a = ours_f32.astype(np.float32).view(np.int32).astype(np.int64)
    b = reference_f64.astype(np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


def classify(scene, rays, ours):
    """(agree, ties) masks: the device's answer equals the FP64 restatement's, or
    differs by an explained near-tie; asserts that nothing is unexplained. The
    disagreements are counted first (the classification tests every primitive of
    the scene for each of them), so a broken traversal fails at once."""
    mine = restatement.intersect(scene, rays.astype(np.float64))
    differ = (ours["hit"] != mine["hit"]) | ((ours["hit"] == 1) & ((ours["object"] != mine["object"]) |
                                                                   (ours["triangle"] != mine["triangle"])))
    assert differ.sum() <= MAX_TIES * len(rays) / 1e6, differ.sum()
    subset = np.flatnonzero(differ)
    klass = np.zeros(len(rays), np.int32)
    if len(subset):
        picked = {k: ours[k][subset] for k in ("hit", "object", "triangle")}
        result = restatement.classify(scene, rays[subset], picked)
        klass[subset] = result["class"]
        unexplained = np.flatnonzero(result["class"] == 2)
        assert len(unexplained) == 0, (len(unexplained), subset[unexplained[:10]], result["detail"][unexplained[:10]])
    assert np.all(klass[subset] == 1)
    return klass == 0, klass == 1


@pytest.mark.parametrize("which", ["room", "trefoil"])
def test_ray_queries_match_the_reference(which, room_path, trefoil_path):
    path = room_path if which == "room" else trefoil_path
    scene = ab.Scene.load(path)
    rays = random_rays(1_000_000, 5, [-2.8, 0.05, -3.5], [2.8, 4.5, 3.0])
    ours = scene.intersect(rays, geometry=True)
    theirs = ref.RefScene(path).intersect(rays.astype(np.float64))
    agree, ties = classify(scene, rays, ours)
    # Where the restatement agrees with the device, so does the reference.
    same = (ours["hit"] == theirs["hit"]) & ((ours["hit"] == 0) | (ours["object"] == theirs["object"]))
    assert np.all(same[agree])
    both = same & (ours["hit"] == 1) & agree
    ulps = ulp_distance(ours["t"][both], theirs["t"][both])
    assert np.all(ulps <= 2), (np.quantile(ulps, [0.5, 0.999, 1.0]), np.sum(ulps > 2))
    np.testing.assert_array_equal(ours["front"][both], theirs["front"][both])
    ndot = np.sum(ours["normal"][both] * theirs["normal"][both], axis=1)
    assert ndot.min() > 1 - 1e-5, ndot.min()
    sdot = np.sum(ours["shading_normal"][both] * theirs["shading_normal"][both], axis=1)
    assert sdot.min() > 1 - 1e-5, sdot.min()


@pytest.mark.parametrize("which", ["trefoil", "icosphere"])
def test_triangle_ids_inside_instances_match_the_restatement(which, trefoil_path, tmp_path_factory):
    """The device's triangle id within an instanced mesh against the FP64
    restatement's (the reference does not expose it), on the instanced trefoil
    and on the 1.31M-triangle icosphere."""
    if which == "trefoil":
        path = trefoil_path
    else:
        path = scenes.icosphere_scene(tmp_path_factory.mktemp("ids") / "icosphere", levels=8)
    scene = ab.Scene.load(path)
    rays = random_rays(1_000_000, 17, [-2.8, 0.05, -3.5], [2.8, 4.5, 3.0])
    ours = scene.intersect(rays)
    mine = restatement.intersect(scene, rays.astype(np.float64))
    agree, ties = classify(scene, rays, ours)
    inside = agree & (mine["triangle"] >= 0)
    assert inside.sum() > 100_000, inside.sum()
    np.testing.assert_array_equal(ours["triangle"][inside], mine["triangle"][inside])
    ulps = ulp_distance(ours["t"][inside], mine["t"][inside])
    assert np.all(ulps <= 2), (np.quantile(ulps, [0.5, 0.999, 1.0]), np.sum(ulps > 2))


def build_flattened(parts):
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
    ours.commit()
    return ours, theirs


def test_flattened_mesh_object_ids_match_the_reference():
    """Meshes added flattened (every triangle its own object): per-triangle
    object ids of 10^6 rays against the reference's Scene::intersect."""
    ours_scene, theirs_scene = build_flattened(scenes.flattened_parts())
    rays = random_rays(1_000_000, 23, [-2.8, 0.05, -3.5], [2.8, 4.5, 3.0])
    ours = ours_scene.intersect(rays)
    theirs = theirs_scene.intersect(rays.astype(np.float64))
    agree, ties = classify(ours_scene, rays, ours)
    same = (ours["hit"] == theirs["hit"]) & ((ours["hit"] == 0) | (ours["object"] == theirs["object"]))
    assert np.all(same[agree])
    hits = agree & (ours["hit"] == 1)
    assert hits.sum() > 300_000, hits.sum()
    # Most hits are on the meshes' triangles, each its own object.
    assert np.mean(ours["object"][hits] > 3) > 0.3
    ulps = ulp_distance(ours["t"][hits], theirs["t"][hits])
    assert np.all(ulps <= 2), (np.quantile(ulps, [0.5, 0.999, 1.0]), np.sum(ulps > 2))
