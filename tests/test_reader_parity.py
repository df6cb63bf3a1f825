"""The scene-file and OBJ readers against the reference's readScene, differentially.

Seeded mutations of valid scene and OBJ texts: dropped and duplicated lines,
dropped tokens, numbers replaced by invalid or extreme values, junk appended.
For every case both readers must accept, with the same object count, or both
reject, with the same message (the reference's SceneParseError text names the
line). The reference is the library built from its own sources under oracle/.
"""

import random
import re

import pytest

import albedo_b200 as ab
from oracle import reference as ref

pytestmark = pytest.mark.skipif(not ref.available(), reason="reference library not built")

SCENE = """\
# A scene using every statement.
camera from 0 2.2 6.5  at 0 0.7 0  up 0 1 0  fov 45
material white diffuse color 0.73 0.73 0.73
material tiles checker even 0.8 0.8 0.8  odd 0.1 0.1 0.1  frequency 2
material marble perlin low 0.2 0.15 0.1  high 0.9 0.85 0.8  scale 3  veins 5
material gold conductor eta 0.156 0.424 1.383  k 3.602 2.472 1.915  roughness 0.25
material glass dielectric ior 1.5 roughness 0
material veined mix first gold second marble scale 2 veins 6 threshold 0.45
sphere 0 -1000 0 radius 1000 material tiles
sphere -1.6 0.7 0 radius 0.7 material marble
sphere 1.6 0.7 0 radius 0.7 material veined
mesh knot knot.obj smooth
mesh slab slab.obj
instance knot material gold  scale 0.5  rotate 0 1 0 30  translate 0 1 0
instance slab material glass  fit 1.5  ground  translate 1 0 -1
area_light 0 4 1 radius 0.8 radiance 6 6 5
point_light -2 3 3 intensity 2 2 2
sky nadir 0.1 0.12 0.15 zenith 0.3 0.35 0.45
"""

KNOT = """\
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
v 0.5 0.5 1
vt 0 0
vt 1 0
vt 1 1
vt 0 1
f 1/1 2/2 5/3
f 2/2 3/3 5/3
f 3/3 4/4 5/3
f 4/4 1/1 5/3
f 1 2 3 4
"""

SLAB = """\
v -1 0 -1
v 1 0 -1
v 1 0 1
v -1 0 1
v -1 0.2 -1
v 1 0.2 -1
v 1 0.2 1
v -1 0.2 1
f 1 2 3
f 1 3 4
f -4 -3 -2
f -4 -2 -1
f 1 2 6 5
f 3 4 8 7
"""

BAD_NUMBERS = ["nan", "-1", "0", "1e400", "-1e-320", "abc", "1e-40", "3.5", "-0", "inf", "99999"]


def read_ours(path):
    try:
        scene = ab.Scene.read(path)
        return "ok", scene.info()["objects"]
    except (ValueError, OSError, IndexError, ab.Unsupported) as e:
        return "error", str(e)


def read_theirs(path):
    try:
        scene = ref.RefScene(path)
        return "ok", scene.object_count()
    except RuntimeError as e:
        return "error", str(e)


def mutations(text, rng, count):
    lines = text.splitlines()
    out = []
    for _ in range(count):
        ls = list(lines)
        kind = rng.randrange(6)
        i = rng.randrange(len(ls))
        words = ls[i].split()
        if kind == 0:
            del ls[i]
        elif kind == 1:
            ls.insert(i, ls[i])
        elif kind == 2 and words:
            del words[rng.randrange(len(words))]
            ls[i] = " ".join(words)
        elif kind == 3 and words:
            numeric = [k for k, w in enumerate(words) if re.fullmatch(r"-?[0-9.eE+-]+", w)]
            if numeric:
                words[rng.choice(numeric)] = rng.choice(BAD_NUMBERS)
                ls[i] = " ".join(words)
        elif kind == 4:
            ls[i] = ls[i] + " " + rng.choice(["junk", "1", "material", "nan"])
        else:
            j = rng.randrange(len(ls))
            ls[i], ls[j] = ls[j], ls[i]
        out.append("\n".join(ls) + "\n")
    return out


def same(case_dir, scene_text, knot_text, slab_text):
    case_dir.mkdir()
    (case_dir / "knot.obj").write_text(knot_text)
    (case_dir / "slab.obj").write_text(slab_text)
    path = case_dir / "case.scene"
    path.write_text(scene_text)
    return read_ours(path), read_theirs(path)


def test_the_unmutated_scene_reads_alike(tmp_path):
    ours, theirs = same(tmp_path / "base", SCENE, KNOT, SLAB)
    assert ours == theirs and ours[0] == "ok", (ours, theirs)


@pytest.mark.parametrize("target", ["scene", "knot", "slab"])
def test_mutated_inputs_are_accepted_or_refused_alike(tmp_path, target):
    rng = random.Random({"scene": 11, "knot": 12, "slab": 13}[target])
    base = {"scene": SCENE, "knot": KNOT, "slab": SLAB}[target]
    cases = mutations(base, rng, 300)
    accepted = refused = 0
    for k, text in enumerate(cases):
        texts = {"scene": SCENE, "knot": KNOT, "slab": SLAB}
        texts[target] = text
        ours, theirs = same(tmp_path / f"case{k}", texts["scene"], texts["knot"], texts["slab"])
        assert ours == theirs, (k, text, ours, theirs)
        accepted += ours[0] == "ok"
        refused += ours[0] == "error"
    assert accepted > 10 and refused > 10, (accepted, refused)


def large_obj(rng: random.Random, vertices: int) -> str:
    """A mesh file of several MB: the reader splits files this large into pieces
    read on separate threads."""
    lines = []
    for i in range(vertices):
        lines.append(f"v {rng.uniform(-1, 1):.9f} {rng.uniform(-1, 1):.9f} {rng.uniform(-1, 1):.9f}")
        lines.append(f"vt {rng.random():.6f} {rng.random():.6f}")
        if i >= 2:
            lines.append(f"f {i - 1}/{i - 1} {i}/{i} -1/-1")
    return "\n".join(lines) + "\n"


def test_large_meshes_with_late_errors_read_alike(tmp_path):
    # Errors placed anywhere in a file of about 5 MB, so in any of its pieces.
    rng = random.Random(21)
    base = large_obj(rng, 60_000).split("\n")
    scene = "camera from 0 0 5 at 0 0 0 up 0 1 0 fov 40\nmaterial white diffuse color 0.5 0.5 0.5\n" \
            "mesh big big.obj\ninstance big material white\n"
    outcomes = []
    for k in range(12):
        lines = list(base)
        if k > 0:
            i = rng.randrange(len(lines) - 1)
            lines[i] = rng.choice([lines[i] + " junk", "f 1 2", f"f {10 ** 9} 1 2", "v 1 nan 2", "vt", lines[i]])
        case = tmp_path / f"case{k}"
        case.mkdir()
        (case / "big.obj").write_text("\n".join(lines))
        (case / "case.scene").write_text(scene)
        ours, theirs = read_ours(case / "case.scene"), read_theirs(case / "case.scene")
        assert ours == theirs, (k, ours, theirs)
        outcomes.append(ours[0])
    assert "ok" in outcomes and "error" in outcomes


BASE = """\
camera from 0 2 6  at 0 0.7 0
material white diffuse color 0.7 0.7 0.7
material gold conductor eta 0.156 0.424 1.383  k 3.602 2.472 1.915
material mixed mix first white second gold scale 2
mesh knot knot.obj
"""

# One statement each, aimed at every check of every statement: the value kinds
# and ranges, fields given twice or unknown, required fields missing, name and
# reference checks, limits within one line, and instance operations.
STATEMENTS = [
    "camera from 0 0 1 at 0 0 0",
    "sky 0.1 0.1 0.1", "sky 0.1 0.1", "sky 0.1 0.1 0.1 extra", "sky nadir 1 1 1", "sky zenith 1 1 1 nadir 1 1 -1",
    "sky nadir 1 1 1 zenith 1 1 1 nadir 1 1 1", "sky 2e6 0 0", "sky nadir 1 1 1 zenith 1 1 1 up 1",
    "material", "material 9bad diffuse color 1 1 1", "material white diffuse color 1 1 1", "material m",
    "material m velvet color 1 1 1", "material m diffuse", "material m diffuse color 1 1", "material m diffuse color 1 1 2",
    "material m diffuse color 1 1 1 color 1 1 1", "material m diffuse colour 1 1 1",
    "material m checker even 1 1 1 odd 0 0 0", "material m checker even 1 1 1 frequency 2",
    "material m checker odd 1 1 1 frequency 2", "material m checker even 1 1 1 odd 0 0 0 frequency 0",
    "material m checker even 1 1 1 odd 0 0 0 frequency -2",
    "material m perlin low 0 0 0 high 1 1 1", "material m perlin low 0 0 0 high 1 1 1 scale 1 veins 101",
    "material m perlin low 0 0 0 high 1 1 1 scale 1 veins -1", "material m perlin high 1 1 1 scale 1",
    "material m conductor eta 1 1 1", "material m conductor k 1 1 1", "material m conductor eta 1 2 2 k 0 1 1",
    "material m conductor eta 0.0001 1 1 k 1 1 1", "material m conductor eta 1 1 1 k 1 1 1 roughness 2",
    "material m conductor eta 1 1 1 k 1 1 2000", "material m dielectric", "material m dielectric ior 0.001",
    "material m dielectric ior 1.5 roughness 1.5", "material m dielectric ior 1.5 ior 1.5",
    "material m mix first white", "material m mix first white second gold",
    "material m mix first white second mixed scale 1", "material m mix first nothing second gold scale 1",
    "material m mix first 7 second gold scale 1", "material m mix first white second gold scale 1 threshold 2",
    "material m mix first white second gold scale 1 veins 200", "material m mix second gold scale 1",
    "sphere 0 0 0 radius 1", "sphere 0 0 radius 1 material white", "sphere 0 0 0 material white",
    "sphere 0 0 0 radius 0 material white", "sphere 0 0 0 radius -1 material white",
    "sphere 0 0 0 radius 1 material ghost", "sphere 0 0 0 radius 1 material white material white",
    "sphere 0 0 0 radius 1e308 material white",
    "sphere 0 0 0 radius 1 material white color 1 1 1", "sphere 0 0 0 radius x material white",
    "point_light 0 0 0", "point_light 0 0 0 intensity 1 1 -1", "point_light 0 0 intensity 1 1 1",
    "area_light 0 3 0 radius 1", "area_light 0 3 0 radiance 1 1 1", "area_light 0 3 0 radius 1 radiance 1 1 1",
    "area_light 0 3 0 radius 0 radiance 1 1 1", "area_light 0 3 0 radius 1 radiance 1 1 1 material ghost",
    "mesh knot knot.obj", "mesh other", "mesh other ../knot.obj", "mesh other /etc/passwd", "mesh other missing.obj",
    "mesh other knot.obj smooth extra", "mesh other . smooth", "mesh 1x knot.obj",
    "instance knot", "instance ghost material white", "instance knot material white material gold",
    "instance knot material white spin 1", "instance knot material white scale 2",
    "instance knot material white scale 2 1", "instance knot material white scale 2 1 3",
    "instance knot material white scale 0", "instance knot material white scale 2 fit 1",
    "instance knot material white rotate 0 0 0 30", "instance knot material white rotate 0 1 0",
    "instance knot material white rotate 0 1 0 x", "instance knot material white fit 0",
    "instance knot material white fit 1 ground", "instance knot material white ground translate 0 1",
    "instance knot material white translate 1e308 0 0 scale 1e10 fit 1",
    "instance knot material white translate 1e308 0 0 scale 1e10 ground",
    "instance knot material white " + " ".join(["translate 0 0 0"] * 17),
    "instance knot material white " + " ".join(["ground"] * 16),
    "warp 1 2 3", "camera", "  # only a comment", "",
]


@pytest.mark.parametrize("statement", STATEMENTS)
def test_each_statement_check_reads_alike(tmp_path, statement):
    """Every statement's checks, one statement at a time after a valid prefix:
    both readers accept with the same object count, or refuse with the same
    message. (Coordinates beyond FP32's range, which the reference accepts and
    the device tables cannot hold, are refused at commit with ALBEDO_UNSUPPORTED;
    tests/test_abi.py covers them.)"""
    ours, theirs = same(tmp_path / "case", BASE + statement + "\n", KNOT, SLAB)
    assert ours == theirs, (statement, ours, theirs)
