"""The C ABI library loads, exports every declared symbol, and its host-side scene
reading agrees with the reference's (CPU only: nothing here launches a kernel)."""

import re
from pathlib import Path

import pytest

import albedo_b200 as ab
from albedo_b200._lib import PROTOTYPES, library
from oracle import reference as ref

HEADER = Path(__file__).resolve().parent.parent / "include" / "albedo_b200.h"


def declared_functions() -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(albedo_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported_and_bound():
    names = declared_functions()
    assert len(names) >= 25
    lib = library()
    for name in names:
        assert hasattr(lib, name), name
        assert name in PROTOTYPES, name


def test_scene_files_read_like_the_reference(room_path, trefoil_path):
    if not ref.available():
        pytest.skip("reference library not built")
    for path in (room_path, trefoil_path):
        ours = ab.Scene.read(path).info()
        assert ours["objects"] == ref.RefScene(path).object_count()


def test_room_scene_layout(room_path):
    info = ab.Scene.read(room_path).info()
    assert info["objects"] == 10  # 4 walls, 5 spheres, the area light
    assert info["lights"] == 3   # area, point, sky
    assert info["stack_capacity"] >= info["stack_need"]


def test_trefoil_scene_layout(trefoil_path):
    info = ab.Scene.read(trefoil_path).info()
    assert info["objects"] == 9  # floor, 4 walls, 3 knots, the area light
    assert info["triangles"] == 2 + 256 * 32 * 2


@pytest.mark.parametrize("text, line, fragment", [
    ("camera from 0 0 0 at 0 0 -1\nsphere 0 0 0 radius -1 material x\n", 2, "not defined"),
    ("camera from 0 0 0 at 0 0 -1\nmaterial m diffuse color 2 0 0\n", 2, "between 0 and 1"),
    ("camera from 0 0 0 at 0 0 -1\nbogus 1 2 3\n", 2, "unknown statement"),
    ("material m diffuse color 0.5 0.5 0.5\n", 0, "no camera"),
    ("camera from 0 0 0 at 0 0 0\n", 1, "distance from camera position"),
    ("camera from 0 0 0 at 0 0 -1\nmaterial m diffuse color 0.5 0.5 0.5\nsphere 0 0 0 radius 0 material m\n", 3,
     "sphere radius"),
])
def test_scene_errors_name_the_line(tmp_path, text, line, fragment):
    path = tmp_path / "bad.scene"
    path.write_text(text)
    with pytest.raises(ab.SceneParseError) as error:
        ab.Scene.read(path)
    message = str(error.value)
    assert fragment in message
    if line:
        assert message.startswith(f"scene line {line}:")


def test_missing_scene_file_is_an_os_error(tmp_path):
    with pytest.raises(OSError):
        ab.Scene.read(tmp_path / "absent.scene")


def test_mesh_paths_cannot_leave_the_scene_directory(tmp_path):
    path = tmp_path / "escape.scene"
    path.write_text("camera from 0 0 0 at 0 0 -1\nmesh m ../outside.obj\n")
    with pytest.raises(ab.SceneParseError, match="relative to the scene"):
        ab.Scene.read(path)


def test_builder_rejects_what_the_reference_rejects():
    scene = ab.Scene.create()
    white = scene.add_material(ab.BasicMaterial(a=(0.5, 0.5, 0.5)))
    with pytest.raises(ValueError, match="sphere radius"):
        scene.add_sphere((0, 0, 0), 0.0, white)
    with pytest.raises(ValueError, match="material 7 is not defined"):
        scene.add_sphere((0, 0, 0), 1.0, 7)
    with pytest.raises(IndexError):
        scene.add_mesh([[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 1, 5]])
    with pytest.raises(ValueError, match="at least one triangle"):
        scene.add_mesh([[0, 0, 0], [1, 0, 0], [2, 0, 0]], [[0, 1, 2]])


def test_geometry_beyond_fp32_range_is_refused_not_rendered_wrong():
    # The reference (FP64) accepts a sphere at 1e300; the device tables are FP32,
    # so preparing the scene reports ALBEDO_UNSUPPORTED instead of storing inf.
    scene = ab.Scene.create()
    white = scene.add_material(ab.BasicMaterial(a=(0.5, 0.5, 0.5)))
    scene.set_camera((0, 0, 5), (0, 0, 0))
    scene.add_sphere((0, 0, 0), 1.0, white)
    scene.add_sphere((1e300, 0, 0), 1.0, white)
    with pytest.raises(ab.Unsupported, match="sphere 1 has a coordinate beyond the FP32 range"):
        scene.prepare()
    huge_but_finite = ab.Scene.create()
    white = huge_but_finite.add_material(ab.BasicMaterial(a=(0.5, 0.5, 0.5)))
    huge_but_finite.set_camera((0, 0, 5), (0, 0, 0))
    huge_but_finite.add_sphere((1e30, 0, 0), 1e29, white)
    huge_but_finite.prepare()
