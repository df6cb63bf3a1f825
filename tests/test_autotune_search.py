"""The autotuner's search (albedo_b200/csrc/autotune.hpp), on the host.

The header is compiled with g++ into a small program that runs the exhaustive
and coordinate-descent searches on synthetic cost functions (tests/cpp/
autotune_search.cpp). Checked: both find the known minimum; every setting is
measured once (memoised); a setting that cannot run (+inf) is never kept; a
starting setting without one value per knob is refused.
"""

import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def output(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("autotune") / "autotune_search"
    subprocess.run(["g++", "-std=c++20", "-O1", str(HERE / "cpp" / "autotune_search.cpp"), "-o", str(exe)],
                   check=True)
    lines = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()
    return {line.split()[0]: line.split()[1:] for line in lines}


def test_exhaustive_finds_the_minimum_measuring_each_setting_once(output):
    words = output["exhaustive"]
    assert words[:3] == ["16", "4", "64"]
    assert "evaluations=36" in words and "calls=36" in words  # 3 x 3 x 4, start among them
    assert "best=1" in words


def test_descent_finds_the_separable_minimum(output):
    words = output["descent"]
    assert words[:3] == ["16", "4", "64"]
    evaluations = int(next(w for w in words if w.startswith("evaluations=")).split("=")[1])
    calls = int(next(w for w in words if w.startswith("calls=")).split("=")[1])
    assert evaluations == calls and evaluations < 36


def test_unrunnable_settings_are_never_kept(output):
    assert output["broken"] == ["16"]


def test_start_needs_one_value_per_knob(output):
    assert output["mismatch"] == ["refused"]
