"""The parallel BVH build gives the one-thread tree (host, CPU only).

Subtrees of large primitive ranges are built on separate threads
(albedo_b200/csrc/host/bvh_build.cpp). tests/cpp/bvh_threads.cpp builds seeded
box sets on 1, 2, 3, 8 and 16 threads and compares every node bit for bit, the
leaf order and the depth. The sets reach SAH splits, cost-chosen leaves, median
splits (coincident centroids; depth past the SAH limit of 32) and sizes on both
sides of the parallel threshold. The one-thread tree is the reference's
(tests/test_host_build.py checks the scenes' trees through bit-exact queries).
"""

import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "albedo_b200" / "csrc"


@pytest.fixture(scope="module")
def lines(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("bvh") / "bvh_threads"
    subprocess.run(["g++", "-std=c++20", "-O2", "-ffp-contract=off", f"-I{CSRC}", str(HERE / "cpp" / "bvh_threads.cpp"),
                    str(CSRC / "host" / "bvh_build.cpp"), str(CSRC / "host" / "host_math.cpp"), "-pthread", "-o",
                    str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()
    return {line.split()[0]: dict(w.split("=") for w in line.split()[1:]) for line in out}


@pytest.mark.parametrize("case", ["uniform", "clustered", "coincident", "geometric", "small1", "small5",
                                  "small8191", "small8192", "small8193", "small16385"])
def test_every_thread_count_builds_the_same_tree(lines, case):
    assert lines[case]["same"] == "1", lines[case]


def test_the_cases_reach_median_splits(lines):
    # Past depth 32 the build splits at the median; coincident centroids never
    # allow a SAH split at all.
    assert int(lines["geometric"]["depth"]) > 32
    assert int(lines["clustered"]["depth"]) > 32
    # 50,000 coincident boxes: median splits only, a balanced tree of 2^14
    # leaves of 3 or 4 boxes.
    assert lines["coincident"]["nodes"] == "32767" and lines["coincident"]["depth"] == "14"
