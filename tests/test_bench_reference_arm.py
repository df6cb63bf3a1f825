"""bench.py's reference arm on the host (no GPU): the reference's own renderImage,
built from its sources, renders the headline frame (the 1.31M-triangle icosphere,
1920x1080) at 16 spp per timed step and prints one JSON line with the benchmark's
keys. Under torchrun only rank 0 works and prints; the other ranks exit at once.
"""

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

from oracle import reference as ref

BENCH = Path(__file__).resolve().parent.parent / "bench.py"

pytestmark = pytest.mark.skipif(not ref.REF_LIBRARY.exists(), reason="reference library not built")


def run_bench(*args, env=None):
    return subprocess.run([sys.executable, str(BENCH), *args], capture_output=True, text=True,
                          timeout=600, env={**os.environ, **(env or {})})


def test_reference_arm_prints_one_line_for_the_headline_frame():
    done = run_bench("--impl", "reference", "--steps", "1", "--warmup", "0")
    assert done.returncode == 0, done.stderr
    lines = [line for line in done.stdout.splitlines() if line.strip()]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["unit"] == "Mpaths/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 0
    config = line["config"]
    assert config["workload"].startswith("icosphere_8_levels_1310720_tris")
    assert config["resolution"] == [1920, 1080]
    assert config["timed_paths_per_step"] == 1920 * 1080 * config["timed_samples_per_axis"] ** 2
    baseline = line["cpu_baseline"]
    assert baseline["kind"] == "reference" and baseline["cores"] >= 1 and baseline["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "Mpaths/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_runs_on_rank_zero_only():
    done = run_bench("--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
                     env={"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert done.returncode == 0, done.stderr
    assert done.stdout.strip() == ""
