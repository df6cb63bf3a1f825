"""Shared fixtures: the repository on sys.path, the `gpu` marker, generated scenes."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def scene_dir(tmp_path_factory) -> Path:
    return tmp_path_factory.mktemp("scenes")


@pytest.fixture(scope="session")
def room_path(scene_dir) -> Path:
    from albedo_b200 import scenes

    return scenes.room_scene(scene_dir / "room")


@pytest.fixture(scope="session")
def trefoil_path(scene_dir) -> Path:
    from albedo_b200 import scenes

    return scenes.trefoil_scene(scene_dir / "trefoil")
