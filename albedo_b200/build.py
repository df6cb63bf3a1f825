"""Builds libalbedo_b200.so in-tree: C++20 host sources with g++, CUDA sources
with nvcc for sm_100a, linked with the static CUDA runtime.

Host sources build with -ffp-contract=off so scene building rounds exactly as
the reference's x86-64 build does (no FMA).
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
CSRC = PACKAGE / "csrc"
BUILD = PACKAGE / "_build"
LIBRARY = PACKAGE / "libalbedo_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-std=c++20", "-O2", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra"]
NVCCFLAGS = ARCH + ["-std=c++20", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                    "-Xptxas", "-v"]


def _cuda_home() -> Path:
    nvcc = shutil.which("nvcc")
    if nvcc:
        return Path(nvcc).resolve().parent.parent
    return Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))


def _sources() -> tuple[list[Path], list[Path]]:
    cpp = sorted(CSRC.rglob("*.cpp"))
    cu = sorted(CSRC.rglob("*.cu"))
    return cpp, cu


def _headers() -> list[Path]:
    return sorted(list(CSRC.rglob("*.hpp")) + list(CSRC.rglob("*.cuh")) + [PACKAGE.parent / "include" / "albedo_b200.h"])


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, headers: list[Path], log: list[str]) -> Path:
    obj = BUILD / (src.relative_to(CSRC).as_posix().replace("/", "__") + ".o")
    if not _stale(obj, [src] + headers):
        return obj
    cuda = _cuda_home()
    if src.suffix == ".cu":
        cmd = [str(cuda / "bin" / "nvcc")] + NVCCFLAGS + ["-c", str(src), "-o", str(obj)]
    else:
        cmd = [os.environ.get("CXX", "g++")] + CXXFLAGS + [f"-I{cuda / 'include'}", "-c", str(src), "-o", str(obj)]
    result = subprocess.run(cmd, capture_output=True, text=True)
    log.append(f"$ {' '.join(cmd)}\n{result.stdout}{result.stderr}")
    if result.returncode != 0:
        raise RuntimeError(f"compiling {src.name} failed:\n{result.stdout}{result.stderr}")
    return obj


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    cpp, cu = _sources()
    headers = _headers()
    log: list[str] = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        objects = list(pool.map(lambda s: _compile(s, headers, log), cpp + cu))
    if _stale(LIBRARY, objects):
        cuda = _cuda_home()
        # Linked beside the library and renamed over it, so a reader never sees
        # a partly written file.
        partial = LIBRARY.with_suffix(".so.partial")
        cmd = [str(cuda / "bin" / "nvcc")] + ARCH + ["-shared", "-cudart", "static", "-o", str(partial)] + [
            str(o) for o in objects]
        result = subprocess.run(cmd, capture_output=True, text=True)
        log.append(f"$ {' '.join(cmd)}\n{result.stdout}{result.stderr}")
        if result.returncode != 0:
            raise RuntimeError(f"linking failed:\n{result.stdout}{result.stderr}")
        os.replace(partial, LIBRARY)
    (BUILD / "build.log").write_text("\n".join(log))
    if verbose:
        print("\n".join(log))
    return LIBRARY


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIBRARY)
