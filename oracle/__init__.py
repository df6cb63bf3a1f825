"""Test infrastructure: the reference renderer built from its own sources, and
restatements of its algorithms, used only as the checker by tests, the smoke
check and the CPU-baseline legs of bench.py."""

import subprocess
from pathlib import Path


def reference_root() -> Path | None:
    """The reference checkout as oracle/Makefile resolves it (ALBEDO_REFERENCE or
    its documented default), or None where it is absent (GPU machines receive
    the prebuilt oracle libraries only)."""
    result = subprocess.run(["make", "-s", "-C", str(Path(__file__).resolve().parent), "reference-root"],
                            capture_output=True, text=True)
    root = Path(result.stdout.strip()) if result.returncode == 0 and result.stdout.strip() else None
    return root if root is not None and (root / "src").exists() else None
