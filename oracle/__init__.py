"""Test infrastructure: the reference renderer built from its own sources, and
restatements of its algorithms, used only as the checker by tests, the smoke
check and the CPU-baseline legs of bench.py."""
