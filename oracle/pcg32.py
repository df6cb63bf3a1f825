"""Test infrastructure: a numpy restatement of the reference's random streams.

    Pcg32 (XSH-RR, 64-bit state), seeding as pcg32_srandom_r   sampling/pcg32.hpp:18-64
    mixBits = SplitMix64 output function                        sampling/sample_generator.hpp:17-22
    SampleGenerator::forPixel: stream = mixBits(y * W + x)      sampling/sample_generator.hpp:35-45
    nextReal = u32 * 2^-32 (double)                             sampling/pcg32.hpp:51-57

Pinned by the reference's known-answer test (tests/sampling/pcg32_test.cpp:12-28:
the first six outputs of PCG32 seeded (42, 54)) and by streams of the reference
library itself.
"""

from __future__ import annotations

import numpy as np

MULTIPLIER = np.uint64(6364136223846793005)


def mix_bits(value) -> np.ndarray:
    v = np.asarray(value, dtype=np.uint64)
    with np.errstate(over="ignore"):
        v = (v ^ (v >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        v = (v ^ (v >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return v ^ (v >> np.uint64(31))


class Pcg32Streams:
    """Many PCG32 generators advanced in lockstep (one per element)."""

    def __init__(self, seed, stream):
        stream = np.asarray(stream, dtype=np.uint64)
        self.inc = (stream << np.uint64(1)) | np.uint64(1)
        self.state = np.zeros_like(self.inc)
        self.next_u32()
        with np.errstate(over="ignore"):
            self.state = self.state + np.asarray(seed, dtype=np.uint64)
        self.next_u32()

    def next_u32(self) -> np.ndarray:
        old = self.state
        with np.errstate(over="ignore"):
            self.state = old * MULTIPLIER + self.inc
        xorshifted = (((old >> np.uint64(18)) ^ old) >> np.uint64(27)) & np.uint64(0xFFFFFFFF)
        rot = old >> np.uint64(59)
        left = (xorshifted << ((np.uint64(32) - rot) & np.uint64(31))) & np.uint64(0xFFFFFFFF)
        return ((xorshifted >> rot) | left).astype(np.uint32)

    def next_real(self) -> np.ndarray:
        return self.next_u32().astype(np.float64) * (1.0 / 4294967296.0)


def pixel_streams(seed: int, xs, ys, width: int) -> Pcg32Streams:
    index = np.asarray(ys, dtype=np.uint64) * np.uint64(width) + np.asarray(xs, dtype=np.uint64)
    return Pcg32Streams(np.full(index.shape, seed, dtype=np.uint64), mix_bits(index))
