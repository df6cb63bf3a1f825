"""The film's output encoding and PPM writer against the reference, on the host.

The device resolve compares each pixel's average against a table of the
smallest double of every byte, built with the reference's transfer function
(color/srgb.cpp:18-36), starting from a per-bucket byte (buckets of doubles by
exponent and top mantissa bits). Here both tables, and the kernels' steps
restated in numpy (two table reads, or one read of a packed entry), are checked against the reference's own
toByte(encodeSrgb(x)) on the golden values of its tests
(tests/color/srgb_test.cpp, tests/image/ppm_test.cpp), on millions of seeded
values and on every value within 2,000 ulps of each threshold, where a rounding
difference could show. The PPM writer (image/ppm.cpp:47-85) is compared byte
for byte with the reference's, including its failures.
"""

import os

import numpy as np
import pytest

import albedo_b200 as ab
from oracle import reference as ref

needs_ref = pytest.mark.skipif(not ref.available(), reason="reference library not built")


def table_bytes(values: np.ndarray) -> np.ndarray:
    """The byte the table gives: the largest b >= 1 with value >= lower[b], else 0."""
    lower = ab.srgb_thresholds()[1:]
    values = np.asarray(values, dtype=np.float64)
    b = np.searchsorted(lower, values, side="right")
    return np.where(np.isnan(values), 0, b).astype(np.uint8)


def bucket_bytes(values: np.ndarray) -> np.ndarray:
    """The device resolve's steps, in numpy: below lower[1] (or NaN) 0, from
    lower[255] 255, else the bucket's start byte plus one comparison."""
    lower, start = ab.srgb_tables()
    v = np.asarray(values, dtype=np.float64)
    out = np.zeros(v.shape, dtype=np.int64)
    with np.errstate(invalid="ignore"):
        mid = (v >= lower[1]) & (v < lower[255])
        out[v >= lower[255]] = 255
    bucket = (v[mid].view(np.int64) >> ab.SRGB_BUCKET_SHIFT) - ab.SRGB_BUCKET_BASE
    assert bucket.min(initial=0) >= 0 and bucket.max(initial=0) < ab.SRGB_BUCKETS
    b = start[bucket].astype(np.int64)
    out[mid] = b + (v[mid] >= lower[b + 1])
    return out.astype(np.uint8)


def packed_table() -> np.ndarray:
    """The tiled kernel's table: one 64-bit entry per bucket holding the start
    byte (bits 48-55) and the low bits of the bucket's threshold (2^shift when it
    holds none)."""
    lower, start = ab.srgb_tables()
    shift = ab.SRGB_BUCKET_SHIFT
    low_mask, none = (1 << shift) - 1, 1 << shift
    packed = np.empty(ab.SRGB_BUCKETS, dtype=np.uint64)
    for k, st in enumerate(start.tolist()):
        low = none
        if st < 255:
            t = int(lower[st + 1:st + 2].view(np.int64)[0])
            if t >> shift == ab.SRGB_BUCKET_BASE + k:
                low = t & low_mask
        packed[k] = (int(st) << 48) | low
    return packed


def packed_bytes(values: np.ndarray) -> np.ndarray:
    """The tiled device kernel's byte lookup, in numpy: one packed entry per
    bucket, its threshold's low bits compared with the value's."""
    lower = ab.srgb_thresholds()
    packed = packed_table()
    shift = ab.SRGB_BUCKET_SHIFT
    low_mask, none = (1 << shift) - 1, 1 << shift
    v = np.asarray(values, dtype=np.float64).reshape(-1)
    bits = v.view(np.int64)
    bucket = np.clip((bits >> shift) - ab.SRGB_BUCKET_BASE, 0, ab.SRGB_BUCKETS - 1)
    entry = packed[bucket]
    byte = (entry >> np.uint64(48)).astype(np.int64) + (
        (bits.astype(np.uint64) & np.uint64(low_mask)) >= (entry & np.uint64((none | low_mask)))).astype(np.int64)
    with np.errstate(invalid="ignore"):
        out = np.where(v >= lower[255], 255, np.where(v >= lower[1], byte, 0))
    return out.astype(np.uint8).reshape(np.shape(values))


def adversarial_accumulators():
    """Sums whose averages fall within 6 ulps of every threshold and bucket edge,
    for counts that are and are not powers of two."""
    lower = ab.srgb_thresholds()[1:]
    edges = ((ab.SRGB_BUCKET_BASE + np.arange(ab.SRGB_BUCKETS + 1, dtype=np.int64)) << ab.SRGB_BUCKET_SHIFT
             ).view(np.float64)
    targets = np.concatenate([lower, edges])
    sums, counts = [], []
    for c in (3, 7, 36, 49, 64, 255, 1_000_003, 2**40 + 3):
        s0 = (targets * float(c)).view(np.int64)
        for d in range(-6, 7):
            sums.append((s0 + d).view(np.float64))
            counts.append(np.full(len(targets), c, dtype=np.uint64))
    return np.concatenate(sums), np.concatenate(counts)


def reference_average_bytes(sums, counts):
    c = np.asarray(counts, dtype=np.uint64)
    with np.errstate(invalid="ignore", divide="ignore"):
        avg = np.where(c > 0, sums / np.where(c > 0, c.astype(np.float64), 1.0), 0.0)
    return ref.srgb_bytes(avg)


def test_thresholds_are_increasing_and_bracket_the_byte_range():
    lower = ab.srgb_thresholds()
    assert lower[0] == -np.inf
    assert np.all(np.diff(lower[1:]) > 0)
    assert 0 < lower[1] < 1e-3 and 0.99 < lower[255] <= 1.0


# (linear value, byte) pairs from the reference's tests: black, white, 50% linear
# is 188 (srgb_test.cpp:56-58), clamping above one and below zero
# (ppm_test.cpp:60-67), NaN and infinities (srgb_test.cpp:52-76).
GOLDEN = [(0.0, 0), (1.0, 255), (0.5, 188), (4.0, 255), (-2.0, 0), (-0.5, 0), (7.0, 255),
          (np.nan, 0), (np.inf, 255), (-np.inf, 0), (0.001, 3), (-0.0, 0)]


@needs_ref
def test_golden_values_from_the_reference_tests():
    values = np.array([v for v, _ in GOLDEN])
    expected = np.array([b for _, b in GOLDEN], dtype=np.uint8)
    assert np.array_equal(ref.srgb_bytes(values), expected)
    assert np.array_equal(table_bytes(values), expected)
    assert np.array_equal(bucket_bytes(values), expected)
    assert np.array_equal(packed_bytes(values), expected)


@needs_ref
def test_table_equals_the_reference_on_seeded_values():
    rng = np.random.default_rng(7)
    values = np.concatenate([
        rng.uniform(-0.1, 1.2, 2_000_000),
        np.exp(rng.uniform(np.log(1e-7), np.log(2.0), 2_000_000)),
        rng.uniform(0.0031, 0.00316, 200_000),  # around the segment switch
        # Arbitrary bit patterns: every sign, exponent and NaN payload.
        rng.integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, 1_000_000, dtype=np.int64).view(np.float64),
    ])
    theirs = ref.srgb_bytes(values)
    assert np.array_equal(table_bytes(values), theirs)
    assert np.array_equal(bucket_bytes(values), theirs)
    assert np.array_equal(packed_bytes(values), theirs)


@needs_ref
def test_table_equals_the_reference_within_2000_ulps_of_every_threshold():
    lower = ab.srgb_thresholds()[1:]
    bits = lower.view(np.int64)[:, None] + np.arange(-2000, 2001, dtype=np.int64)[None, :]
    values = bits.reshape(-1).view(np.float64)
    theirs = ref.srgb_bytes(values)
    assert np.array_equal(table_bytes(values), theirs)
    assert np.array_equal(bucket_bytes(values), theirs)
    assert np.array_equal(packed_bytes(values), theirs)
    # Each threshold is where the reference's byte steps up.
    assert np.array_equal(ref.srgb_bytes(lower), np.arange(1, 256, dtype=np.uint8))
    below = np.nextafter(lower, -np.inf)
    assert np.array_equal(ref.srgb_bytes(below), np.arange(0, 255, dtype=np.uint8))


@needs_ref
def test_averages_next_to_every_decision_give_the_reference_bytes():
    sums, counts = adversarial_accumulators()
    with np.errstate(invalid="ignore"):
        averages = sums / counts.astype(np.float64)
    np.testing.assert_array_equal(packed_bytes(averages), reference_average_bytes(sums, counts))


def test_every_bucket_holds_at_most_one_threshold():
    lower, start = ab.srgb_tables()
    edges = ((ab.SRGB_BUCKET_BASE + np.arange(ab.SRGB_BUCKETS + 1, dtype=np.int64)) << ab.SRGB_BUCKET_SHIFT).view(np.float64)
    inside = np.searchsorted(lower[1:], edges[1:], side="left") - np.searchsorted(lower[1:], edges[:-1], side="right")
    assert inside.max() <= 1
    assert np.array_equal(start, table_bytes(edges[:-1]))
    assert edges[0] < lower[1] and lower[255] <= edges[-1]


TWO_PIXEL_PPM = b"P6\n2 1\n255\n\xFF\x00\x00\xBC\xBC\xBC"


def test_two_pixel_image_writes_the_reference_test_bytes(tmp_path):
    # ppm_test.cpp:22-33: a red pixel beside a 50%-gray one.
    rgb = np.array([[[255, 0, 0], [188, 188, 188]]], dtype=np.uint8)
    path = tmp_path / "two.ppm"
    ab.write_ppm(path, rgb)
    assert path.read_bytes() == TWO_PIXEL_PPM


def test_overwrites_a_longer_existing_file(tmp_path):
    path = tmp_path / "old.ppm"
    path.write_bytes(b"x" * 64)
    ab.write_ppm(path, np.array([[[255, 0, 0], [188, 188, 188]]], dtype=np.uint8))
    assert path.read_bytes() == TWO_PIXEL_PPM


@needs_ref
@pytest.mark.parametrize("shape", [(1, 1), (2, 3), (37, 53), (270, 480)])
def test_files_equal_the_reference_writer(tmp_path, shape):
    h, w = shape
    rng = np.random.default_rng(h * 1000 + w)
    averages = rng.uniform(-0.2, 1.4, size=(h, w, 3))
    averages.reshape(-1)[rng.choice(averages.size, size=max(1, averages.size // 50))] = np.nan
    ours, theirs = tmp_path / "ours.ppm", tmp_path / "theirs.ppm"
    ab.write_ppm(ours, ref.srgb_bytes(averages))
    ref.write_ppm(theirs, averages)
    assert ours.read_bytes() == theirs.read_bytes()


@needs_ref
def test_unopenable_path_fails_with_the_reference_message(tmp_path):
    path = tmp_path / "missing_dir" / "image.ppm"
    with pytest.raises(OSError) as ours:
        ab.write_ppm(path, np.zeros((1, 2, 3), dtype=np.uint8))
    with pytest.raises(RuntimeError) as theirs:
        ref.write_ppm(path, np.zeros((1, 2, 3)))
    assert str(ours.value) == str(theirs.value) == f"cannot open '{path}' for writing"


@needs_ref
@pytest.mark.skipif(not os.path.exists("/dev/full"), reason="needs /dev/full")
@pytest.mark.parametrize("shape", [(1, 2), (256, 256)])
def test_failed_writes_report_like_the_reference(shape):
    # /dev/full accepts the open and fails every write: a small image fails on
    # close, a large one while its rows are written (ppm_test.cpp:135-172).
    h, w = shape
    with pytest.raises(OSError) as ours:
        ab.write_ppm("/dev/full", np.zeros((h, w, 3), dtype=np.uint8))
    with pytest.raises(RuntimeError) as theirs:
        ref.write_ppm("/dev/full", np.zeros((h, w, 3)))
    assert str(ours.value) == str(theirs.value)
    stream_message = "failed to write PPM image"
    assert (stream_message in str(ours.value)) == (h * w > 2)


def test_refused_writes_leave_the_target_alone(tmp_path):
    # A size the writer refuses fails before anything is opened; a directory in
    # the way of the file fails the open and is left as it was.
    path = tmp_path / "image.ppm"
    with pytest.raises(ValueError, match="invalid image size 0x1"):
        ab.write_ppm(path, np.zeros((1, 0, 3), dtype=np.uint8))
    assert not path.exists()
    (tmp_path / "dir.ppm").mkdir()
    with pytest.raises(OSError, match="cannot open"):
        ab.write_ppm(tmp_path / "dir.ppm", np.zeros((1, 1, 3), dtype=np.uint8))
    assert (tmp_path / "dir.ppm").is_dir()


def test_invalid_shapes_are_refused():
    with pytest.raises(ValueError):
        ab.write_ppm("unused.ppm", np.zeros((2, 2), dtype=np.uint8))
