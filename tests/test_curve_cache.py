"""The curve cache's host side against the reference (src/curve_cache.cpp
compiled into oracle/_ref): blobs byte-identical to build_curve_cache, the
same build errors, and validate_curve_cache's message for every check,
including which failure is reported first when several are present.

The corruption cases are shared with tests/test_curve_cache_gpu.py, which
holds the device check to the same messages."""
import ctypes

import numpy as np
import pytest

from nanoxgen_b200.asset import aligned_empty

HAS_TEXCOORDS, HAS_PATCH, HAS_FACE, HAS_IDS, HAS_MOTION = 1, 2, 4, 8, 16


def reference_vector():
    """The reference's own fixture (tests/test_main.cpp:617-634)."""
    counts = [2, 3]
    pts = [[0, 0, 0, 0.01], [0, 1, 0, 0.005], [1, 0, 0, 0.02], [1, 1, 0, 0.01], [1, 2, 0, 0.002]]
    return dict(point_counts=counts, points=pts, texcoords=[[0, 0], [0, 1], [1, 0], [1, 0.5], [1, 1]],
                patch_uvs=[[0.2, 0.3], [0.7, 0.8]], face_uvs=[[0.1, 0.2], [0.6, 0.7]], face_ids=[3, 9],
                motion_times=[0.5], motion_points=[[p[0] + 0.25, p[1], p[2]] for p in pts])


def random_cache(rng, strands=300, samples=2, sections=HAS_TEXCOORDS | HAS_PATCH | HAS_FACE | HAS_IDS | HAS_MOTION):
    counts = rng.integers(2, 40, strands).astype(np.uint32)
    n = int(counts.sum())
    pts = rng.normal(size=(n, 4)).astype(np.float32)
    pts[:, 3] = np.abs(pts[:, 3]) * 0.01
    d = dict(point_counts=counts, points=pts)
    if sections & HAS_TEXCOORDS:
        d["texcoords"] = rng.random((n, 2), np.float32)
    if sections & HAS_PATCH:
        d["patch_uvs"] = rng.random((strands, 2), np.float32)
    if sections & HAS_FACE:
        d["face_uvs"] = rng.random((strands, 2), np.float32)
    if sections & HAS_IDS:
        d["face_ids"] = rng.integers(0, 1000, strands).astype(np.uint32)
    if sections & HAS_MOTION and samples:
        d["motion_times"] = np.sort(rng.random(samples).astype(np.float32)) + np.arange(samples, dtype=np.float32)
        d["motion_points"] = rng.normal(size=(samples * n, 3)).astype(np.float32)
    return d


def aligned_copy(blob, misalign=0):
    out = aligned_empty(blob.size + misalign)[misalign:]
    out[:] = blob
    return out


def header_of(blob):
    from nanoxgen_b200._abi import CurveCacheHeader
    return CurveCacheHeader.from_buffer(blob)


def rehash(blob):
    from nanoxgen_b200.curve_cache import content_hash
    header_of(blob).content_hash = content_hash(blob[128:])


def section(blob, offset_field, dtype):
    off = getattr(header_of(blob), offset_field)
    return blob[off:].view(dtype) if off % np.dtype(dtype).itemsize == 0 else None


# (name, corrupt(blob) -> blob).  Element corruptions rehash, so the checks
# after the content hash are reached.
def _set(field, value):
    def f(b):
        setattr(header_of(b), field, value(getattr(header_of(b), field)))
        return b
    return f


def _element(offset_field, dtype, index, value, width=1):
    def f(b):
        off = getattr(header_of(b), offset_field)
        arr = b[off:].view(dtype)
        arr[index * width:(index + 1) * width] = value if np.ndim(value) else [value] * width
        rehash(b)
        return b
    return f


def _chain(*fs):
    def f(b):
        for g in fs:
            b = g(b)
        return b
    return f


def _point(i, k, v):
    def f(b):
        arr = section(b, "points_offset", np.float32)
        arr[4 * i + k] = v
        rehash(b)
        return b
    return f


def _flat(field, dtype, i, v):
    def f(b):
        arr = section(b, field, dtype)
        arr[i] = v
        rehash(b)
        return b
    return f


CORRUPTIONS = [
    ("valid", lambda b: b),
    ("bad magic", _set("magic", lambda v: v ^ 1)),
    ("bad version", _set("version_major", lambda v: 2)),
    ("unknown flags", _set("flags", lambda v: v | 128)),
    ("size mismatch", _set("byte_size", lambda v: v + 16)),
    ("no strands", _set("strand_count", lambda v: 0)),
    ("motion flag without samples", _set("flags", lambda v: v & ~HAS_MOTION)),
    ("points out of bounds", _set("points_offset", lambda v: v + 4)),
    ("texcoords past the end", _set("texcoords_offset", lambda v: 1 << 40)),
    ("content hash", lambda b: (b.__setitem__(-1, b[-1] ^ 1), b)[1]),
    ("short curve", _flat("point_counts_offset", np.uint32, 7, 1)),
    ("count sum", _flat("point_counts_offset", np.uint32, 3, 60)),
    ("nan x", _point(11, 0, np.nan)),
    ("inf z", _point(12, 2, np.inf)),
    ("negative radius", _point(13, 3, -1e-3)),
    ("nan texcoord", _flat("texcoords_offset", np.float32, 2 * 20 + 1, np.nan)),
    ("texcoord before point", _chain(_flat("texcoords_offset", np.float32, 2 * 5, np.nan), _point(9, 1, np.nan))),
    ("point before texcoord", _chain(_flat("texcoords_offset", np.float32, 2 * 9, np.nan), _point(9, 1, np.nan))),
    ("motion times not increasing", _flat("motion_times_offset", np.float32, 1, -5.0)),
    ("nan motion time", _flat("motion_times_offset", np.float32, 0, np.nan)),
    ("nan motion point", _flat("motion_points_offset", np.float32, 3 * 100 + 2, np.nan)),
    ("points before motion", _chain(_flat("motion_points_offset", np.float32, 0, np.nan), _point(30, 3, -1.0))),
    ("nan patch uv", _flat("patch_uvs_offset", np.float32, 2 * 40, np.nan)),
    ("nan face uv", _flat("face_uvs_offset", np.float32, 2 * 41 + 1, np.inf)),
    ("face before patch", _chain(_flat("patch_uvs_offset", np.float32, 2 * 50, np.nan),
                                 _flat("face_uvs_offset", np.float32, 2 * 49, np.nan))),
    ("patch before face at one strand", _chain(_flat("patch_uvs_offset", np.float32, 2 * 49, np.nan),
                                               _flat("face_uvs_offset", np.float32, 2 * 49, np.nan))),
    ("motion before uvs", _chain(_flat("patch_uvs_offset", np.float32, 0, np.nan),
                                 _flat("motion_points_offset", np.float32, 7, np.nan))),
]


def corrupted(name):
    rng = np.random.default_rng(5)
    blob = aligned_copy(__import__("nanoxgen_b200.curve_cache", fromlist=["x"]).build_curve_cache(
        **random_cache(rng)))
    return dict(CORRUPTIONS)[name](blob)


def test_reference_vector_is_byte_identical(nxg_lib, reference):
    from nanoxgen_b200.curve_cache import build_curve_cache, header, validate_curve_cache
    mine = build_curve_cache(**reference_vector())
    theirs = reference.curve_cache_build(**reference_vector())
    assert mine.tobytes() == theirs.tobytes()
    h = header(mine)
    assert (h.strand_count, h.point_count, h.motion_sample_count) == (2, 5, 1)
    assert validate_curve_cache(mine) == ""
    bad = aligned_copy(mine)
    bad[-1] ^= 1
    assert validate_curve_cache(bad) == reference.curve_cache_validate(bad) == "curve-cache content hash mismatch"


@pytest.mark.parametrize("sections", [0, HAS_TEXCOORDS, HAS_PATCH | HAS_IDS, HAS_MOTION, 31])
def test_random_caches_are_byte_identical(nxg_lib, reference, sections):
    from nanoxgen_b200.curve_cache import build_curve_cache, validate_curve_cache
    rng = np.random.default_rng(sections + 1)
    d = random_cache(rng, strands=257, samples=3, sections=sections)
    mine = build_curve_cache(**d)
    assert mine.tobytes() == reference.curve_cache_build(**d).tobytes()
    assert validate_curve_cache(mine) == ""


def test_build_errors_match_reference(nxg_lib, reference):
    from nanoxgen_b200.curve_cache import build_curve_cache
    pts = [[0, 0, 0, 0.1]] * 5
    cases = [
        dict(point_counts=[], points=[]),
        dict(point_counts=[1, 4], points=pts),
        dict(point_counts=[2, 2], points=pts),
        dict(point_counts=[2, 3], points=pts, texcoords=[[0, 0]] * 4),
        dict(point_counts=[2, 3], points=pts, patch_uvs=[[0, 0]]),
        dict(point_counts=[2, 3], points=pts, face_uvs=[[0, 0]] * 3),
        dict(point_counts=[2, 3], points=pts, face_ids=[1]),
        dict(point_counts=[2, 3], points=pts, motion_times=[0.1]),
        dict(point_counts=[2, 3], points=pts, motion_times=[0.1], motion_points=[[0, 0, 0]] * 4),
        dict(point_counts=[2, 3], points=pts, motion_times=[0.2, 0.1], motion_points=[[0, 0, 0]] * 10),
        dict(point_counts=[2, 3], points=pts, motion_times=[np.nan], motion_points=[[0, 0, 0]] * 5),
    ]
    for d in cases:
        with pytest.raises(ValueError) as theirs:
            reference.curve_cache_build(**d)
        with pytest.raises(ValueError) as mine:
            build_curve_cache(**d)
        assert str(mine.value) == str(theirs.value), d


@pytest.mark.parametrize("name", [c[0] for c in CORRUPTIONS])
def test_validation_messages_match_reference(nxg_lib, reference, name):
    from nanoxgen_b200.curve_cache import validate_curve_cache
    blob = corrupted(name)
    expected = reference.curve_cache_validate(blob)
    assert validate_curve_cache(blob) == expected
    if name != "valid":
        assert expected != ""


def test_small_and_misaligned_blobs(nxg_lib, reference):
    from nanoxgen_b200.curve_cache import validate_curve_cache
    blob = corrupted("valid")
    small = aligned_copy(blob[:100])
    assert validate_curve_cache(small) == reference.curve_cache_validate(small)
    shifted = aligned_copy(blob, misalign=16)
    assert validate_curve_cache(shifted) == reference.curve_cache_validate(shifted) == \
        "curve-cache base is not 64-byte aligned"


def test_point_checksum_restated(nxg_lib):
    # Per point, SplitMix64's finaliser of (xy ^ i * G) + zw * K (xy, zw its
    # two 64-bit words), summed modulo 2^64, restated in numpy.
    from nanoxgen_b200.curve_cache import header, point_checksum
    blob = corrupted("valid")
    h = header(blob)
    words = blob[h.points_offset:h.points_offset + 16 * h.point_count].view(np.uint64).reshape(-1, 2)
    with np.errstate(over="ignore"):
        index = np.arange(words.shape[0], dtype=np.uint64)
        z = (words[:, 0] ^ (index * np.uint64(0x9e3779b97f4a7c15))) + words[:, 1] * np.uint64(0xd6e8feb86659fd93)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
        z = z ^ (z >> np.uint64(31))
        total = int(z.sum(dtype=np.uint64))
    assert point_checksum(blob) == total
