"""The device check of the curve cache (nxg_curve_cache_validate_device)
against the reference's validate_curve_cache: the same message for every
corruption of tests/test_curve_cache.py (header failures are found on the
host copy of the header and raised; element failures in one device pass,
the first in the reference's order), except the content hash, which the
device does not recompute; the point-count sum and the bit checksum equal
the host's on a large cache."""
import numpy as np
import pytest

from test_curve_cache import CORRUPTIONS, aligned_copy, corrupted, random_cache, reference_vector

pytestmark = pytest.mark.gpu


def _device_message(blob):
    from nanoxgen_b200.curve_cache import DeviceCurveCache
    d = DeviceCurveCache(blob)
    try:
        d.validate()
    except ValueError as header_failure:
        return str(header_failure), None
    return d.outcome()[0], d


@pytest.mark.parametrize("name", [c[0] for c in CORRUPTIONS])
def test_device_messages_match_reference(cuda, nxg_lib, reference, name):
    blob = corrupted(name)
    message, _ = _device_message(blob)
    expected = reference.curve_cache_validate(blob)
    if name == "content hash":
        assert expected == "curve-cache content hash mismatch" and message == ""
    else:
        assert message == expected


def test_reference_vector_on_device(cuda, nxg_lib):
    from nanoxgen_b200.curve_cache import build_curve_cache, point_checksum
    blob = build_curve_cache(**reference_vector())
    message, d = _device_message(blob)
    _, point_sum, checksum = d.outcome()
    assert (message, point_sum, checksum) == ("", 5, point_checksum(blob))


def test_large_cache_sum_and_checksum(cuda, nxg_lib):
    # 200,000 strands of 2..39 CVs (about 4M points) with two motion samples
    # and every optional section: the device's sum and checksum are the
    # host's; then one NaN near the end and one negative radius earlier.
    from nanoxgen_b200.curve_cache import build_curve_cache, header, point_checksum
    from test_curve_cache import _point
    rng = np.random.default_rng(99)
    blob = aligned_copy(build_curve_cache(**random_cache(rng, strands=200_000, samples=2)))
    message, d = _device_message(blob)
    _, point_sum, checksum = d.outcome()
    h = header(blob)
    assert message == "" and point_sum == h.point_count and checksum == point_checksum(blob)
    n = h.point_count
    bad = _point(n - 3, 0, np.nan)(_point(n // 2, 3, -1.0)(blob))
    assert _device_message(bad)[0] == "curve cache contains an invalid point or radius"
