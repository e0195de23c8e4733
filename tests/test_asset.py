"""Asset builder and validator of libnxg_b200.so against the reference
(asset.cpp:229-362) -- host code, no GPU."""
import hashlib

import numpy as np
import pytest

from nanoxgen_b200 import fixtures
from nanoxgen_b200.asset import Asset, build_asset, recompute_hash, validate_asset

def _inputs():
    return [("unit", fixtures.reference_unit_fixture()), ("area", fixtures.reference_area_fixture()),
            ("benchmark", fixtures.reference_benchmark_fixture()),
            ("plain_sphere", fixtures.plain_sphere().build_input)]


@pytest.mark.parametrize("name,src", _inputs())
def test_builder_byte_identical_to_reference(nxg_lib, reference, name, src):
    mine = build_asset(src).buffer
    theirs = reference.build_asset(src)
    assert mine.size == theirs.size
    assert np.array_equal(mine, theirs)


def test_stencil_slots_equal_reference_patch(nxg_lib, reference):
    from helpers import patch_stencil
    src = fixtures.plain_sphere().build_input
    assert np.array_equal(build_asset(src, stencil_slots=4).buffer, patch_stencil(reference.build_asset(src), 4))


def test_builder_pinned_against_golden(nxg_lib):
    g = np.load(__file__.replace("test_asset.py", "golden/plain_sphere.npz"))
    assert np.array_equal(build_asset(fixtures.plain_sphere().build_input, 4).buffer, g["asset"])


def test_builder_workers_do_not_change_bytes(nxg_lib):
    w = fixtures.large_sphere(strands=1000, guides=256, n_lon=60, n_rings=41)
    a = build_asset(w.build_input, 8, workers=1).buffer
    b = build_asset(w.build_input, 8, workers=7).buffer
    assert np.array_equal(a, b)


def _corruptions(blob):
    out = []
    b = blob.copy(); b[-1] ^= 1; out.append(("last byte", b))                      # test_main.cpp:61-63
    b = blob.copy(); b[0] ^= 1; out.append(("magic", b))
    b = blob.copy(); b[8] = 9; out.append(("version", b))
    b = blob.copy(); b[48:52] = np.frombuffer(np.uint32(4).tobytes(), np.uint8); out.append(("stencil size", b))
    b = blob.copy(); b[16:24] = np.frombuffer(np.uint64(blob.size + 1).tobytes(), np.uint8); out.append(("byte size", b))
    b = blob.copy(); b[56:64] = np.frombuffer(np.uint64(blob.size).tobytes(), np.uint8); out.append(("positions off", b))
    b = blob[:100].copy(); out.append(("truncated", b))
    return out


def test_validator_messages_match_reference(nxg_lib, reference):
    blob = build_asset(fixtures.reference_unit_fixture()).buffer
    assert validate_asset(blob) == "" == reference.validate_asset(blob)
    for what, bad in _corruptions(blob):
        assert validate_asset(bad) == reference.validate_asset(bad) != "", what
    # a rehashed triangle index out of range (asset.cpp:326-331)
    bad = blob.copy()
    off = int(bad[80:88].view(np.uint64)[0])
    bad[off:off + 4] = np.frombuffer(np.uint32(99).tobytes(), np.uint8)
    recompute_hash(bad)
    assert validate_asset(bad) == reference.validate_asset(bad) == "triangle index out of bounds"


def test_validator_rejects_out_of_range_stencil_and_alias(nxg_lib):
    """Additions over the reference validator: indices a kernel would follow."""
    blob = build_asset(fixtures.reference_unit_fixture()).buffer
    st = blob.copy()
    off = int(st[112:120].view(np.uint64)[0])
    st[off:off + 4] = np.frombuffer(np.uint32(5).tobytes(), np.uint8)
    recompute_hash(st)
    assert validate_asset(st) == "guide stencil index out of bounds"
    al = blob.copy()
    off = int(al[88:96].view(np.uint64)[0])
    al[off + 4:off + 8] = np.frombuffer(np.uint32(3).tobytes(), np.uint8)
    recompute_hash(al)
    assert validate_asset(al) == "alias table index out of bounds"


def test_builder_input_errors(nxg_lib):
    src = fixtures.reference_unit_fixture()
    bad = fixtures.reference_unit_fixture()
    bad.triangles = np.array([[0, 1, 7]], np.uint32)
    with pytest.raises(ValueError, match="triangle index out of bounds"):
        build_asset(bad)
    bad = fixtures.reference_unit_fixture()
    bad.positions = np.zeros((3, 3), np.float32)
    with pytest.raises(ValueError, match="zero total area"):
        build_asset(bad)
    bad = fixtures.reference_unit_fixture()
    bad.guides.cv_counts = np.array([1], np.uint32)
    bad.guides.cvs = bad.guides.cvs[:1]
    with pytest.raises(ValueError, match="2..65535 CVs"):
        build_asset(bad)
    assert build_asset(src).nbytes > 0


def test_asset_save_load_round_trip(nxg_lib, tmp_path):
    a = build_asset(fixtures.reference_unit_fixture())
    path = str(tmp_path / "unit.nxg")
    a.save(path)
    from nanoxgen_b200.asset import load_asset
    assert np.array_equal(load_asset(path).buffer, a.buffer)
    with open(path, "r+b") as fh:
        fh.seek(-1, 2)
        last = fh.read(1)
        fh.seek(-1, 2)
        fh.write(bytes([last[0] ^ 1]))
    with pytest.raises(ValueError, match="content hash mismatch"):
        load_asset(path)
    assert hashlib.sha256(a.bytes()).hexdigest()
    assert Asset(a.bytes()).nbytes == a.nbytes


def test_device_stencil_entry_rejects_bad_arguments(nxg_lib):
    """nxg_build_stencils_device checks its arguments before any CUDA call."""
    from nanoxgen_b200._abi import ERRORS
    f = nxg_lib.nxg_build_stencils_device
    p = 256  # never dereferenced: every call below fails its argument check
    assert f(p, 3, p, 1, p, p, 1, 9, p, None) == ERRORS["InvalidArgument"]      # stencil_slots > 8
    assert f(None, 3, p, 1, p, p, 1, 8, p, None) == ERRORS["InvalidArgument"]   # NULL positions
    assert f(p, 3, p, 0, p, p, 1, 8, p, None) == ERRORS["InvalidArgument"]      # no triangles
    assert f(p, 3, p, 1, p, p, 0, 8, p, None) == ERRORS["InvalidArgument"]      # no guides
    assert f(p, 3, p, 1, p, p, 1, 8, p + 4, None) == ERRORS["MisalignedOutput"]  # stencil not 16-byte aligned


def test_device_build_without_a_device_fails_loudly(nxg_lib):
    """With no usable CUDA device the device build raises with the CUDA error
    text instead of falling back to the host search."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from nanoxgen_b200.asset import build_asset_device
    with pytest.raises(ValueError, match="device stencil search"):
        build_asset_device(fixtures.reference_unit_fixture(), 8)
