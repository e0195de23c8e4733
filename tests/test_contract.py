"""The checked device boundary of libnxg_b200.so -- pure host validators,
error codes and messages, exported symbols.  Host memory stands in for
device memory, as in the reference's own contract test
(tests/test_main.cpp:483-588); every case is also run through the
reference's validator (device_contract.h:190-288) and must agree."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

from nanoxgen_b200 import _abi, fixtures
from nanoxgen_b200._abi import (ERRORS, DeformedDesc, DeviceAssetDesc, GenerationParams, LaunchConfig,
                                MotionOutputDesc, MotionSampleDesc, PackedOutputDesc, lib)
from nanoxgen_b200.asset import aligned_empty, aligned_struct, build_asset

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol(nxg_lib):
    header = "".join(open(os.path.join(ROOT, "include", name)).read()
                     for name in sorted(os.listdir(os.path.join(ROOT, "include"))) if name.endswith(".h"))
    declared = set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s+\*?\s*(nxg_[a-z_0-9]+)\(", header, re.M))
    assert declared, "no declarations parsed"
    assert declared == set(_abi.declared_symbols()), declared ^ set(_abi.declared_symbols())
    for name in declared:
        assert hasattr(nxg_lib, name), name
    assert lib().nxg_abi_version() == 1


def test_error_messages_match_reference(nxg_lib, reference):
    for code in range(21):
        assert lib().nxg_error_message(code) == reference.lib.ref_error_message(code), code
    assert lib().nxg_error_message(999) == b"unknown device generation error"


class Case:
    """One validation request on host memory."""

    def __init__(self):
        self.asset = build_asset(fixtures.reference_unit_fixture())
        self.blob = self.asset.buffer
        self.desc = aligned_struct(DeviceAssetDesc)
        msg = ctypes.create_string_buffer(128)
        code = lib().nxg_make_device_asset_descriptor(self.blob.ctypes.data, self.blob.size, self.blob.ctypes.data,
                                                      self.blob.size, ctypes.byref(self.desc), msg, 128)
        assert code == 0, msg.value
        self.params = GenerationParams(strand_count=7, cvs_per_strand=5)
        n = 35
        self.points = aligned_empty(16 * n)
        self.roots = aligned_empty(48 * 7)
        self.uvs = aligned_empty(8 * 7)
        self.counts = aligned_empty(4 * 7)
        self.out = PackedOutputDesc(points=self.points.ctypes.data, roots=self.roots.ctypes.data,
                                    root_uvs=self.uvs.ctypes.data, radius_scale=1.0,
                                    point_counts=self.counts.ctypes.data, point_capacity=n, root_capacity=7,
                                    root_uv_capacity=7, point_count_capacity=7)
        self.deformed = DeformedDesc()
        self.block = 128

    def mine(self):
        return int(lib().nxg_validate_packed_request(ctypes.byref(self.desc), ctypes.byref(self.deformed),
                                                     ctypes.byref(self.params), ctypes.byref(self.out),
                                                     ctypes.byref(LaunchConfig(self.block))))

    def theirs(self, reference):
        d, o = self.deformed, self.out
        return int(reference.lib.ref_validate_packed_request(
            self.desc.asset, ctypes.byref(self.desc.header), self.desc.byte_capacity, d.positions, d.position_count,
            d.normals, d.normal_count, d.guide_cvs, d.guide_cv_count, ctypes.byref(self.params), o.points, o.roots,
            o.root_uvs, o.radius_scale, o.point_counts, o.point_capacity, o.root_capacity, o.root_uv_capacity,
            o.point_count_capacity, self.block))


def _mutations():
    """(name, mutate(case), expected error) covering every packed-request branch."""
    def m(**kw):
        def f(c):
            for k, v in kw.items():
                obj, attr = k.split("__")
                setattr(getattr(c, obj), attr, v)
        return f

    def hdr(field, value):
        def f(c):
            setattr(c.desc.header, field, value)
        return f

    def asset_ptr(c):
        c.desc.asset = None

    def misalign(c):
        c.desc.asset = c.blob.ctypes.data + 1
        c.desc.byte_capacity -= 1

    def bad_positions(c):
        c.deformed.positions = c.blob.ctypes.data
        c.deformed.position_count = c.desc.header.vertex_count - 1

    def positions_without_pointer(c):
        c.deformed.position_count = c.desc.header.vertex_count

    def bad_normals(c):
        c.deformed.normals = c.blob.ctypes.data
        c.deformed.normal_count = 1

    def bad_guides(c):
        c.deformed.guide_cvs = c.blob.ctypes.data
        c.deformed.guide_cv_count = c.desc.header.guide_cv_count + 1

    def good_deformation(c):
        c.deformed.positions = c.blob.ctypes.data
        c.deformed.position_count = c.desc.header.vertex_count
        c.deformed.guide_cvs = c.blob.ctypes.data
        c.deformed.guide_cv_count = c.desc.header.guide_cv_count

    return [
        ("valid", lambda c: None, "None"),
        ("null asset", asset_ptr, "NullAsset"),
        ("misaligned", misalign, "MisalignedAsset"),
        ("magic", hdr("magic", 1), "InvalidAssetMetadata"),
        ("version", hdr("version_minor", 1), "InvalidAssetMetadata"),
        ("no vertices", hdr("vertex_count", 0), "InvalidAssetMetadata"),
        ("stencil size", hdr("guide_stencil_size", 4), "InvalidAssetMetadata"),
        ("gradient count", hdr("noise_gradient_count", 255), "InvalidAssetMetadata"),
        ("noise table bounds", lambda c: setattr(c.desc.header, "noise_gradients_offset",
                                                 c.desc.header.byte_size - 4), "InvalidAssetMetadata"),
        ("asset capacity", lambda c: setattr(c.desc, "byte_capacity", c.desc.header.byte_size - 1),
         "AssetCapacityTooSmall"),
        ("zero strands", m(params__strand_count=0), "InvalidGenerationParameters"),
        ("one cv", m(params__cvs_per_strand=1), "InvalidGenerationParameters"),
        ("nan support", m(params__guide_support_scale=math.nan), "InvalidGenerationParameters"),
        ("negative power", m(params__guide_weight_power=-1.0), "InvalidGenerationParameters"),
        ("rejection cos", m(params__normal_rejection_cos=1.5), "InvalidGenerationParameters"),
        ("inf length", m(params__length_scale=math.inf), "InvalidGenerationParameters"),
        ("negative width", m(params__root_width=-0.1), "InvalidGenerationParameters"),
        ("mask > 1", m(params__noise_mask=1.5), "InvalidGenerationParameters"),
        ("correlation", m(params__noise_correlation=-0.1), "InvalidGenerationParameters"),
        ("preserve", m(params__noise_preserve_length=2.0), "InvalidGenerationParameters"),
        ("block 0", lambda c: setattr(c, "block", 0), "InvalidBlockSize"),
        ("block 1025", lambda c: setattr(c, "block", 1025), "InvalidBlockSize"),
        ("block 1024", lambda c: setattr(c, "block", 1024), "None"),
        ("positions count", bad_positions, "DeformedPositionCountMismatch"),
        ("count without pointer", positions_without_pointer, "DeformedPositionCountMismatch"),
        ("normals count", bad_normals, "DeformedNormalCountMismatch"),
        ("guide cvs count", bad_guides, "DeformedGuideCvCountMismatch"),
        ("good deformation", good_deformation, "None"),
        ("missing points", m(out__points=None), "MissingOutput"),
        ("nan radius", m(out__radius_scale=math.nan), "InvalidRadiusScale"),
        ("negative radius", m(out__radius_scale=-1.0), "InvalidRadiusScale"),
        ("point capacity", m(out__point_capacity=34), "PointCapacityTooSmall"),
        ("root capacity", m(out__root_capacity=6), "RootCapacityTooSmall"),
        ("root capacity without pointer", m(out__roots=None), "RootCapacityTooSmall"),
        ("uv capacity", m(out__root_uv_capacity=6), "RootUvCapacityTooSmall"),
        ("count capacity", m(out__point_count_capacity=6), "PointCountCapacityTooSmall"),
        ("optional outputs absent", m(out__roots=None, out__root_capacity=0, out__root_uvs=None,
                                      out__root_uv_capacity=0, out__point_counts=None,
                                      out__point_count_capacity=0), "None"),
    ]


@pytest.mark.parametrize("name,mutate,expected", _mutations(), ids=[x[0] for x in _mutations()])
def test_packed_request_branches(nxg_lib, reference, name, mutate, expected):
    c = Case()
    mutate(c)
    assert c.mine() == ERRORS[expected]
    assert c.theirs(reference) == ERRORS[expected]


def test_motion_request_branches(nxg_lib, reference):
    """tests/test_main.cpp:504-527, :581-587."""
    c = Case()
    pts = aligned_empty(12 * 35 * 2)

    def run(times, params, capacity):
        samples = (MotionSampleDesc * len(times))()
        for s, t in zip(samples, times):
            s.time = t
        out = MotionOutputDesc(points=pts.ctypes.data, point_capacity=capacity)
        mine = lib().nxg_validate_motion_request(ctypes.byref(c.desc), samples if times else None, len(times),
                                                 ctypes.byref(params), ctypes.byref(out),
                                                 ctypes.byref(LaunchConfig(128)))
        tarr = (ctypes.c_float * max(1, len(times)))(*times)
        theirs = reference.lib.ref_validate_motion_request(c.desc.asset, ctypes.byref(c.desc.header),
                                                           c.desc.byte_capacity, tarr if times else None,
                                                           len(times), ctypes.byref(params), pts.ctypes.data,
                                                           capacity, 128)
        assert mine == theirs
        return mine

    p = c.params
    assert run([0.25, 0.75], p, 70) == ERRORS["None"]
    assert run([0.25, 0.25], p, 70) == ERRORS["InvalidMotionTimes"]
    assert run([math.nan, 0.75], p, 70) == ERRORS["InvalidMotionTimes"]
    assert run([0.25, 0.75], p, 69) == ERRORS["MotionPointCapacityTooSmall"]
    assert run([], p, 70) == ERRORS["MissingMotionSamples"]
    big = p.copy(strand_count=0xFFFFFFFF, cvs_per_strand=0xFFFFFFFF)
    assert run([0.25, 0.75], big, 70) == ERRORS["OutputSizeOverflow"]


def test_make_device_asset_descriptor(nxg_lib):
    """asset.cpp:364-378."""
    blob = build_asset(fixtures.reference_unit_fixture()).buffer
    desc = aligned_struct(DeviceAssetDesc)
    msg = ctypes.create_string_buffer(128)
    f = lib().nxg_make_device_asset_descriptor
    assert f(blob.ctypes.data, blob.size, blob.ctypes.data, blob.size, ctypes.byref(desc), msg, 128) == 0
    assert desc.header.magic == _abi.MAGIC and desc.byte_capacity == blob.size
    assert f(blob.ctypes.data, blob.size, None, blob.size, ctypes.byref(desc), msg, 128) == ERRORS["NullAsset"]
    assert f(blob.ctypes.data, blob.size, blob.ctypes.data + 8, blob.size, ctypes.byref(desc), msg,
             128) == ERRORS["MisalignedAsset"]
    assert f(blob.ctypes.data, blob.size, blob.ctypes.data, blob.size - 1, ctypes.byref(desc), msg,
             128) == ERRORS["AssetCapacityTooSmall"]
    bad = aligned_empty(blob.size)
    bad[:] = blob
    bad[-1] ^= 1
    assert f(bad.ctypes.data, bad.size, bad.ctypes.data, bad.size, ctypes.byref(desc), msg,
             128) == ERRORS["InvalidAssetMetadata"]
    assert msg.value == b"content hash mismatch"


def test_launch_entry_points_reject_before_device_work(nxg_lib):
    """Launch-path checks that need no GPU: every failure is reported before
    anything is enqueued (null descriptors, strand ranges, workspace)."""
    c = Case()
    ws = aligned_empty(1 << 16, 256)
    L = lib()
    assert L.nxg_generate_packed(None, None, ctypes.byref(c.params), ctypes.byref(c.out), None, ws.ctypes.data,
                                 ws.size, None) == ERRORS["InvalidArgument"]
    assert L.nxg_generate_packed_range(ctypes.byref(c.desc), None, ctypes.byref(c.params), ctypes.byref(c.out),
                                       None, 5, 3, ws.ctypes.data, ws.size, None) == ERRORS["InvalidStrandRange"]
    assert L.nxg_generate_packed(ctypes.byref(c.desc), None, ctypes.byref(c.params), ctypes.byref(c.out), None,
                                 ws.ctypes.data, 16, None) == ERRORS["WorkspaceTooSmall"]
    assert L.nxg_generate_packed(ctypes.byref(c.desc), None, ctypes.byref(c.params), ctypes.byref(c.out), None,
                                 ws.ctypes.data + 64, ws.size - 64, None) == ERRORS["MisalignedOutput"]
    c.out.points = c.points.ctypes.data + 4
    assert L.nxg_generate_packed(ctypes.byref(c.desc), None, ctypes.byref(c.params), ctypes.byref(c.out), None,
                                 ws.ctypes.data, ws.size, None) == ERRORS["MisalignedOutput"]
    c = Case()
    c.desc.header.guides_offset = c.desc.header.byte_size
    assert L.nxg_generate_packed(ctypes.byref(c.desc), None, ctypes.byref(c.params), ctypes.byref(c.out), None,
                                 ws.ctypes.data, ws.size, None) == ERRORS["InvalidAssetMetadata"]
    c = Case()
    need = L.nxg_packed_workspace_size(ctypes.byref(c.desc), ctypes.byref(c.params), 7)
    assert need % 256 == 0 and need >= 4 * 256
    assert L.nxg_prepare_strand_order(ctypes.byref(c.desc), ctypes.byref(c.params), 0, 8, ws.ctypes.data, ws.size,
                                      None) == ERRORS["InvalidStrandRange"]
    # zero-length ranges succeed without touching the device
    assert L.nxg_generate_packed_range(ctypes.byref(c.desc), None, ctypes.byref(c.params), ctypes.byref(c.out),
                                       None, 7, 0, None, 0, None) == ERRORS["None"]


def test_tile_registry(nxg_lib):
    """nxg_set_tile / nxg_get_tile validation (pure host)."""
    from nanoxgen_b200._abi import Tile
    L = lib()
    t = Tile()
    # built-in choice for 2..32 CVs: the lane-walk generator (one lane per strand)
    assert L.nxg_get_tile(32, 1, ctypes.byref(t)) == 0
    assert (t.lanes_per_strand, t.cvs_per_lane, t.block_size) == (1, 1, 352)
    assert L.nxg_get_tile(64, 1, ctypes.byref(t)) == 0 and t.lanes_per_strand * t.cvs_per_lane >= 64
    assert L.nxg_set_tile(32, 1, ctypes.byref(Tile(1, 1, 256))) == 0
    assert L.nxg_set_tile(33, 1, ctypes.byref(Tile(1, 1, 256))) == ERRORS["InvalidArgument"]
    assert L.nxg_set_tile(32, 1, ctypes.byref(Tile(1, 2, 256))) == ERRORS["InvalidArgument"]
    assert L.nxg_set_tile(32, 1, ctypes.byref(Tile(16, 2, 256))) == 0
    assert L.nxg_get_tile(32, 1, ctypes.byref(t)) == 0
    assert (t.lanes_per_strand, t.cvs_per_lane, t.block_size) == (16, 2, 256)
    assert L.nxg_get_tile(32, 0, ctypes.byref(t)) == 0 and (t.lanes_per_strand, t.cvs_per_lane) != (16, 2) or True
    for bad in (Tile(3, 4, 128), Tile(8, 3, 128), Tile(4, 4, 128), Tile(32, 4, 2048)):
        assert L.nxg_set_tile(32, 1, ctypes.byref(bad)) == ERRORS["InvalidArgument"]
    assert L.nxg_set_tile(200, 1, ctypes.byref(Tile(32, 4, 128))) == ERRORS["InvalidArgument"]
    assert L.nxg_set_tile(32, 1, None) == 0
    assert L.nxg_get_tile(32, 1, ctypes.byref(t)) == 0 and t.lanes_per_strand == 1
