"""nxg_generate_packed_static_scratch: generation for callers that cannot
allocate device memory (a plugin whose host application owns every
allocation and its budget, or a frame loop where cudaMalloc would
synchronise the device).  The library then uses its own fixed 4 MiB device
scratch instead of a caller workspace.

Collected last on purpose (file name), so that a failure here cannot hide
any other test; it passes on its own in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

from helpers import max_position_error

pytestmark = pytest.mark.gpu


def test_static_scratch_matches_workspace_path_on_two_calls(cuda, nxg_lib, oracle):
    import torch

    from nanoxgen_b200 import _abi, fixtures
    from nanoxgen_b200._abi import LaunchConfig, lib
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import DeviceAsset, allocate_outputs, generate_packed, packed_output_descriptor

    w = fixtures.plain_sphere()
    asset = build_asset(w.build_input, w.stencil_slots)
    dasset = DeviceAsset(asset, cuda)
    params = w.params
    P = int(params.cvs_per_strand)
    need = int(lib().nxg_packed_workspace_size(ctypes.byref(dasset.desc), ctypes.byref(params), params.strand_count))
    assert need <= _abi.STATIC_SCRATCH_BYTES

    reference = generate_packed(dasset, params, 1.5)          # caller-workspace entry point
    torch.cuda.synchronize()
    ref_points = reference.points.cpu().numpy()
    ref_roots = reference.roots.cpu().numpy()
    ref_counts = reference.point_counts.cpu().numpy()
    tol = 1e-5 * asset.bbox_diagonal()
    orc_points, orc_roots, _, orc_counts = oracle.generate(asset.buffer, params, 1.5, threads=8)

    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):                                      # the scratch keeps the last call's contents
        points, roots, uvs, counts = allocate_outputs(params.strand_count, P, cuda)
        points.fill_(float("nan"))
        out = packed_output_descriptor(points, roots, uvs, counts, 1.5)
        code = lib().nxg_generate_packed_static_scratch(ctypes.byref(dasset.desc), None, ctypes.byref(params),
                                                        ctypes.byref(out), ctypes.byref(LaunchConfig(128)), stream)
        assert code == 0, _abi.ERROR_BY_CODE.get(code)
        torch.cuda.synchronize()
        got = points.cpu().numpy()
        assert np.isfinite(got).all(), call
        assert max_position_error(got, ref_points) <= tol, call
        assert float(np.abs(got[:, 3] - ref_points[:, 3]).max()) <= tol, call
        assert np.array_equal(roots.cpu().numpy(), ref_roots) and np.array_equal(counts.cpu().numpy(), ref_counts)
        # and against the oracle directly: roots bit-exact, positions within 1e-5 x diagonal
        assert roots.cpu().numpy().tobytes() == orc_roots.tobytes(), call
        assert np.array_equal(counts.cpu().numpy().view(np.uint32), orc_counts), call
        assert max_position_error(got, orc_points) <= tol, call


def test_static_scratch_rejects_requests_beyond_its_size(cuda, nxg_lib):
    """A request needing more than NXG_STATIC_SCRATCH_BYTES fails cleanly
    before any device work (the output is never written)."""
    import torch

    from nanoxgen_b200 import _abi, fixtures
    from nanoxgen_b200._abi import LaunchConfig, lib
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import DeviceAsset, packed_output_descriptor

    w = fixtures.plain_sphere()
    dasset = DeviceAsset(build_asset(w.build_input, w.stencil_slots), cuda)
    params = w.params.copy(strand_count=2_000_000, cvs_per_strand=2)
    points = torch.zeros((params.strand_count * 2, 4), device=cuda)
    out = packed_output_descriptor(points)
    code = lib().nxg_generate_packed_static_scratch(ctypes.byref(dasset.desc), None, ctypes.byref(params),
                                                    ctypes.byref(out), ctypes.byref(LaunchConfig(128)), None)
    assert code == _abi.ERRORS["StaticScratchLimit"]
    assert b"static scratch" in lib().nxg_error_message(code)
    torch.cuda.synchronize()
    assert float(points.abs().max()) == 0.0
