"""Motion samples through the C ABI: nxg_generate_motion_packed (per-sample
float4 buffers) and nxg_generate_motion (the reference's sample-major Vec3
contract, device_contract.h:42-53), against the single-frame entry point and
the oracle's generate_packed_deformed_cpu restatement."""
import ctypes

import numpy as np
import pytest

from helpers import max_position_error

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def motion(cuda, nxg_lib):
    import torch

    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import DeformedGeometry, DeviceAsset
    w = fixtures.plain_sphere()
    asset = build_asset(w.build_input, w.stencil_slots)
    frames = fixtures.motion_frames(w.build_input, 5)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)
    geoms = [DeformedGeometry(dev(p), dev(n), dev(g)) for p, n, g in
             zip(frames.positions, frames.normals, frames.guide_cvs)]
    return w, asset, DeviceAsset(asset, cuda), frames, geoms


def test_motion_packed_matches_single_frames_and_oracle(motion, oracle):
    import torch

    from nanoxgen_b200.generator import generate_motion_packed, generate_packed
    w, asset, d, frames, geoms = motion
    outs = generate_motion_packed(d, w.params, geoms, frames.times, radius_scale=1.5)
    torch.cuda.synchronize()
    tol = 1e-5 * asset.bbox_diagonal()
    for i, (out, geom) in enumerate(zip(outs, geoms)):
        single = generate_packed(d, w.params, 1.5, geom)
        torch.cuda.synchronize()
        assert torch.equal(out.points, single.points), i             # same kernels, one order for all samples
        assert torch.equal(out.roots, single.roots)
        pts, roots, _, counts = oracle.generate(asset.buffer, w.params, 1.5, positions=frames.positions[i],
                                                normals=frames.normals[i], guide_cvs=frames.guide_cvs[i], threads=8)
        mine = out.points.cpu().numpy()
        assert max_position_error(mine, pts) <= tol, i
        got_roots = out.roots_numpy()
        assert np.array_equal(got_roots["triangle_index"], roots["triangle_index"])
        assert got_roots.tobytes() == roots.tobytes()
    # identities shared across samples: same triangles and barycentrics at every time
    r0 = outs[0].roots_numpy()
    for out in outs[1:]:
        r = out.roots_numpy()
        assert np.array_equal(r["triangle_index"], r0["triangle_index"])
        assert np.array_equal(r["barycentric"], r0["barycentric"])


def test_motion_vec3_contract(motion):
    import torch

    from nanoxgen_b200.generator import generate_motion, generate_motion_packed
    w, asset, d, frames, geoms = motion
    vec3 = generate_motion(d, w.params, geoms, frames.times)
    packed = generate_motion_packed(d, w.params, geoms, frames.times)
    torch.cuda.synchronize()
    for i, out in enumerate(packed):
        assert torch.equal(vec3[i], out.points[:, :3]), i


def test_motion_validation_codes(motion):
    from nanoxgen_b200._abi import ERRORS, NxgError
    from nanoxgen_b200.generator import generate_motion, generate_motion_packed
    w, asset, d, frames, geoms = motion
    with pytest.raises(NxgError) as e:
        generate_motion_packed(d, w.params, geoms[:2], [0.5, 0.5])
    assert e.value.code == ERRORS["InvalidMotionTimes"]
    with pytest.raises(NxgError) as e:
        generate_motion(d, w.params, geoms[:2], [0.0, float("nan")])
    assert e.value.code == ERRORS["InvalidMotionTimes"]
    with pytest.raises(NxgError) as e:
        generate_motion(d, w.params, [], [])
    assert e.value.code == ERRORS["MissingMotionSamples"]
    import torch
    small = torch.empty((2, w.params.strand_count * w.params.cvs_per_strand - 1, 3), device="cuda")
    with pytest.raises(NxgError) as e:
        generate_motion(d, w.params, geoms[:2], [0.0, 1.0], points=small)
    assert e.value.code == ERRORS["MotionPointCapacityTooSmall"]


def test_motion_in_one_graph(motion):
    """All samples captured as one CUDA graph and replayed."""
    import torch

    from nanoxgen_b200.generator import allocate_outputs, generate_motion_packed
    w, asset, d, frames, geoms = motion
    S, P = w.params.strand_count, w.params.cvs_per_strand
    eager = [o.points.clone() for o in generate_motion_packed(d, w.params, geoms, frames.times)]
    outputs = [allocate_outputs(S, P, "cuda") for _ in geoms]
    d.workspace(w.params, S)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        generate_motion_packed(d, w.params, geoms, frames.times, outputs=outputs, stream=s)
    for o in outputs:
        o[0].zero_()
    g.replay()
    torch.cuda.synchronize()
    for o, e in zip(outputs, eager):
        assert torch.equal(o[0], e)
