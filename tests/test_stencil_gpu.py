"""The asset build's all-pairs searches on the GPU (stencil.cu: the
per-triangle stencil, asset.cpp:252-269, and the automatic support radius's
nearest roots, asset.cpp:88-97) against the host builder (host.cpp), which
the CPU suite pins byte for byte to the reference's own build_asset and to
the golden plain-sphere blob."""
import numpy as np
import pytest
import torch

from nanoxgen_b200 import fixtures
from nanoxgen_b200.asset import AssetBuildInput, GuideSet, build_asset, build_asset_device
from nanoxgen_b200.generator import build_stencils

pytestmark = pytest.mark.gpu


def _ties_and_penalties() -> AssetBuildInput:
    """Every guide of the plain sphere twice (equal scores, ordered by guide
    index), every other copy with its root normal flipped (the 1e20 penalty),
    and two zero-area triangles (the (0, 1, 0) fallback face normal)."""
    src = fixtures.plain_sphere().build_input
    g = src.guides
    n = g.cv_counts.size
    counts = np.concatenate([g.cv_counts, g.cv_counts])
    cvs = np.concatenate([g.cvs, g.cvs])
    normals = np.concatenate([g.root_normals, g.root_normals])
    normals[1::2] *= -1.0
    guides = GuideSet(cv_counts=counts, cvs=cvs, root_normals=normals,
                      root_uvs=np.concatenate([g.root_uvs, g.root_uvs]),
                      triangles=np.concatenate([g.triangles, g.triangles]),
                      barycentrics=np.concatenate([g.barycentrics, g.barycentrics]),
                      support_radii=np.zeros(2 * n, np.float32))
    tris = np.concatenate([src.triangles, np.array([[0, 0, 1], [2, 2, 2]], np.uint32)])
    return AssetBuildInput(src.positions, tris, guides, src.normals, src.texcoords)


def _few_guides(count: int) -> AssetBuildInput:
    src = fixtures.plain_sphere().build_input
    g = src.guides
    cv = int(g.cv_counts[0])
    guides = GuideSet(cv_counts=g.cv_counts[:count], cvs=g.cvs[:count * cv], root_normals=g.root_normals[:count],
                      root_uvs=g.root_uvs[:count], triangles=g.triangles[:count],
                      barycentrics=g.barycentrics[:count], support_radii=g.support_radii[:count])
    return AssetBuildInput(src.positions, src.triangles, guides, src.normals, src.texcoords)


def _mixed_radii() -> AssetBuildInput:
    """Given support radii on some guides, automatic ones (0, negative, NaN)
    on the rest: only the automatic ones take the GPU's nearest-root search."""
    src = fixtures.plain_sphere().build_input
    g = src.guides
    radii = np.zeros(g.cv_counts.size, np.float32)
    radii[::3] = 0.05
    radii[1::7] = -1.0
    radii[2::11] = np.nan
    guides = GuideSet(cv_counts=g.cv_counts, cvs=g.cvs, root_normals=g.root_normals, root_uvs=g.root_uvs,
                      triangles=g.triangles, barycentrics=g.barycentrics, support_radii=radii)
    return AssetBuildInput(src.positions, src.triangles, guides, src.normals, src.texcoords)


def _inputs():
    return [("unit", fixtures.reference_unit_fixture()), ("area", fixtures.reference_area_fixture()),
            ("benchmark", fixtures.reference_benchmark_fixture()),
            ("plain_sphere", fixtures.plain_sphere().build_input),
            ("ties_and_penalties", _ties_and_penalties()), ("one_guide", _few_guides(1)),
            ("five_guides", _few_guides(5)), ("mixed_radii", _mixed_radii()),
            ("large_sphere", fixtures.large_sphere(strands=1000).build_input)]


@pytest.mark.parametrize("name,src", _inputs(), ids=[n for n, _ in _inputs()])
@pytest.mark.parametrize("slots", [8, 3])
def test_device_build_is_byte_identical(nxg_lib, name, src, slots):
    mine = build_asset_device(src, slots).buffer
    host = build_asset(src, slots).buffer
    assert mine.size == host.size
    assert np.array_equal(mine, host)


def test_device_build_matches_golden(nxg_lib):
    g = np.load(__file__.replace("test_stencil_gpu.py", "golden/plain_sphere.npz"))
    assert np.array_equal(build_asset_device(fixtures.plain_sphere().build_input, 4).buffer, g["asset"])


def test_device_build_on_a_torch_stream(nxg_lib):
    src = fixtures.plain_sphere().build_input
    s = torch.cuda.Stream()
    assert np.array_equal(build_asset_device(src, 8, stream=s).buffer, build_asset(src, 8).buffer)


def _device_inputs(src, asset):
    g = asset.guides()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return (dev(np.asarray(src.positions, np.float32)),
            dev(np.asarray(src.triangles, np.uint32).view(np.int32)),
            dev(g["root_position"].astype(np.float32)), dev(g["root_normal"].astype(np.float32)))


@pytest.mark.parametrize("slots", [0, 8, 1])
def test_stencil_entry_point_rows(nxg_lib, slots):
    src = _ties_and_penalties()
    host = build_asset(src, slots)
    pos, tris, roots, normals = _device_inputs(src, host)
    rows = build_stencils(pos, tris, roots, normals, slots).cpu().numpy().view(np.uint32)
    assert np.array_equal(rows, host.stencil().reshape(-1, 8))


def test_out_of_range_triangle_gets_invalid_row(nxg_lib):
    src = fixtures.plain_sphere().build_input
    host = build_asset(src, 8)
    pos, tris, roots, normals = _device_inputs(src, host)
    v = pos.shape[0]
    bad = torch.tensor([[0, 1, v], [v + 5, 0, 1]], dtype=torch.int32, device="cuda")
    rows = build_stencils(pos, torch.cat([tris, bad]), roots, normals).cpu().numpy().view(np.uint32)
    assert np.array_equal(rows[:-2], host.stencil().reshape(-1, 8))
    assert (rows[-2:] == 0xFFFFFFFF).all()
