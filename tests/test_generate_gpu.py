"""Parity of the CUDA generator (nxg_generate_packed through the C ABI)
against the oracle and the reference's golden outputs.

Bars (stated per assertion): root triangle indices, stencil indices, nearest
guides and point counts bit-exact; positions and radii within 1e-5 of the
mesh bounding-box diagonal.
"""
import os

import numpy as np
import pytest

from helpers import max_position_error, patch_stencil

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-5  # x mesh bounding-box diagonal


@pytest.fixture(scope="module")
def torch_cuda(cuda, nxg_lib):
    import torch
    return torch


def _gen(torch_cuda, asset, params, radius_scale=1.0, deformed=None, **kw):
    from nanoxgen_b200.generator import DeviceAsset, generate_packed
    d = asset if isinstance(asset, DeviceAsset) else DeviceAsset(asset)
    out = generate_packed(d, params, radius_scale, deformed, **kw)
    torch_cuda.cuda.synchronize()
    roots = out.roots_numpy() if out.roots is not None else None
    return (out.points.cpu().numpy(), roots,
            out.root_uvs.cpu().numpy() if out.root_uvs is not None else None,
            out.point_counts.cpu().numpy().view(np.uint32) if out.point_counts is not None else None)


def _compare(asset, params, mine, theirs, tol=TOL, radius_scale=1.0):
    diag = asset.bbox_diagonal()
    pts, roots, uvs, counts = mine
    rpts, rroots, ruvs, rcounts = theirs[:4]
    assert np.array_equal(roots["triangle_index"], rroots["triangle_index"])       # bit-exact
    assert np.array_equal(roots.view(np.uint8), rroots.view(np.uint8))              # whole RootSample bit-exact
    assert np.array_equal(counts, rcounts) and np.all(counts == params.cvs_per_strand)
    assert np.array_equal(uvs, ruvs)
    err = max_position_error(pts, rpts)
    assert err <= tol * diag, "max position error %.3g > %.3g" % (err, tol * diag)
    rerr = float(np.abs(pts[:, 3] - rpts[:, 3]).max())
    assert rerr <= tol * diag
    return err / diag


@pytest.fixture(scope="module")
def sphere(nxg_lib):
    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    w = fixtures.plain_sphere()
    return w, build_asset(w.build_input, w.stencil_slots)


def test_plain_sphere_full_parity(torch_cuda, oracle, sphere):
    w, asset = sphere
    for params in (w.params, w.params.copy(noise_amplitude=0.0),
                   w.params.copy(noise_mask=0.83, noise_correlation=0.35, noise_preserve_length=0.4),
                   w.params.copy(noise_preserve_length=1.0, seed=99)):
        mine = _gen(torch_cuda, asset, params, 1.5)
        theirs = oracle.generate(asset.buffer, params, 1.5, threads=8)
        rel = _compare(asset, params, mine, theirs)
        print("plain sphere max rel error %.3g" % rel)


def test_stencil_indices_bit_exact(torch_cuda, oracle, sphere):
    from nanoxgen_b200.generator import DeviceAsset, query_strand_states
    w, asset = sphere
    d = DeviceAsset(asset)
    ids = np.arange(0, w.params.strand_count, 7, dtype=np.uint32)
    for params in (w.params, w.params.copy(normal_rejection_cos=0.5, guide_support_scale=0.4)):
        states = query_strand_states(d, params, ids)
        for s, st in zip(ids, states):
            ref = oracle.strand_state(asset.buffer, params, int(s))
            assert np.array_equal(st["indices"], ref["indices"]), s
            assert st["nearest"] == ref["nearest"], s
            assert st["root"].tobytes() == ref["root"].tobytes(), s
            assert st["weight_sum"] == pytest.approx(ref["weight_sum"], rel=1e-5)
            np.testing.assert_allclose(st["weights"], ref["weights"], rtol=1e-5, atol=1e-7)


INVALID = 0xFFFFFFFF


def _reference_mode(ref) -> int:
    """interpolate_offset's choice (generate.h:261-266): 0 blend, 1 nearest
    guide, 2 root normal."""
    if ref["weight_sum"] > np.float32(1e-12):
        return 0
    return 1 if ref["nearest"] != INVALID else 2


def _check_walk_state(st, ref, strand, power):
    """The walk's weights are either exact or fast ones whose error is bounded
    (walk_needs_exact_weights): each within (p * 4e-7 + 1e-5) relative for the
    fast power, plus 1e-5 of the weight sum for the base's cancellation."""
    mode = _reference_mode(ref)
    assert st["mode"] == mode, strand
    assert st["nearest"] == ref["nearest"], strand
    if mode == 0:
        used = ref["indices"] != INVALID
        n = int(used.sum())
        assert st["slot_count"] == n, strand
        assert np.array_equal(st["guides"][:n], ref["indices"][used]), strand          # slot order kept
        want = ref["weights"][used].astype(np.float64)
        got = st["weights"][:n].astype(np.float64)
        bound = 2.0 * (power * 4e-7 + 1e-5) * want + 1e-5 * float(ref["weight_sum"])
        assert np.all(np.abs(got - want) <= bound), (strand, got, want)
    elif mode == 1:
        assert st["slot_count"] == 1 and st["guides"][0] == ref["nearest"] and st["weights"][0] == 1.0, strand
    else:
        assert st["slot_count"] == 0, strand
    return mode


def test_walk_stencil_decisions_bit_exact(torch_cuda, oracle, sphere):
    """The lane walk's own setup step (nxg_query_walk_states), which is what
    generates every strand of 2..32 CVs: its blended guides in slot order, its
    nearest guide and its blend / nearest / normal choice against the
    reference's make_guide_blend_state and interpolate_offset
    (generate.h:214-266).  The parameter sets include rejection-heavy,
    narrow-support and high-power cases, where many strands fall back to the
    nearest guide or sit near the 1e-12 weight-sum threshold."""
    from nanoxgen_b200.generator import DeviceAsset, query_walk_states
    w, asset = sphere
    d = DeviceAsset(asset)
    ids = np.arange(0, w.params.strand_count, 3, dtype=np.uint32)
    modes = np.zeros(3, np.int64)
    for params in (w.params, w.params.copy(normal_rejection_cos=0.5, guide_support_scale=0.4),
                   w.params.copy(guide_weight_power=40.0, guide_support_scale=0.7),
                   w.params.copy(guide_weight_power=0.5, guide_support_scale=0.15),
                   w.params.copy(normal_rejection_cos=0.999, guide_support_scale=0.3)):
        states = query_walk_states(d, params, ids)
        for s, st in zip(ids, states):
            modes[_check_walk_state(st, oracle.strand_state(asset.buffer, params, int(s)), int(s),
                                    params.guide_weight_power)] += 1
    assert modes.min() > 0, modes  # every mode was exercised


def test_walk_blend_threshold_decision(torch_cuda, oracle, nxg_lib):
    """Weight sums within a few parts per million of the 1e-12 threshold.
    One guide, so the sum is its weight (1 - d/r)^p; the power is stepped one
    float at a time across the value that puts a strand's weight at 1e-12.
    The fast weights the walk blends with are further than that from the
    reference's, so the walk must take the decision on exactly rounded
    weights.  The only allowed disagreement is where the reference's own sum
    is within 4 ulp of 1e-12 (CUDA's powf and the host's may differ in the
    last bit)."""
    from nanoxgen_b200 import fixtures
    from nanoxgen_b200._abi import GenerationParams
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import DeviceAsset, query_walk_states
    asset = build_asset(fixtures.reference_unit_fixture())
    d = DeviceAsset(asset)
    base = GenerationParams(strand_count=64, cvs_per_strand=8, seed=5, guide_weight_power=1.0)
    threshold = np.float32(1e-12)
    checked = flips_possible = 0
    for strand in range(0, 64, 8):
        x = float(oracle.strand_state(asset.buffer, base, strand)["weights"][0])
        if not 0.05 < x < 0.9999:
            continue
        p_star = np.float32(np.log(1e-12) / np.log(x))
        powers = [p_star]
        for _ in range(24):
            powers.append(np.nextafter(powers[-1], np.float32(np.inf)))
            powers.insert(0, np.nextafter(powers[0], np.float32(-np.inf)))
        for pw in powers:
            params = base.copy(guide_weight_power=float(pw))
            st = query_walk_states(d, params, [strand])[0]
            ref = oracle.strand_state(asset.buffer, params, strand)
            near = abs(int(np.float32(ref["weight_sum"]).view(np.int32)) - int(threshold.view(np.int32))) <= 4
            if near:
                flips_possible += 1
                continue
            _check_walk_state(st, ref, strand, float(pw))
            checked += 1
    assert checked >= 300, checked
    print("threshold scan: %d decisions checked, %d within 4 ulp skipped" % (checked, flips_possible))


@pytest.mark.parametrize("name", ["unit_fixture.npz", "plain_sphere.npz"])
def test_golden_outputs(torch_cuda, name):
    """Against the reference's own outputs committed under tests/golden."""
    from nanoxgen_b200._abi import GenerationParams
    from nanoxgen_b200.asset import Asset
    g = np.load(os.path.join(GOLDEN, name))
    asset = Asset(g["asset"])
    rs = float(g["radius_scale"])
    k = 0
    while "params%d" % k in g:
        params = GenerationParams.from_buffer_copy(g["params%d" % k].tobytes())
        pts, roots, uvs, counts = _gen(torch_cuda, asset, params, rs)
        ids = g["strands"]
        ids = ids[ids < params.strand_count]
        P = int(params.cvs_per_strand)
        idx = (ids[:, None] * P + np.arange(P)[None, :]).reshape(-1)
        n = ids.size
        theirs = (g["points%d" % k][: n * P], g["roots%d" % k].view(roots.dtype)[:n], g["uvs%d" % k][:n],
                  g["counts%d" % k][:n])
        _compare(asset, params, (pts[idx], roots[ids], uvs[ids], counts[ids]), theirs)
        k += 1


def test_unit_fixture_known_answers(torch_cuda, nxg_lib):
    """tests/test_main.cpp:66-100 on the device path."""
    from nanoxgen_b200 import fixtures
    from nanoxgen_b200._abi import GenerationParams
    from nanoxgen_b200.asset import build_asset
    asset = build_asset(fixtures.reference_unit_fixture())
    pts, roots, _, _ = _gen(torch_cuda, asset, GenerationParams(strand_count=1, cvs_per_strand=3, seed=7))
    assert abs(pts[1, 1] - 0.5) < 1e-6 and abs(pts[2, 1] - 1.0) < 1e-6
    assert abs((pts[2, 0] - roots["position"][0, 0]) - 0.25) < 1e-6
    params = GenerationParams(strand_count=128, cvs_per_strand=7, seed=42)
    a = _gen(torch_cuda, asset, params)
    b = _gen(torch_cuda, asset, params)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))            # bitwise deterministic
    assert np.array_equal(a[0][::7, :3], a[1]["position"])             # CV 0 is the root


@pytest.mark.parametrize("cvs", [2, 3, 8, 12, 17, 24, 32, 33, 48, 64, 65, 100, 128, 129, 200])
def test_cv_counts_and_tile_shapes(torch_cuda, oracle, sphere, cvs):
    w, asset = sphere
    params = w.params.copy(strand_count=777, cvs_per_strand=cvs,
                           noise_preserve_length=0.3 if cvs % 2 else 0.0)
    _compare(asset, params, _gen(torch_cuda, asset, params), oracle.generate(asset.buffer, params, threads=8))


def test_fallbacks_and_degenerate_stencils(torch_cuda, oracle, sphere):
    """Zero blend weight -> nearest guide; every guide rejected -> normal * t
    (generate.h:261-266)."""
    w, asset = sphere
    for params in (w.params.copy(guide_support_scale=0.0, strand_count=3000),
                   w.params.copy(guide_support_scale=0.05, strand_count=3000),
                   w.params.copy(normal_rejection_cos=1.0, strand_count=3000),
                   w.params.copy(guide_weight_power=0.0, length_scale=1.7, strand_count=3000)):
        _compare(asset, params, _gen(torch_cuda, asset, params), oracle.generate(asset.buffer, params, threads=8))


def test_asset_without_texcoords_and_single_guide(torch_cuda, oracle, nxg_lib):
    from nanoxgen_b200 import fixtures
    from nanoxgen_b200._abi import GenerationParams
    from nanoxgen_b200.asset import build_asset
    for src in (fixtures.reference_area_fixture(), fixtures.reference_benchmark_fixture()):
        asset = build_asset(src)
        for params in (GenerationParams(strand_count=2000, cvs_per_strand=12, seed=23),
                       GenerationParams(strand_count=2000, cvs_per_strand=12, seed=23, noise_amplitude=0.043,
                                        noise_frequency=3.17, noise_mask=0.83, noise_correlation=0.35,
                                        noise_preserve_length=0.4)):
            _compare(asset, params, _gen(torch_cuda, asset, params), oracle.generate(asset.buffer, params))


def test_deformed_geometry(torch_cuda, oracle, sphere):
    import torch
    from nanoxgen_b200.generator import DeformedGeometry
    w, asset = sphere
    rng = np.random.default_rng(11)
    pos = (asset.positions() + rng.normal(0, 0.02, asset.positions().shape)).astype(np.float32)
    nrm = asset.normals()
    gcv = (asset.guide_cvs() + rng.normal(0, 0.01, asset.guide_cvs().shape)).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    for kw in ({"positions": pos}, {"positions": pos, "normals": nrm}, {"normals": nrm},
               {"positions": pos, "normals": nrm, "guide_cvs": gcv}, {"guide_cvs": gcv}):
        deformed = DeformedGeometry(**{k: dev(v) for k, v in kw.items()})
        mine = _gen(torch_cuda, asset, w.params, 1.0, deformed)
        theirs = oracle.generate(asset.buffer, w.params, 1.0, threads=8, **kw)
        _compare(asset, w.params, mine, theirs)


def test_range_generation_matches_full(torch_cuda, sphere):
    w, asset = sphere
    full = _gen(torch_cuda, asset, w.params)
    P = w.params.cvs_per_strand
    for first, count in ((0, 1), (1234, 4321), (9999, 1), (5000, 5000)):
        part = _gen(torch_cuda, asset, w.params, first_strand=first, count=count)
        assert np.array_equal(part[0], full[0][first * P:(first + count) * P])
        assert np.array_equal(part[1].view(np.uint8), full[1][first:first + count].view(np.uint8))


def test_optional_outputs_and_errors(torch_cuda, sphere):
    import torch
    from nanoxgen_b200._abi import ERRORS, NxgError
    from nanoxgen_b200.generator import DeviceAsset, generate_packed
    w, asset = sphere
    d = DeviceAsset(asset)
    pts_only = generate_packed(d, w.params, want_roots=False)
    torch.cuda.synchronize()
    full = _gen(torch_cuda, d, w.params)
    assert np.array_equal(pts_only.points.cpu().numpy(), full[0])
    small = torch.empty((w.params.strand_count * w.params.cvs_per_strand - 1, 4), device="cuda")
    with pytest.raises(NxgError) as e:
        generate_packed(d, w.params, points=small)
    assert e.value.code == ERRORS["PointCapacityTooSmall"]
    with pytest.raises(NxgError) as e:
        generate_packed(d, w.params, radius_scale=float("nan"))
    assert e.value.code == ERRORS["InvalidRadiusScale"]
    with pytest.raises(NxgError) as e:
        generate_packed(d, w.params.copy(cvs_per_strand=1))
    assert e.value.code == ERRORS["InvalidGenerationParameters"]
    base = torch.empty((w.params.strand_count * w.params.cvs_per_strand + 1, 4), device="cuda")
    shifted = base.view(-1)[1:1 + w.params.strand_count * w.params.cvs_per_strand * 4].view(-1, 4)
    with pytest.raises(NxgError) as e:
        generate_packed(d, w.params, points=shifted)
    assert e.value.code == ERRORS["MisalignedOutput"]


def test_graph_capture_replays_identically(torch_cuda, sphere):
    import torch
    from nanoxgen_b200.generator import DeviceAsset, allocate_outputs, generate_packed
    w, asset = sphere
    d = DeviceAsset(asset)
    P = w.params.cvs_per_strand
    pts, roots, uvs, pc = allocate_outputs(w.params.strand_count, P, "cuda")
    eager = generate_packed(d, w.params).points.clone()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    d.workspace(w.params, w.params.strand_count)
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        generate_packed(d, w.params, points=pts, roots=roots, root_uvs=uvs, point_counts=pc, stream=s)
    pts.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(pts, eager)


def test_large_sphere_full_size_parity(torch_cuda, oracle, nxg_lib):
    """The 1,000,000 x 32 single-description workload: every strand against
    the oracle (multi-threaded), plus the size-independent properties."""
    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    w = fixtures.large_sphere()
    asset = build_asset(w.build_input, w.stencil_slots)
    mine = _gen(torch_cuda, asset, w.params)
    assert np.all(mine[3] == 32)
    assert np.array_equal(mine[0][::32, :3], mine[1]["position"])     # CV 0 == root, bitwise
    theirs = oracle.generate(asset.buffer, w.params, threads=os.cpu_count() or 8)
    rel = _compare(asset, w.params, mine, theirs)
    print("large sphere max rel error %.3g" % rel)


@pytest.mark.parametrize("block", [1, 32, 100, 256, 1024])
def test_launch_block_sizes(torch_cuda, sphere, block):
    """DeviceLaunchConfig::block_size anywhere in [1, 1024] (device_contract.h:54-56,
    :165-167) launches and leaves the output unchanged."""
    w, asset = sphere
    ref = _gen(torch_cuda, asset, w.params)
    out = _gen(torch_cuda, asset, w.params, block_size=block)
    assert all(np.array_equal(x, y) for x, y in zip(ref, out))


@pytest.mark.parametrize("block", [64, 96, 320, 352])
def test_lane_walk_ctas_match_oracle(torch_cuda, oracle, sphere, block):
    """The lane-walk generator with noise as producer/consumer warp pairs
    (64 threads) and as three-, ten- and eleven-warp CTAs (the last with ten
    lattice columns per axis instead of twelve), over CV counts that do and
    do not fill a warp, with and without preserveLength."""
    from nanoxgen_b200.generator import set_tile
    w, asset = sphere
    for cvs, preserve in ((7, 0.0), (17, 0.3), (32, 0.0), (32, 0.6)):
        params = w.params.copy(strand_count=2500, cvs_per_strand=cvs, noise_preserve_length=preserve)
        try:
            set_tile(cvs, True, 1, 1, block)
            _compare(asset, params, _gen(torch_cuda, asset, params), oracle.generate(asset.buffer, params, threads=8))
        finally:
            set_tile(cvs, True)


@pytest.mark.parametrize("block", [320, 352])
def test_lane_walk_direct_noise_when_the_lattice_overflows(torch_cuda, oracle, sphere, block):
    """At a high noise frequency a strand spans more lattice columns than the
    lane walk keeps (12 per axis in ten-warp CTAs, 10 in eleven-warp ones);
    its warp then evaluates gradient noise directly.  Also frequencies near
    either limit, where some warps fit and others do not."""
    from nanoxgen_b200.generator import set_tile
    w, asset = sphere
    try:
        set_tile(32, True, 1, 1, block)
        for frequency in (60.0, 14.0, 11.0):
            params = w.params.copy(strand_count=3000, cvs_per_strand=32, noise_frequency=frequency)
            _compare(asset, params, _gen(torch_cuda, asset, params), oracle.generate(asset.buffer, params, threads=8))
    finally:
        set_tile(32, True)


def test_every_tile_matches_oracle_and_autotuner(torch_cuda, oracle, sphere):
    """Each admissible tile (lanes per strand x CVs per lane) is a different
    lane layout of the same arithmetic: all stay within tolerance of the
    oracle; the autotuner registers one of them."""
    from nanoxgen_b200.generator import DeviceAsset, allocate_outputs, autotune, get_tile, set_tile
    w, asset = sphere
    d = DeviceAsset(asset)
    theirs = oracle.generate(asset.buffer, w.params, threads=8)
    P = w.params.cvs_per_strand
    try:
        for lanes, ppt in ((1, 1), (4, 4), (8, 2), (8, 4), (16, 1), (16, 2), (32, 1)):
            set_tile(P, True, lanes, ppt, 128)
            _compare(asset, w.params, _gen(torch_cuda, d, w.params), theirs)
        # the lane walk as producer/consumer warp pairs (64-thread CTAs) and
        # as ten- and eleven-warp CTAs
        for block in (64, 320, 352):
            set_tile(P, True, 1, 1, block)
            _compare(asset, w.params, _gen(torch_cuda, d, w.params), theirs)
        pts, *_ = allocate_outputs(w.params.strand_count, P, "cuda")
        (lanes, ppt, block), ms = autotune(d, w.params, pts, repeats=2)
        assert (lanes == 1 or lanes * ppt >= P) and ms > 0.0
        assert get_tile(P, True) == (lanes, ppt, block)
        _compare(asset, w.params, _gen(torch_cuda, d, w.params), theirs)
    finally:
        set_tile(P, True)


def test_host_pipeline_runs_match_direct_generation(torch_cuda, sphere):
    """HostPipeline (host asset in, host arrays out, ranges read back while
    later ranges generate, a run's upload and generation under the previous
    run's readback): two consecutive runs leave exactly the arrays that one
    direct generation of the whole request produces."""
    from nanoxgen_b200.generator import HostPipeline
    w, asset = sphere
    params = w.params.copy(strand_count=20000)
    pts, roots, uvs, counts = _gen(torch_cuda, asset, params)
    pipe = HostPipeline(asset, params, 1.0, chunks=5, device="cuda")
    for _ in range(2):
        pipe.run()
    torch_cuda.cuda.synchronize()
    assert np.array_equal(pipe.host_points.numpy(), pts)
    assert np.array_equal(pipe.host_roots.numpy().reshape(-1).view(np.uint8),
                          np.ascontiguousarray(roots).reshape(-1).view(np.uint8))
    assert np.array_equal(pipe.host_uvs.numpy(), uvs)
    assert np.array_equal(pipe.host_counts.numpy().view(np.uint32), counts)
