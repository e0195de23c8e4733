"""The Classic FX passes on the GPU (nxg_classic_fx_apply) against the
reference's apply_xgen_classic_float_runtime_plan_cpu on the same input
curves (the reference generator's output for the plain sphere).

Bars: the surviving strand set and order bit-exact (the drop rule on cLength
and width, CutFX's cut-to-nothing); positions and radii of the survivors
within 1e-5 of the mesh bounding-box diagonal (NoiseFX's frame uses CUDA's
acos/cos/sin, so it agrees to rounding rather than bit for bit).  rand() is
not exercised: the reference's runtime requires a per-strand SeExpr prefix
for it, which this runtime does not bind.
"""
import numpy as np
import pytest

from helpers import max_position_error

pytestmark = pytest.mark.gpu

TOL = 1e-5  # x mesh bounding-box diagonal
NOISE = dict(mask="1", magnitude="0.05", magnitudeScale="1", frequency="4", correlation="20", preserveLength="0")


def _make_curves(reference, strands, cvs):
    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    w = fixtures.plain_sphere(strands=strands, cvs=cvs)
    asset = build_asset(w.build_input, w.stencil_slots)
    params = w.params.copy(noise_amplitude=0.0)
    pts, roots, uvs, counts, _ = reference.generate(reference.handle(asset.buffer), params, 1.0)
    rng = np.random.default_rng(17)
    tangents = rng.normal(size=(roots.size, 3)).astype(np.float32)
    tangents[::97] = 0.0
    return asset, int(params.cvs_per_strand), pts, roots, uvs, counts, tangents


@pytest.fixture(scope="module")
def curves(cuda, nxg_lib, reference):
    """The reference generator's curves of 6,000 strands x 16 CVs on the
    plain sphere (noise off), with one surface tangent per strand (some of
    them zero, which the NoiseFX frame replaces by its fallback)."""
    return _make_curves(reference, 6000, 16)


def _clump_guides(curves, count=48, seed=5, with_reference_positions=False, unassigned=0.1):
    """ClumpingFX guides taken from `count` of the curves (their CVs, root
    normals and uvs), random tangents (some zero) and SeExpr prefixes, and a
    guide per strand (the nearest guide root; a share of strands without)."""
    _, P, pts, roots, uvs, counts, _ = curves
    rng = np.random.default_rng(seed)
    pick = rng.choice(counts.size, count, replace=False)
    axes = pts.reshape(-1, P, 4)[pick, :, :3].copy()
    axes += rng.normal(scale=0.01, size=axes.shape).astype(np.float32) * (np.arange(P) > 0)[None, :, None]
    tangents = rng.normal(size=(count, 3)).astype(np.float32)
    tangents[::7] = 0.0
    d = ((roots["position"][:, None, :] - axes[None, :, 0, :]) ** 2).sum(-1)
    strand_guides = d.argmin(1).astype(np.uint32)
    strand_guides[rng.random(counts.size) < unassigned] = 0xFFFFFFFF
    g = dict(axes=axes, normals=roots["normal"][pick].astype(np.float32), tangents=tangents,
             uvs=uvs[pick].astype(np.float32), prefixes=rng.integers(0, 2**32, count, dtype=np.uint32),
             strand_guides=strand_guides)
    if with_reference_positions:
        g["reference_positions"] = axes[:, 0, :] + rng.normal(scale=0.05, size=(count, 3)).astype(np.float32)
    return g


def _run(curves, reference, primitive, effects, radius_scale=1.0, description_id=5, name="desc:hairA",
         clumps=(), prefixes=None):
    import torch

    from nanoxgen_b200.classic import ClumpGuides, FxPlan, classic_fx_apply
    from nanoxgen_b200.generator import PackedCurves
    asset, P, pts, roots, uvs, counts, tangents = curves
    plan = FxPlan(primitive, effects, description_id, name)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    mine = PackedCurves(strand_count=counts.size, cvs_per_strand=P, points=dev(pts),
                        roots=dev(roots.view(np.int32).reshape(-1, 12)), root_uvs=dev(uvs),
                        point_counts=dev(counts.view(np.int32)))
    guides = [ClumpGuides(c["axes"], c["normals"], c["tangents"], c["uvs"], c["prefixes"], c["strand_guides"],
                          c.get("reference_positions"), noise_table=c.get("noise_table", True)) for c in clumps]
    status = classic_fx_apply(plan, mine, dev(tangents) if plan.has_noise else None, radius_scale,
                              random_prefixes=None if prefixes is None else dev(prefixes.view(np.int32)),
                              clumps=guides)
    torch.cuda.synchronize()
    rplan = reference.classic_plan_fx(primitive, effects, description_id, name)
    assert rplan.fallback_reasons == [] and rplan.effect_counts[2] == len(effects)
    freqs = rplan.info()["pref_noise"]
    inputs = np.stack([reference.classic_noise(roots["position"], f) for f in freqs], 1) if len(freqs) else None
    theirs = reference.classic_apply_fx(rplan, pts, counts, roots, uvs, P, radius_scale, inputs,
                                        tangents if plan.has_noise else None, workers=8, random_prefixes=prefixes,
                                        clumps=[{k: v for k, v in c.items() if k != "noise_table"} for c in clumps])
    return (status.cpu().tolist(), mine.points.cpu().numpy(), mine.point_counts.cpu().numpy().view(np.uint32)), theirs


def _check(curves, mine, theirs):
    asset, P, _, roots, _, _, _ = curves
    status, pts, counts = mine
    rpts, rcounts, rroots, _ = theirs
    assert status == [0, 0]
    kept = counts != 0
    assert np.all(counts[kept] == P)
    assert kept.sum() == rcounts.size                                            # the same survivors ...
    np.testing.assert_array_equal(roots[kept]["triangle_index"], rroots["triangle_index"])  # ... in order
    sel = np.repeat(kept, P)
    diag = asset.bbox_diagonal()
    err = max_position_error(pts[sel], rpts) / diag
    rerr = float(np.abs(pts[sel, 3].astype(np.float64) - rpts[:, 3]).max(initial=0.0)) / diag
    assert err <= TOL, "max position error %.3g x diag" % err
    assert rerr <= TOL, "max radius error %.3g x diag" % rerr
    return err, int(kept.sum())


def test_noise_fx(curves, reference):
    mine, theirs = _run(curves, reference, {"length": "0.9", "width": "0.01"}, [("noise", NOISE)])
    err, kept = _check(curves, mine, theirs)
    print("NoiseFX: max error %.3g x diag, %d strands" % (err, kept))


def test_noise_fx_preserve_length_and_per_cv_magnitude(curves, reference):
    noise = dict(NOISE, magnitude="0.04*rampUI(0,0.2,1:1,1,1)", magnitudeScale="1.5", frequency="6",
                 preserveLength="50", correlation="0")
    mine, theirs = _run(curves, reference, {"width": "0.012"}, [("noise", noise)], radius_scale=2.0)
    _check(curves, mine, theirs)


def test_cut_fx(curves, reference):
    # hash($id) spreads the cut over the strands; a few amounts exceed the
    # strand's length, so those strands are cut to nothing and dropped.
    mine, theirs = _run(curves, reference, {"width": "0.01"}, [("cut", {"amount": "0.02 + 0.6*hash($id)"})])
    err, kept = _check(curves, mine, theirs)
    assert kept < 6000
    print("CutFX: max error %.3g x diag, %d of 6000 strands kept" % (err, kept))


def test_chain_with_width_profile(curves, reference):
    effects = [("noise", NOISE), ("cut", {"amount": "$cLength*0.25"}),
               ("noise", dict(NOISE, magnitude="$cWidth*3", frequency="9", correlation="60", preserveLength="30"))]
    primitive = {"length": "0.7 + 0.3*hash($id, 2)", "width": "0.008 + 0.004*hash($id, 3)", "taper": "0.8",
                 "taperStart": "0.25", "widthRamp": "rampUI(0,1,1:0.5,0.6,2:1,0.3,1)"}
    mine, theirs = _run(curves, reference, primitive, effects, radius_scale=1.5)
    err, kept = _check(curves, mine, theirs)
    print("noise, cut, noise + width profile: max error %.3g x diag, %d strands" % (err, kept))


@pytest.mark.parametrize("cvs", [2, 3, 64])
def test_cvs_extremes(cuda, nxg_lib, reference, cvs):
    # 1,000 strands (a ragged last warp of 8) at the smallest and the largest
    # CV counts the pass takes; 64 CVs need more than 48 KB of planes.
    curves = _make_curves(reference, 1000, cvs)
    effects = [("noise", NOISE), ("cut", {"amount": "$cLength*0.3*hash($id)"})]
    primitive = {"length": "0.8 + 0.2*hash($id, 2)", "width": "0.01", "taper": "0.5", "taperStart": "0.2"}
    mine, theirs = _run(curves, reference, primitive, effects)
    _check(curves, mine, theirs)


def test_drop_rule(curves, reference):
    mine, theirs = _run(curves, reference, {"length": "hash($id)*0.0006 + 0.00001", "width": "hash($id, 7)*0.0003"},
                        [("cut", {"amount": "$cLength*0.2"})])
    _, kept = _check(curves, mine, theirs)
    assert 300 < kept < 5700


def test_errors_are_reported(curves, reference):
    import torch

    from nanoxgen_b200._abi import ERRORS
    from nanoxgen_b200.classic import FxPlan, classic_fx_apply
    from nanoxgen_b200.generator import PackedCurves
    _, P, pts, roots, uvs, counts, _ = curves
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    fresh = lambda: PackedCurves(strand_count=counts.size, cvs_per_strand=P, points=dev(pts),
                                 roots=dev(roots.view(np.int32).reshape(-1, 12)), root_uvs=dev(uvs),
                                 point_counts=dev(counts.view(np.int32)))
    # NoiseFX without the strands' surface tangents
    status = classic_fx_apply(FxPlan({}, [("noise", NOISE)]), fresh(), None)
    assert status.cpu().tolist() == [ERRORS["InvalidArgument"], counts.size]
    # a negative length for part of the strands
    status = classic_fx_apply(FxPlan({"length": "hash($id) - 0.5"}), fresh(), None)
    st = status.cpu().tolist()
    assert st[0] == ERRORS["ExpressionDomain"] and 0 < st[1] < counts.size


CLUMP = dict(mask="1", clump="0.8", clumpScale="0.2*rampUI(0,0,1:1,1,1)", noise="0.05", noiseScale="1",
             noiseFrequency="5", noiseCorrelation="20")


def test_clump_prepare_matches_reference(curves, reference):
    # prepare_xgen_classic_clump_runtime_data on the device: render axes and
    # spline lengths bit for bit.
    import torch

    from nanoxgen_b200.classic import ClumpGuides
    g = _clump_guides(curves)
    mine = ClumpGuides(g["axes"], g["normals"], g["tangents"], g["uvs"], g["prefixes"], g["strand_guides"])
    torch.cuda.synchronize()
    render, lengths = reference.classic_clump_prepare(g["axes"])
    np.testing.assert_array_equal(mine.render_axes.cpu().numpy().view(np.uint32), render.view(np.uint32))
    np.testing.assert_array_equal(mine.spline_lengths.cpu().numpy().view(np.uint32), lengths.view(np.uint32))


@pytest.mark.parametrize("path", ["per guide", "per strand", "strand input"])
def test_clump_fx(curves, reference, path):
    # The guide noise from the per-guide table, evaluated per strand (no
    # table), and per strand because a guide-noise program reads $id.
    g = dict(_clump_guides(curves), noise_table=path != "per strand")
    clump = dict(CLUMP, noiseScale="0.5 + hash($id)") if path == "strand input" else CLUMP
    mine, theirs = _run(curves, reference, {"width": "0.01"}, [("clump", clump)], clumps=[g])
    err, kept = _check(curves, mine, theirs)
    print("ClumpingFX (%s): max error %.3g x diag, %d strands" % (path, err, kept))


def test_clump_without_noise_is_exact(curves, reference):
    # No guide noise: the cut to the guide's length and the pull use IEEE
    # arithmetic only, so the points agree bit for bit.
    g = _clump_guides(curves, seed=9)
    clump = dict(CLUMP, noise="0", clump="0.3 + 0.7*hash($id)", mask="hash($id, 4)")
    mine, theirs = _run(curves, reference, {"width": "0.01"}, [("clump", clump)], clumps=[g])
    status, pts, counts = mine
    kept = counts != 0
    np.testing.assert_array_equal(pts[np.repeat(kept, curves[1])].view(np.uint32), theirs[0].view(np.uint32))


def test_clump_chain_with_reference_positions_and_rand(curves, reference):
    # Clump (guide-noise domains given, rand() in the guide noise with the
    # guides' prefixes) between NoiseFX and CutFX, rand() in the strands'
    # programs with their prefixes, two clump modules.
    rng = np.random.default_rng(3)
    prefixes = rng.integers(0, 2**32, curves[5].size, dtype=np.uint32)
    g1 = _clump_guides(curves, seed=11, with_reference_positions=True)
    g2 = _clump_guides(curves, count=24, seed=12, unassigned=0.5)
    clump1 = dict(CLUMP, noise="0.04*rand(0.5, 1.5)", noiseScale="rampUI(0,0.2,1:1,1,1)", mask="0.9")
    clump2 = dict(CLUMP, clump="rand()", clumpScale="0.1", noise="0.02", noiseCorrelation="70")
    effects = [("noise", NOISE), ("clump", clump1), ("cut", {"amount": "$cLength*0.2*rand()"}), ("clump", clump2)]
    primitive = {"length": "0.7 + 0.3*rand(7)", "width": "0.01", "taper": "0.5"}
    mine, theirs = _run(curves, reference, primitive, effects, clumps=[g1, g2], prefixes=prefixes)
    err, kept = _check(curves, mine, theirs)
    print("noise, clump, cut, clump with rand(): max error %.3g x diag, %d strands" % (err, kept))


def test_rand_needs_prefixes(curves, reference):
    import torch

    from nanoxgen_b200._abi import ERRORS
    from nanoxgen_b200.classic import FxPlan, classic_fx_apply
    from nanoxgen_b200.generator import PackedCurves
    _, P, pts, roots, uvs, counts, _ = curves
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    c = PackedCurves(strand_count=counts.size, cvs_per_strand=P, points=dev(pts),
                     roots=dev(roots.view(np.int32).reshape(-1, 12)), root_uvs=dev(uvs),
                     point_counts=dev(counts.view(np.int32)))
    plan = FxPlan({"length": "0.5 + rand()"})
    assert plan.uses_random
    status = classic_fx_apply(plan, c, None)
    assert status.cpu().tolist() == [ERRORS["InvalidArgument"], counts.size]
    # a clump module without its guides
    status = classic_fx_apply(FxPlan({}, [("clump", CLUMP)]), c, None)
    assert status.cpu().tolist() == [ERRORS["InvalidArgument"], counts.size]
