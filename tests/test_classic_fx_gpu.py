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


@pytest.fixture(scope="module")
def curves(cuda, nxg_lib, reference):
    """The reference generator's curves of 6,000 strands x 16 CVs on the
    plain sphere (noise off), with one surface tangent per strand (some of
    them zero, which the NoiseFX frame replaces by its fallback)."""
    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    w = fixtures.plain_sphere(strands=6000)
    asset = build_asset(w.build_input, w.stencil_slots)
    params = w.params.copy(noise_amplitude=0.0)
    pts, roots, uvs, counts, _ = reference.generate(reference.handle(asset.buffer), params, 1.0)
    rng = np.random.default_rng(17)
    tangents = rng.normal(size=(roots.size, 3)).astype(np.float32)
    tangents[::97] = 0.0
    return asset, int(params.cvs_per_strand), pts, roots, uvs, counts, tangents


def _run(curves, reference, primitive, effects, radius_scale=1.0, description_id=5, name="desc:hairA"):
    import torch

    from nanoxgen_b200.classic import FxPlan, classic_fx_apply
    from nanoxgen_b200.generator import PackedCurves
    asset, P, pts, roots, uvs, counts, tangents = curves
    plan = FxPlan(primitive, effects, description_id, name)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    mine = PackedCurves(strand_count=counts.size, cvs_per_strand=P, points=dev(pts),
                        roots=dev(roots.view(np.int32).reshape(-1, 12)), root_uvs=dev(uvs),
                        point_counts=dev(counts.view(np.int32)))
    status = classic_fx_apply(plan, mine, dev(tangents) if plan.has_noise else None, radius_scale)
    torch.cuda.synchronize()
    rplan = reference.classic_plan_fx(primitive, effects, description_id, name)
    assert rplan.fallback_reasons == [] and rplan.effect_counts[2] == len(effects)
    freqs = rplan.info()["pref_noise"]
    inputs = np.stack([reference.classic_noise(roots["position"], f) for f in freqs], 1) if len(freqs) else None
    theirs = reference.classic_apply_fx(rplan, pts, counts, roots, uvs, P, radius_scale, inputs,
                                        tangents if plan.has_noise else None, workers=8)
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
