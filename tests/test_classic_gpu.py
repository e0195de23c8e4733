"""The exact Classic-expression runtime on the GPU against the reference's
CPU runtime.

Bars: per-root length and width scalars bit-exact (every op the reference
evaluates with correctly rounded float arithmetic; gamma/contrast, which go
through powf/log2f, within 4 ulp); the fused application (scale about the
first point, width radius, drop rule) against
apply_xgen_classic_float_runtime_plan_cpu: surviving strand set and point
counts bit-exact, positions and radii within 1e-5 of the mesh bounding-box
diagonal.
"""
import re

import numpy as np
import pytest

from helpers import max_position_error

pytestmark = pytest.mark.gpu

TOL = 1e-5
LENGTH = "0.5*(1+0.4*noise($Prefg*6))*clamp(1-$v,0.2,1)"
WIDTH = "0.01*(1+0.3*noise($Prefg*20))"


@pytest.fixture(scope="module")
def sphere(cuda, nxg_lib):
    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import DeviceAsset
    w = fixtures.plain_sphere()
    asset = build_asset(w.build_input, w.stencil_slots)
    return w, asset, DeviceAsset(asset)


def _params(w, strands=20000, cvs=16):
    from nanoxgen_b200._abi import GenerationParams
    p = GenerationParams()
    for name, _ in GenerationParams._fields_:
        setattr(p, name, getattr(w.params, name))
    p.strand_count, p.cvs_per_strand = strands, cvs
    return p


def _reference_roots(reference, asset, params):
    return reference.generate(reference.handle(asset.buffer), params)[1]


def _rewrite_text(source, expression):
    """The source with each noise($Prefg*k) replaced by its input name (what
    the Classic rewrite hands the scalar compiler)."""
    freqs = [float(f) for f in expression.pref_noise_frequencies]
    return re.sub(r"noise\(\$Prefg\*([-+0-9.e]+)\)",
                  lambda m: "$__nxg_pref_noise_%d" % freqs.index(float(np.float32(m.group(1)))), source)


def _bind(program, roots, reference, frequencies):
    """The reference runtime's inputs for each root, by input name."""
    cols = []
    for name in program.describe()["inputs"]:
        if name.startswith("__nxg_pref_noise_"):
            cols.append(reference.classic_noise(roots["position"], frequencies[int(name.rsplit("_", 1)[1])]))
        elif name == "id":
            cols.append(np.arange(roots.size, dtype=np.float32))
        elif name == "u":
            cols.append(roots["uv"][:, 0].copy())
        elif name == "v":
            cols.append(roots["uv"][:, 1].copy())
        elif name == "cWidth":
            cols.append(np.zeros(roots.size, np.float32))
        else:
            raise AssertionError(name)
    return np.stack(cols, 1) if cols else np.zeros((roots.size, 0), np.float32)


def _device_scalars(sphere, params, length=None, width=None, description_id=3, patch="scalp:pSphere1"):
    import torch
    from nanoxgen_b200.classic import Expression, ScalarPlan, root_scalars
    plan = ScalarPlan(Expression.classic(length, "length") if length else None,
                      Expression.classic(width, "width") if width else None, description_id, patch)
    out, status = root_scalars(sphere[2], params, plan)
    torch.cuda.synchronize()
    return out.cpu().numpy(), status.cpu().numpy(), plan


def _reference_scalars(reference, roots, source, attribute, description_id=3):
    from nanoxgen_b200.classic import Expression
    rewritten = Expression.classic(source, attribute)
    prog, msg = reference.compile_expression(_rewrite_text(source, rewritten), attribute, "SplinePrimitive")
    assert prog is not None, msg
    inputs = _bind(prog, roots, reference, rewritten.pref_noise_frequencies)
    face = None
    if "rand" in source:
        face = np.array([reference.runtime_face_seed(description_id, "pSphere1", int(t))
                         for t in roots["triangle_index"]], np.float32)
    return prog.evaluate(inputs, roots["uv"][:, 0].copy(), roots["uv"][:, 1].copy(), face)


def test_cfg5_scalars_bit_exact(sphere, reference):
    w, asset, _ = sphere
    params = _params(w)
    roots = _reference_roots(reference, asset, params)
    mine, status, _ = _device_scalars(sphere, params, LENGTH, WIDTH)
    assert status.tolist() == [0, 0]
    ref_len, ok_len = _reference_scalars(reference, roots, LENGTH, "length")
    ref_wid, ok_wid = _reference_scalars(reference, roots, WIDTH, "width")
    assert ok_len.all() and ok_wid.all()
    np.testing.assert_array_equal(mine[:, 0].view(np.uint32), ref_len.view(np.uint32))
    np.testing.assert_array_equal(mine[:, 1].view(np.uint32), ref_wid.view(np.uint32))


EXACT_PROGRAMS = [
    "fit($u, 0, 1, -2, 2) + smoothstep($v, 0.2, 0.8)",
    "$v > 0.5 ? min($u, 0.3) : max($u, 0.6)",
    "hash($id, 2.5) * 0.5 + hash($u)",
    "rand() + rand(7) + rand(0.2, 0.4) + rand(1, 2, $id)",
    "rampUI(0,0.2,1:0.5,1,2:1,0.25,3) + rampUI(0.3,0.5,0)",
    "!($u < 0.5) || $v == $v && $id != 3",
    "$a = noise($Prefg*3); $b = noise($Prefg*-1.5); ($a - $b) / (1 + $a * $b)",
    "-$u + clamp($v * 3 - 1, 0, 1) - $cWidth",
]


@pytest.mark.parametrize("source", EXACT_PROGRAMS)
def test_scalar_ops_bit_exact(sphere, reference, source):
    w, asset, _ = sphere
    params = _params(w, strands=4096)
    roots = _reference_roots(reference, asset, params)
    mine, status, _ = _device_scalars(sphere, params, width=source)
    theirs, ok = _reference_scalars(reference, roots, source, "width")
    assert ok.all() and status[0] == 0
    np.testing.assert_array_equal(mine[:, 1].view(np.uint32), theirs.view(np.uint32))
    assert np.all(mine[:, 0] == 1.0)  # no length expression: scale 1


@pytest.mark.parametrize("source", ["gamma($u * 0.9 + 0.05, 2.2)", "contrast($v * 0.98 + 0.01, 0.3)"])
def test_transcendental_ops_within_ulps(sphere, reference, source):
    w, asset, _ = sphere
    params = _params(w, strands=4096)
    roots = _reference_roots(reference, asset, params)
    mine, _, _ = _device_scalars(sphere, params, width=source)
    theirs, ok = _reference_scalars(reference, roots, source, "width")
    assert ok.all()
    ulps = np.abs(mine[:, 1].view(np.int32).astype(np.int64) - theirs.view(np.int32).astype(np.int64))
    assert ulps.max() <= 4


def test_domain_errors_are_reported(sphere):
    w, _, _ = sphere
    params = _params(w, strands=1000)
    _, status, _ = _device_scalars(sphere, params, length="$v - 0.5")  # negative for part of the roots
    assert status[0] == 72 and 0 < status[1] < 1000
    _, status, _ = _device_scalars(sphere, params, width="1 / ($v - $v)")  # non-finite everywhere
    assert status[0] == 72 and status[1] == 1000


def test_clength_and_unknown_inputs_are_refused(sphere):
    from nanoxgen_b200._abi import NxgError
    w, _, _ = sphere
    params = _params(w, strands=100)
    with pytest.raises(NxgError, match="ExpressionInput"):
        _device_scalars(sphere, params, length="$cLength * 2")
    with pytest.raises(NxgError, match="ExpressionInput"):
        _device_scalars(sphere, params, width="$P")


def _classic_pair(sphere, reference, params, length, width, ref_length, ref_width, radius_scale=1.0):
    """(mine, theirs) for the fused application and the reference runtime.
    The reference binds $v through a PTEX column (its Classic runtime has no
    $v); the programs are otherwise the same."""
    import torch
    from nanoxgen_b200.classic import generate_packed_classic
    w, asset, dasset = sphere
    scalars, status, plan = _device_scalars(sphere, params, length, width)
    assert status[0] == 0
    out = generate_packed_classic(dasset, params, torch.from_numpy(scalars).cuda(), length is not None,
                                  width is not None, radius_scale)
    torch.cuda.synchronize()
    mine = (out.points.cpu().numpy(), out.point_counts.cpu().numpy().view(np.uint32), out.roots_numpy())
    pts, roots, uvs, counts, _ = reference.generate(reference.handle(asset.buffer), params, radius_scale)
    rplan = reference.classic_plan(length=ref_length, width=ref_width)
    assert rplan.fallback_reasons == []
    info = rplan.info()
    cols = [roots["uv"][:, 1].copy()] * info["ptex"]
    cols += [reference.classic_noise(roots["position"], f) for f in info["pref_noise"]]
    inputs = np.stack(cols, 1) if cols else None
    theirs = reference.classic_apply(rplan, pts, counts, roots, uvs, params.cvs_per_strand, radius_scale, inputs)
    return mine, theirs


def _check_application(asset, params, mine, theirs):
    pts, counts, roots = mine
    rpts, rcounts, rroots, _ = theirs
    P = params.cvs_per_strand
    kept = counts != 0
    assert np.all(counts[kept] == P)
    # the surviving strands, in order, are the reference's compacted set
    assert kept.sum() == rcounts.size
    np.testing.assert_array_equal(roots[kept]["triangle_index"], rroots["triangle_index"])
    sel = np.repeat(kept, P)
    diag = asset.bbox_diagonal()
    err = max_position_error(pts[sel], rpts)
    assert err <= TOL * diag, "max position error %.3g" % (err / diag)
    assert float(np.abs(pts[sel, 3] - rpts[:, 3]).max(initial=0.0)) <= TOL * diag
    return err / diag


def test_cfg5_application_matches_reference(sphere, reference):
    w, asset, _ = sphere
    params = _params(w, strands=20000, cvs=24)
    mine, theirs = _classic_pair(sphere, reference, params, LENGTH, WIDTH,
                                 LENGTH.replace("$v", "map('v.ptx')"), WIDTH)
    rel = _check_application(asset, params, mine, theirs)
    assert mine[1].min() == params.cvs_per_strand  # nothing dropped in this configuration
    print("cfg5-style application: max position error %.3g x bbox diagonal" % rel)


def test_drop_rule_matches_reference(sphere, reference):
    # Scales and widths spread across the 1e-4 thresholds, so strands are
    # dropped by width, by the root-tip chord bound and by the sampled
    # spline length near the threshold.
    w, asset, _ = sphere
    params = _params(w, strands=20000, cvs=16)
    length = "hash($id) * 0.0006"
    width = "hash($id, 7) * 0.0003"
    mine, theirs = _classic_pair(sphere, reference, params, length, width, length, width)
    _check_application(asset, params, mine, theirs)
    dropped = int((mine[1] == 0).sum())
    assert 2000 < dropped < 18000


def test_length_only_keeps_taper_radius(sphere, reference):
    w, asset, _ = sphere
    params = _params(w, strands=5000, cvs=12)
    length = "0.5 + noise($Prefg*6)"
    mine, theirs = _classic_pair(sphere, reference, params, length, None, length, None, radius_scale=2.0)
    _check_application(asset, params, mine, theirs)


def test_serial_generator_path(sphere, reference):
    # P > 128 takes the serial generator and the Classic post-pass.
    w, asset, _ = sphere
    params = _params(w, strands=600, cvs=150)
    length = "hash($id) * 0.0004 + 0.00005"
    mine, theirs = _classic_pair(sphere, reference, params, length, WIDTH, length, WIDTH)
    _check_application(asset, params, mine, theirs)
