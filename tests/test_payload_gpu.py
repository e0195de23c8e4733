"""nxg_build_curve_batches on the device against the reference's
build_curve_batches (src/curve_payload.cpp): point counts, float4 points,
root uvs, motion positions and batch boundaries bit for bit (the reference's
batches concatenated), for fixed and variable CV counts, copies and
resampling, identity and affine transforms, widths and constant widths, root
uvs from either source, motion samples with their own counts; the device
count checks report the reference's first error."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

AFFINE = (0.9, -0.2, 0.1, 0.5, 0.3, 1.1, -0.4, -2.0, 0.05, 0.2, 0.8, 1.25)


def _curves(rng, strands, counts=None, fixed=0, widths=True, uvs=False, roots=False, constant_width=0.0):
    n = int(np.sum(counts)) if counts is not None else strands * fixed
    d = dict(points=rng.normal(size=(n, 3)).astype(np.float32), strands=strands, fixed=fixed,
             constant_width=constant_width)
    if counts is not None:
        d["counts"] = np.asarray(counts, np.uint32)
    if widths:
        d["widths"] = (rng.random(n) * 0.02).astype(np.float32)
    if uvs:
        d["root_uvs"] = rng.random((strands, 2)).astype(np.float32)
    if roots:
        r = np.zeros((strands, 12), np.float32)
        r[:, 6:8] = rng.random((strands, 2))
        d["roots"] = r
    return d


def _device(d):
    import torch

    from nanoxgen_b200.payload import Curves
    dev = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return Curves(points=dev(d["points"]), strand_count=d["strands"], fixed_cvs_per_strand=d["fixed"],
                  point_counts=dev(None if d.get("counts") is None else d["counts"].view(np.int32)),
                  widths=dev(d.get("widths")), root_uvs=dev(d.get("root_uvs")), roots=dev(d.get("roots")),
                  constant_width=d["constant_width"])


def _compare(reference, base, samples=(), **kw):
    import torch

    from nanoxgen_b200.payload import build_curve_batches
    theirs = reference.build_curve_batches(
        {k: (v.view(np.uint8) if k == "roots" else v) for k, v in base.items()},
        [(t, s) for t, s in samples], per_batch=kw.get("max_strands_per_batch", 65536),
        resample=kw.get("resample_cv_count", 0), radius_scale=kw.get("radius_scale", 1.0),
        transform=kw.get("transform", (1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0)))
    mine = build_curve_batches(_device(base), [(t, _device(s)) for t, s in samples], **kw)
    torch.cuda.synchronize()
    assert mine.error() == ""
    total = theirs["points"].shape[0]
    bits = lambda a: np.ascontiguousarray(a).view(np.uint32)
    np.testing.assert_array_equal(mine.point_counts.cpu().numpy().view(np.uint32), theirs["point_counts"])
    np.testing.assert_array_equal(bits(mine.points.cpu().numpy()[:total]), bits(theirs["points"]))
    np.testing.assert_array_equal(mine.batch_first_point.cpu().numpy().view(np.uint64), theirs["batch_first_point"])
    if theirs["root_uvs"] is not None:
        np.testing.assert_array_equal(bits(mine.root_uvs.cpu().numpy()), bits(theirs["root_uvs"]))
    if samples:
        np.testing.assert_array_equal(bits(mine.motion_points.cpu().numpy()[:len(samples) * total]),
                                      bits(theirs["motion_points"]))
    return mine, theirs


def test_fixed_copy_with_motion(cuda, nxg_lib, reference):
    rng = np.random.default_rng(1)
    base = _curves(rng, 5000, fixed=12, uvs=True)
    samples = [(0.25, _curves(rng, 5000, fixed=12)), (0.75, _curves(rng, 5000, fixed=12))]
    _compare(reference, base, samples, max_strands_per_batch=1024, radius_scale=0.7)


@pytest.mark.parametrize("transform", [None, AFFINE])
def test_fixed_copy_batches_straddle_quads(cuda, nxg_lib, reference, transform):
    # The flat path with 35-point batches (7 strands x 5 CVs) and an odd
    # total: four-point groups cross batch boundaries and the end.
    rng = np.random.default_rng(6)
    base = _curves(rng, 1001, fixed=5, widths=False, roots=True, constant_width=0.02)
    samples = [(0.1, _curves(rng, 1001, fixed=5)), (0.9, _curves(rng, 1001, fixed=5))]
    kw = dict(max_strands_per_batch=7)
    if transform:
        kw["transform"] = transform
    _compare(reference, base, samples, **kw)


def test_variable_resample_transform(cuda, nxg_lib, reference):
    rng = np.random.default_rng(2)
    counts = rng.integers(2, 70, 20000)
    base = _curves(rng, 20000, counts=counts, widths=False, roots=True, constant_width=0.013)
    other = rng.integers(2, 70, 20000)
    samples = [(0.0, _curves(rng, 20000, counts=other)), (0.5, _curves(rng, 20000, fixed=9)),
               (1.0, _curves(rng, 20000, counts=counts))]
    _compare(reference, base, samples, max_strands_per_batch=777, resample_cv_count=16, radius_scale=1.5,
             transform=AFFINE)


def test_variable_copy_counts_differ_per_sample(cuda, nxg_lib, reference):
    # Without resampling a sample whose strand has another count is resampled
    # to the base's count; one with the same count is copied.
    rng = np.random.default_rng(3)
    counts = rng.integers(2, 40, 70000)
    other = counts.copy()
    other[::3] = rng.integers(2, 40, other[::3].size)
    base = _curves(rng, 70000, counts=counts, uvs=True)
    _compare(reference, base, [(0.1, _curves(rng, 70000, counts=other))], transform=AFFINE)


def test_single_batch_and_tiny_batches(cuda, nxg_lib, reference):
    rng = np.random.default_rng(4)
    counts = rng.integers(2, 6, 333)
    base = _curves(rng, 333, counts=counts)
    _compare(reference, base, max_strands_per_batch=1)
    _compare(reference, base, max_strands_per_batch=333, resample_cv_count=2)


def test_generated_frame(cuda, nxg_lib, reference):
    # The generator's own output as the payload source: 200,000 strands x 24
    # CVs of the large description, positions and radii (widths = 2 radius).
    import torch

    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import DeviceAsset, generate_packed
    w = fixtures.large_sphere(strands=200_000, cvs=24)
    out = generate_packed(DeviceAsset(build_asset(w.build_input, w.stencil_slots), cuda), w.params)
    torch.cuda.synchronize()
    pts = out.points.cpu().numpy()
    base = dict(points=np.ascontiguousarray(pts[:, :3]), strands=200_000, fixed=24,
                widths=np.ascontiguousarray(2.0 * pts[:, 3]), root_uvs=out.root_uvs.cpu().numpy(),
                constant_width=0.0)
    _compare(reference, base, max_strands_per_batch=65536, resample_cv_count=8, transform=AFFINE)


@pytest.mark.parametrize("case", ["short base", "base size", "short motion", "host after device"])
def test_device_checks_report_the_first_error(cuda, nxg_lib, reference, case):
    import torch

    from nanoxgen_b200.payload import build_curve_batches
    rng = np.random.default_rng(5)
    counts = rng.integers(2, 9, 3000)
    base = _curves(rng, 3000, counts=counts)
    samples = [(0.5, _curves(rng, 3000, counts=counts))]
    if case == "short base":
        base["counts"][17] = 1
        samples[0][1]["counts"][5] = 0
    elif case == "base size":
        base["points"] = base["points"][:-1]
        base["widths"] = base["widths"][:-1]
    elif case == "short motion":
        samples[0][1]["counts"][99] = 1
    else:  # valid counts, a non-finite sample time: reported after the device checks pass
        samples = [(float("nan"), samples[0][1])]
    with pytest.raises(ValueError) as e:
        reference.build_curve_batches(base, samples)
    mine = build_curve_batches(_device(base), [(t, _device(s)) for t, s in samples])
    torch.cuda.synchronize()
    assert mine.error() == str(e.value)
