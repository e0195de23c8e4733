"""Host-side checks of nxg_build_curve_batches against the reference's
build_curve_batches (src/curve_payload.cpp:142-211): every check the host can
make returns the reference's message, in the reference's order.  The calls
carry device pointers that are never dereferenced (each case fails on the
host first), so the file runs only where no device is present."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.skipif(torch.cuda.is_available(), reason="host-only failure paths with placeholder pointers")

FAKE = 1 << 20
IDENTITY = (1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0)


def _host_error(base, samples=(), per_batch=64, resample=0, radius_scale=1.0, transform=IDENTITY):
    from nanoxgen_b200._abi import (ERRORS, CurveSet, MotionSet, PayloadOptions, PayloadOutput, lib)
    desc = CurveSet(base["strands"], base.get("fixed", 0), FAKE if base.get("counts") is not None else None, FAKE,
                    base["n"], FAKE if base.get("widths") else None, None, None, base.get("constant_width", 0.1), 0)
    motion = (MotionSet * max(1, len(samples)))(*(
        MotionSet(t, 0, CurveSet(c["strands"], c.get("fixed", 0), FAKE if c.get("counts") is not None else None,
                                 FAKE, c["n"], None, None, None, c.get("constant_width", 0.1), 0))
        for t, c in samples))
    options = PayloadOptions(per_batch, resample, radius_scale, (ctypes.c_float * 12)(*transform))
    out = PayloadOutput(FAKE, FAKE, None, FAKE, FAKE)
    status = (ctypes.c_uint32 * 2)()
    host_error = ctypes.c_uint32()
    code = lib().nxg_build_curve_batches(ctypes.byref(desc), motion, len(samples), ctypes.byref(options),
                                         ctypes.byref(out), FAKE, 1 << 30, ctypes.addressof(status),
                                         ctypes.byref(host_error), None)
    assert code == ERRORS["InvalidArgument"], code
    return lib().nxg_payload_error_message(host_error.value).decode()


def _reference_error(reference, base, samples=(), **kw):
    def arrays(d):
        n = d["n"]
        out = dict(points=np.zeros((n, 3)), strands=d["strands"], fixed=d.get("fixed", 0),
                   constant_width=d.get("constant_width", 0.1))
        if d.get("widths"):
            out["widths"] = np.ones(n)
        return out
    with pytest.raises(ValueError) as e:
        reference.build_curve_batches(arrays(base), [(t, arrays(c)) for t, c in samples], **kw)
    return str(e.value)


FIXED = dict(strands=4, fixed=3, n=12)
CASES = [
    ("no strand limit", dict(base=FIXED, per_batch=0)),
    ("resample to one CV", dict(base=FIXED, resample=1)),
    ("negative radius scale", dict(base=FIXED, radius_scale=-1.0)),
    ("nan radius scale", dict(base=FIXED, radius_scale=float("nan"))),
    ("no strands", dict(base=dict(strands=0, fixed=3, n=0))),
    ("no counts", dict(base=dict(strands=4, fixed=1, n=4))),
    ("point size", dict(base=dict(strands=4, fixed=3, n=11))),
    ("constant width", dict(base=dict(FIXED, constant_width=-0.5))),
    ("strand limit before width", dict(base=dict(FIXED, constant_width=-0.5), per_batch=0)),
    ("motion time", dict(base=FIXED, samples=[(float("nan"), FIXED)])),
    ("motion strands", dict(base=FIXED, samples=[(0.5, dict(strands=3, fixed=4, n=12))])),
    ("motion counts", dict(base=FIXED, samples=[(0.5, dict(strands=4, fixed=0, n=12))])),
    ("motion point size", dict(base=FIXED, samples=[(0.5, dict(strands=4, fixed=3, n=13))])),
    ("motion width", dict(base=FIXED, samples=[(0.5, dict(FIXED, constant_width=float("inf")))])),
    ("second sample", dict(base=FIXED, samples=[(0.5, FIXED), (0.6, dict(strands=4, fixed=3, n=1))])),
    ("transform", dict(base=FIXED, transform=(1, 0, 0, float("inf"), 0, 1, 0, 0, 0, 0, 1, 0))),
    ("base before transform", dict(base=dict(strands=4, fixed=3, n=2),
                                   transform=(float("nan"),) + IDENTITY[1:])),
]


@pytest.mark.parametrize("name,case", CASES, ids=[c[0] for c in CASES])
def test_host_checks_match_reference(nxg_lib, reference, name, case):
    kw = {k: v for k, v in case.items() if k not in ("base", "samples")}
    samples = case.get("samples", ())
    assert _host_error(case["base"], samples, **kw) == _reference_error(reference, case["base"], samples, **kw)
