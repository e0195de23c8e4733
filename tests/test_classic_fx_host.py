"""Host-side checks of the Classic FX entry points without a GPU.

nxg_classic_fx_plan_upload packs the plan on the host and then copies it to
the device: on a machine without a device a well-formed plan gets through the
packing to the copy, which fails with the CUDA error, while a malformed plan
is refused before it with InvalidArgument.  The argument checks of
nxg_classic_fx_apply and nxg_classic_clump_prepare run before any launch.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.skipif(torch.cuda.is_available(),
                                reason="tells packing from copying by the copy's failure without a device")

NOISE = dict(mask="1", magnitude="0.05", magnitudeScale="1", frequency="4", correlation="20", preserveLength="0")
CLUMP = dict(mask="1", clump="0.8", clumpScale="0.2*rampUI(0,0,1:1,1,1)", noise="0.05*rand()", noiseScale="1",
             noiseFrequency="5", noiseCorrelation="20")
FAKE_DEVICE = 1 << 20  # never dereferenced: the copy fails first without a device


def _codes():
    from nanoxgen_b200._abi import ERRORS
    return ERRORS


def _upload(desc):
    from nanoxgen_b200._abi import lib
    return lib().nxg_classic_fx_plan_upload(ctypes.byref(desc), FAKE_DEVICE, lib().nxg_classic_fx_plan_bytes(), None)


@pytest.mark.parametrize("effects", [
    [("noise", NOISE)],
    [("cut", {"amount": "$cLength*0.2"})],
    [("clump", CLUMP)],
    [("noise", NOISE), ("clump", CLUMP), ("cut", {"amount": "0.1"}), ("clump", CLUMP), ("noise", NOISE)],
])
def test_well_formed_plans_pack(nxg_lib, effects):
    from nanoxgen_b200.classic import FxPlan
    plan = FxPlan({"length": "0.8", "width": "0.01", "taper": "0.5", "widthRamp": "rampUI(0,1,1:1,0.5,1)"},
                  effects, 3, "desc:a")
    assert _upload(plan.descriptor()) == _codes()["Cuda"]


def test_malformed_plans_are_refused(nxg_lib):
    from nanoxgen_b200 import _abi
    from nanoxgen_b200.classic import FxPlan
    invalid = _codes()["InvalidArgument"]
    for kind, values in (("noise", NOISE), ("clump", CLUMP)):
        plan = FxPlan({}, [(kind, values)])
        desc = plan.descriptor()
        fx = desc.effects[0]
        for name, _ in _abi.ClassicFx._fields_[2:]:
            if getattr(fx, name) is None:
                continue
            saved = getattr(fx, name)
            setattr(fx, name, None)  # a required attribute missing
            assert _upload(desc) == invalid, (kind, name)
            setattr(fx, name, saved)
        assert _upload(desc) == _codes()["Cuda"]
        fx.type = 3  # no such module
        assert _upload(desc) == invalid
    plan = FxPlan({}, [("cut", {"amount": "0.1"})] * 8)
    desc = plan.descriptor()
    desc.effect_count = 9
    assert _upload(desc) == invalid


def test_plan_reports_rand_and_clumps(nxg_lib):
    from nanoxgen_b200.classic import FxPlan
    assert not FxPlan({"length": "0.5"}, [("noise", NOISE)]).uses_random
    plan = FxPlan({}, [("clump", CLUMP), ("cut", {"amount": "0.1"}), ("clump", dict(CLUMP, noise="0"))])
    assert plan.uses_random and plan.clump_count == 2


def test_apply_and_prepare_argument_checks(nxg_lib):
    from nanoxgen_b200 import _abi
    lib = _abi.lib()
    invalid = _codes()["InvalidArgument"]
    status = ctypes.c_uint32 * 2
    curves = _abi.ClassicFxCurves(FAKE_DEVICE, FAKE_DEVICE, FAKE_DEVICE, None, None, 10, 16, 0, 1.0, None, None, 0,
                                  0)
    guides = (_abi.ClassicClumpGuides * 9)()
    curves.clumps = guides
    curves.clump_count = 9  # more clump modules than a plan holds
    assert lib.nxg_classic_fx_apply(FAKE_DEVICE, ctypes.byref(curves), ctypes.addressof(status()), None) == invalid
    curves.clump_count = 1  # a module whose strand guides are missing
    assert lib.nxg_classic_fx_apply(FAKE_DEVICE, ctypes.byref(curves), ctypes.addressof(status()), None) == invalid
    guides[0].strand_guides = FAKE_DEVICE
    guides[0].guide_count = 4  # with guides but no guide arrays
    assert lib.nxg_classic_fx_apply(FAKE_DEVICE, ctypes.byref(curves), ctypes.addressof(status()), None) == invalid
    for cvs in (2, 65):
        assert lib.nxg_classic_clump_prepare(FAKE_DEVICE, 4, cvs, FAKE_DEVICE, FAKE_DEVICE, None) == invalid
    assert lib.nxg_classic_clump_prepare(None, 0, 8, None, None, None) == _codes()["None"]
    axes = np.zeros((4, 8, 3), np.float32)
    assert lib.nxg_classic_clump_prepare(axes.ctypes.data, 4, 8, None, None, None) == invalid
