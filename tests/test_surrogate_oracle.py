"""The surrogate's CPU oracle (oracle/mlp_reference.py) pinned by central
finite differences in float64 (no BF16 rounding), and its parameter layout
against the library's constants.  Host only."""
import numpy as np

from oracle import mlp_reference as ref


def _header(rng):
    return dict(input_offset=rng.normal(0, 0.1, 8).astype(np.float32),
                input_scale=rng.uniform(0.5, 2.0, 8).astype(np.float32),
                output_offset=np.array([0.3, 0.01], np.float32), output_scale=np.array([0.1, 0.002], np.float32))


def _params(rng):
    p = rng.normal(0, 0.3, ref.PARAMETERS) * ref.used_mask()
    return p


def test_layout_matches_library(nxg_lib):
    from nanoxgen_b200 import _abi
    assert ref.PARAMETERS == _abi.SURROGATE_PARAMETERS
    assert ref.used_mask().sum() == 64 * 9 + 2 * 64 * 65 + 2 * 65


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    header = _header(rng)
    params = _params(rng)
    feats = rng.normal(0, 1, (64, 8)).astype(np.float32)
    targets = np.stack([rng.uniform(0.1, 0.7, 64), rng.uniform(0.009, 0.014, 64)], 1).astype(np.float32)
    loss, grad = ref.loss_and_gradients(params, feats, targets, header, emulate=False)
    used = np.flatnonzero(ref.used_mask())
    pick = rng.choice(used, 60, replace=False)
    h = 1e-6
    for i in pick:
        up, dn = params.copy(), params.copy()
        up[i] += h
        dn[i] -= h
        lu, _ = ref.loss_and_gradients(up, feats, targets, header, emulate=False)
        ld, _ = ref.loss_and_gradients(dn, feats, targets, header, emulate=False)
        fd = (lu - ld) / (2 * h)
        assert abs(fd - grad[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, grad[i])
    assert np.all(grad[~ref.used_mask()] == 0.0)


def test_bf16_rounding_is_nearest_even():
    ulp = 2.0 ** -7  # BF16 spacing in [1, 2)
    x = np.array([1.0, 1.0 + ulp / 2, 1.0 + ulp / 4, 1.0 + 1.5 * ulp, 1.0 + 0.75 * ulp, -2.5], np.float32)
    np.testing.assert_array_equal(ref.bf16(x), [1.0, 1.0, 1.0, 1.0 + 2 * ulp, 1.0 + ulp, -2.5])
