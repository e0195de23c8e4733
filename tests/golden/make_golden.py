"""Writes the golden fixtures in this folder from the reference's own CPU
implementation (oracle/_ref/libnxg_ref.so, built from the reference checkout
by oracle/Makefile).  Run here, where the reference exists; the .npz files
are committed so tests on hosts without the reference compare against them.

    python tests/golden/make_golden.py

Each file holds an asset blob built by the reference's build_asset, the
GenerationParams used, a set of strand ids, and generate_packed_cpu's outputs
for those strands (float4 points, RootSample records, root UVs, point
counts) plus make_strand_generation_state for a subset.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from nanoxgen_b200 import fixtures  # noqa: E402
from nanoxgen_b200._abi import GenerationParams  # noqa: E402
from oracle.checker import Reference  # noqa: E402
from helpers import patch_stencil  # noqa: E402


def dump(name, ref, blob, params_list, strand_ids, state_ids, radius_scale=1.0):
    h = ref.handle(blob)
    out = {"asset": blob, "strands": np.asarray(strand_ids, np.uint32),
           "state_strands": np.asarray(state_ids, np.uint32), "radius_scale": np.float32(radius_scale)}
    for k, params in enumerate(params_list):
        pts, roots, uvs, counts, _ = ref.generate(h, params, radius_scale, workers=8)
        P = int(params.cvs_per_strand)
        idx = (np.asarray(strand_ids)[:, None] * P + np.arange(P)[None, :]).reshape(-1)
        out["params%d" % k] = np.frombuffer(bytes(params), np.uint8)
        out["points%d" % k] = pts[idx]
        out["roots%d" % k] = roots[strand_ids].view(np.uint8)
        out["uvs%d" % k] = uvs[strand_ids]
        out["counts%d" % k] = counts[strand_ids]
        states = np.stack([ref.strand_state(h, params, int(s)) for s in state_ids])
        out["states%d" % k] = states.view(np.uint8)
    np.savez_compressed(os.path.join(HERE, name), **out)


def main():
    ref = Reference()
    rng = np.random.default_rng(7)
    # Reference unit fixture (tests/test_main.cpp:39-53) with its test parameters.
    unit = ref.build_asset(fixtures.reference_unit_fixture())
    unit_params = [
        GenerationParams(strand_count=128, cvs_per_strand=7, seed=42),
        GenerationParams(strand_count=257, cvs_per_strand=11, seed=91, noise_amplitude=0.03),
        GenerationParams(strand_count=19, cvs_per_strand=11, seed=117, root_width=0.03, tip_width=0.002,
                         noise_amplitude=0.04, noise_frequency=3.25),
        GenerationParams(strand_count=32, cvs_per_strand=33, seed=173, noise_amplitude=0.24,
                         noise_frequency=2.25, noise_correlation=0.75, noise_preserve_length=0.4),
    ]
    dump("unit_fixture.npz", ref, unit, unit_params, np.arange(19), np.arange(8), radius_scale=1.5)
    # Plain sphere workload (2,048 triangles, 64 guides, K = 4).
    w = fixtures.plain_sphere()
    sphere = patch_stencil(ref.build_asset(w.build_input), 4)
    sphere_params = [w.params, w.params.copy(noise_amplitude=0.0),
                     w.params.copy(noise_mask=0.83, noise_correlation=0.35, noise_preserve_length=0.4)]
    ids = np.sort(rng.choice(w.params.strand_count, 384, replace=False))
    dump("plain_sphere.npz", ref, sphere, sphere_params, ids, ids[:48])
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
