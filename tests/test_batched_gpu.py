"""Several descriptions in one persistent launch (nxg_generate_batched)
against the oracle per description, and against single-description
generation."""
import numpy as np
import pytest

from helpers import max_position_error

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch(cuda, nxg_lib):
    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import DeviceAsset
    b = fixtures.batched_descriptions(count=7, n_lon=80, n_rings=41, strands=(300, 6000), guides=(40, 160), seed=7)
    assets = [build_asset(w.build_input, w.stencil_slots) for w in b.workloads]
    return b, assets, [DeviceAsset(a, cuda) for a in assets]


def test_batched_matches_oracle_per_description(batch, oracle):
    import torch

    from nanoxgen_b200.generator import BatchRunner
    b, assets, dassets = batch
    cvs = sorted({int(w.params.cvs_per_strand) for w in b.workloads})
    assert len(cvs) >= 4 and any(w.params.noise_amplitude == 0 for w in b.workloads)
    runner = BatchRunner(dassets, [w.params for w in b.workloads], radius_scale=1.25)
    runner.run()
    torch.cuda.synchronize()
    for w, asset, out in zip(b.workloads, assets, runner.curves()):
        pts, roots, uvs, counts = oracle.generate(asset.buffer, w.params, 1.25, threads=8)
        mine = out.points.cpu().numpy()
        assert max_position_error(mine, pts) <= 1e-5 * asset.bbox_diagonal(), w.name
        assert float(np.abs(mine[:, 3] - pts[:, 3]).max()) <= 1e-5 * asset.bbox_diagonal()
        assert out.roots_numpy().tobytes() == roots.tobytes(), w.name
        assert np.array_equal(out.point_counts.cpu().numpy().view(np.uint32), counts)
        assert np.array_equal(out.root_uvs.cpu().numpy(), uvs)


def test_batched_graph_replay_and_single_description_agreement(batch):
    import torch

    from nanoxgen_b200.generator import BatchRunner, generate_packed
    b, assets, dassets = batch
    runner = BatchRunner(dassets, [w.params for w in b.workloads])
    runner.run()
    torch.cuda.synchronize()
    eager = [c.points.clone() for c in runner.curves()]
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        runner.run(stream=s)
    for c in runner.curves():
        c.points.zero_()
    g.replay()
    torch.cuda.synchronize()
    for c, e, w, d, a in zip(runner.curves(), eager, b.workloads, dassets, assets):
        assert torch.equal(c.points, e)
        single = generate_packed(d, w.params)
        torch.cuda.synchronize()
        assert max_position_error(single.points.cpu().numpy(), e.cpu().numpy()) <= 1e-5 * a.bbox_diagonal()


def test_batched_classic_matches_single_description_classic(batch):
    # nxg_generate_batched_classic with per-description Classic scalars (one
    # description left without) against nxg_generate_packed_classic per
    # description: identical drop decisions and point counts, positions and
    # radii within 1e-5 of the bounding-box diagonal.
    import torch

    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.classic import Expression, ScalarPlan, generate_packed_classic, root_scalars
    from nanoxgen_b200.generator import BatchRunner, generate_packed
    b, assets, dassets = batch
    plan = ScalarPlan(Expression.classic("hash($id) * 0.0005 + " + fixtures.CLASSIC_LENGTH, "length"),
                      Expression.classic("hash($id, 3) * 0.0002 + 0.00005", "width"))
    params = [w.params for w in b.workloads]
    scalars = [root_scalars(d, p, plan)[0] for d, p in zip(dassets, params)]
    scalars[2] = None
    runner = BatchRunner(dassets, params)
    runner.run(scalars=scalars)
    torch.cuda.synchronize()
    dropped = 0
    for i, (c, d, p, a) in enumerate(zip(runner.curves(), dassets, params, assets)):
        if scalars[i] is None:
            single = generate_packed(d, p)
        else:
            single = generate_packed_classic(d, p, scalars[i])
        torch.cuda.synchronize()
        assert torch.equal(c.point_counts, single.point_counts), i
        dropped += int((c.point_counts == 0).sum())
        diag = a.bbox_diagonal()
        assert max_position_error(c.points.cpu().numpy(), single.points.cpu().numpy()) <= 1e-5 * diag
        assert float((c.points[:, 3] - single.points[:, 3]).abs().max()) <= 1e-5 * diag
    assert dropped > 0
