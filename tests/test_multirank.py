"""The N-GPU path's host logic on CPU: two gloo ranks shard one description
by strand range (no data-path collective), the shards reproduce the
single-process result exactly, and timings reduce as the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

S_PER_RANK = 700


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch
    import torch.distributed as dist

    from nanoxgen_b200 import distributed, fixtures
    from nanoxgen_b200.asset import build_asset
    from oracle.checker import Oracle

    r, n = distributed.init("gloo", timeout_s=60)
    assert (r, n) == (rank, world)
    w = fixtures.plain_sphere(strands=S_PER_RANK * world)
    asset = build_asset(w.build_input, w.stencil_slots)
    first, count = distributed.shard(S_PER_RANK, rank)
    pts, roots, _, _ = Oracle().generate(asset.buffer, w.params, first=first, count=count)
    distributed.barrier()
    gathered = [torch.zeros(count * w.params.cvs_per_strand, 4) for _ in range(world)]
    dist.all_gather(gathered, torch.from_numpy(pts))
    slowest = distributed.max_over_ranks(float(rank + 1))
    if rank == 0:
        np.save(os.path.join(out_dir, "sharded.npy"), torch.cat(gathered).numpy())
        np.save(os.path.join(out_dir, "max.npy"), np.array([slowest]))
    distributed.finalize()


def test_two_rank_strand_sharding(tmp_path, nxg_lib, oracle):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    w = fixtures.plain_sphere(strands=S_PER_RANK * world)
    whole, _, _, _ = oracle.generate(build_asset(w.build_input, w.stencil_slots).buffer, w.params, threads=4)
    assert np.array_equal(np.load(tmp_path / "sharded.npy"), whole)
    assert float(np.load(tmp_path / "max.npy")[0]) == 2.0


def _device_rank_main(rank, world, port, out_dir):
    """One rank of the device test: its strand range through
    nxg_generate_packed_range on cuda:0, gathered to rank 0 over gloo."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch
    import torch.distributed as dist

    from nanoxgen_b200 import distributed, fixtures
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import DeviceAsset, generate_packed

    r, n = distributed.init("gloo", timeout_s=120)
    assert (r, n) == (rank, world)
    torch.cuda.set_device(0)
    w = fixtures.large_sphere(strands=DEVICE_S_PER_RANK * world, cvs=32)
    asset = build_asset(w.build_input, w.stencil_slots)
    first, count = distributed.shard(DEVICE_S_PER_RANK, rank)
    out = generate_packed(DeviceAsset(asset, "cuda"), w.params, first_strand=first, count=count)
    torch.cuda.synchronize()
    pts = out.points.cpu()
    rts = out.roots.cpu()
    distributed.barrier()
    gathered = [torch.zeros_like(pts) for _ in range(world)]
    gathered_roots = [torch.zeros_like(rts) for _ in range(world)]
    dist.all_gather(gathered, pts)
    dist.all_gather(gathered_roots, rts)
    if rank == 0:
        np.save(os.path.join(out_dir, "points.npy"), torch.cat(gathered).numpy())
        np.save(os.path.join(out_dir, "roots.npy"), torch.cat(gathered_roots).numpy())
    distributed.finalize()


DEVICE_S_PER_RANK = 150_000


@pytest.mark.gpu
def test_two_ranks_generate_their_ranges_on_the_device(tmp_path, cuda, nxg_lib):
    """The product path of the N-GPU bench: two ranks (both on cuda:0; no
    kernel waits on another rank) generate their strand ranges with
    nxg_generate_packed_range; the gathered shards equal one process's
    whole-description generation bit for bit."""
    import torch

    from nanoxgen_b200 import fixtures
    from nanoxgen_b200.asset import build_asset
    from nanoxgen_b200.generator import DeviceAsset, generate_packed
    world = 2
    mp.start_processes(_device_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    w = fixtures.large_sphere(strands=DEVICE_S_PER_RANK * world, cvs=32)
    whole = generate_packed(DeviceAsset(build_asset(w.build_input, w.stencil_slots), cuda), w.params)
    torch.cuda.synchronize()
    assert np.array_equal(np.load(tmp_path / "points.npy").view(np.uint32), whole.points.cpu().numpy().view(np.uint32))
    assert np.array_equal(np.load(tmp_path / "roots.npy"), whole.roots.cpu().numpy())


@pytest.mark.parametrize("total,world", [(10, 3), (1_000_000, 8), (7, 8)])
def test_even_split_covers_every_strand_once(total, world):
    from nanoxgen_b200.distributed import split
    ranges = [split(total, r, world) for r in range(world)]
    assert sum(c for _, c in ranges) == total
    assert all(ranges[i][0] + ranges[i][1] == ranges[i + 1][0] for i in range(world - 1))
    assert max(c for _, c in ranges) - min(c for _, c in ranges) <= 1
