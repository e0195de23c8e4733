"""One process per GPU: the strand range of each rank and the collectives
the benchmark needs around (never inside) the data path.

Strands are independent (generate.h:81-84 derives every random draw from the
global strand id), so a description shards by strand range with no data
exchange: rank r of N generates strands [r*S, (r+1)*S) of an N*S-strand
description through nxg_generate_packed_range.
"""
from __future__ import annotations

import datetime
import os
from typing import Optional, Tuple

import torch
import torch.distributed as dist


def shard(strands_per_rank: int, rank: int) -> Tuple[int, int]:
    """(first strand, strand count) of `rank` for weak scaling."""
    return rank * strands_per_rank, strands_per_rank


def split(total: int, rank: int, world: int) -> Tuple[int, int]:
    """(first strand, strand count) of `rank` when `total` strands are split
    as evenly as possible over `world` ranks (strong scaling)."""
    base, extra = divmod(total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def init(backend: str, device: Optional[torch.device] = None, timeout_s: int = 300) -> Tuple[int, int]:
    """Initialise the default process group from the torchrun environment
    (MASTER_ADDR defaults to 127.0.0.1); returns (rank, world size)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and not dist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        kwargs = {"timeout": datetime.timedelta(seconds=timeout_s)}
        if device is not None and backend == "nccl":
            kwargs["device_id"] = device
        dist.init_process_group(backend, **kwargs)
    return rank, world


def barrier() -> None:
    if dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def max_over_ranks(value: float, device: Optional[torch.device] = None) -> float:
    """The largest `value` of all ranks (timings are reported as the max)."""
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def finalize() -> None:
    if dist.is_initialized():
        dist.destroy_process_group()
