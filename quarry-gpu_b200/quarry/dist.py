"""Process-per-GPU plumbing for the engine's multi-GPU runs.

One process per GPU (launched by torchrun; RANK / LOCAL_RANK / WORLD_SIZE / MASTER_* from the
environment), torch.distributed over NCCL on GPUs, or gloo on CPU for the host-side tests.
The hot path's units are independent -- rays, query points, whole scenes -- so ranks shard
them with no data-path collective: every rank builds its own replica of a scene (a build
takes milliseconds) and works on its own slice.  The only collectives are a barrier around a
timed region and a maximum over ranks of the measured time.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Ranks:
    world: int
    rank: int
    local: int
    backend: str | None  # None when world == 1 (no process group)


def init(backend: str | None = None, timeout_s: float = 120.0) -> Ranks:
    """Joins the process group described by the environment (world 1: no group)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return Ranks(1, 0, 0, None)
    import torch
    import torch.distributed as dist

    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    kw = {}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return Ranks(world, rank, local, backend)


def barrier(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(r: Ranks, value: float) -> float:
    """The maximum of `value` over all ranks (every rank gets it)."""
    if r.world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    dev = "cuda" if r.backend == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def destroy(r: Ranks) -> None:
    if r.world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def shard(count: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [begin, end) slice of `count` units for `rank`; sizes differ by at most 1
    and the slices tile [0, count) in rank order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(count, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def scene_shard(scenes: int, rank: int, world: int) -> list[int]:
    """Scenes of a batch for `rank`: round robin, so uneven scene sizes spread over ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(range(rank, scenes, world))


def rank_seed(base: int, rank: int, stride: int = 100_000) -> int:
    """Seed of a rank's own synthetic inputs under weak scaling (rank 0 keeps `base`)."""
    return base + stride * rank
