"""Multi-process path on CPU: two gloo ranks shard rays and scenes the way the GPU runs do
(the oracle stands in for the device traversal) and agree on the timing collectives."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

from quarry import dist

ROOT = Path(__file__).resolve().parents[1]


def test_shard_tiles_the_range():
    for count in (0, 1, 7, 10_001):
        for world in (1, 2, 3, 8):
            parts = [dist.shard(count, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == count
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [e - b for b, e in parts]
            assert max(sizes) - min(sizes) <= 1
    got = sorted(s for r in range(3) for s in dist.scene_shard(10, r, 3))
    assert got == list(range(10))
    with pytest.raises(ValueError):
        dist.shard(10, 2, 2)
    assert dist.rank_seed(1000, 0) == 1000 and dist.rank_seed(1000, 2) != dist.rank_seed(1000, 1)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "quarry-gpu_b200"))
    os.environ.update(WORLD_SIZE=str(world), RANK=str(rank), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as tdist

    import oracle
    from quarry import dist as qd
    from quarry import workloads

    r = qd.init(backend="gloo", timeout_s=60)
    assert (r.world, r.rank, r.backend) == (world, rank, "gloo")
    # rays: every rank traces its own contiguous slice over its own replica of the scene
    tris = workloads.terrain(16, 1)
    rays = workloads.down_rays(10_001, 0.0, 16.0, 0.0, 16.0, 100.0, 3)
    b, e = qd.shard(rays.shape[0], rank, world)
    mine = oracle.LBVH("tri", tris).raycast(rays[b:e])
    gathered = [None] * world
    tdist.all_gather_object(gathered, (b, e, mine))
    # scenes: round robin over ranks, per-scene results gathered on every rank
    cfg = workloads.batch_config(terrains=3, clouds=2, tri_range=(500, 2_000),
                                 point_range=(500, 2_000), query_range=(20, 60))
    scenes = cfg.terrains + cfg.clouds
    per = {i: oracle.LBVH(scenes[i].kind, scenes[i].items).closest(scenes[i].closest)
           for i in qd.scene_shard(len(scenes), rank, world)}
    allper = [None] * world
    tdist.all_gather_object(allper, per)
    t = qd.max_over_ranks(r, 1.5 + rank)
    qd.barrier(r)
    if rank == 0:
        full = oracle.LBVH("tri", tris).raycast(rays)
        got = np.concatenate([g[2] for g in sorted(gathered, key=lambda g: g[0])])
        merged = {k: v for d in allper for k, v in d.items()}
        ok = (np.array_equal(got, full) and t == 1.5 + world - 1
              and sorted(merged) == list(range(len(scenes)))
              and all(np.array_equal(merged[i], oracle.LBVH(scenes[i].kind, scenes[i].items)
                                     .closest(scenes[i].closest)) for i in merged))
        Path(out_dir, "result").write_text("ok" if ok else "mismatch")
    qd.destroy(r)


def test_two_gloo_ranks_shard_and_agree(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(rk, world, port, str(tmp_path))) for rk in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a gloo rank did not finish")
        assert p.exitcode == 0
    assert (tmp_path / "result").read_text() == "ok"
