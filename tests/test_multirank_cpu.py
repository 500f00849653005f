"""Multi-rank host logic on CPU (gloo, world size 2): the batch is sharded by cloth with no collective inside a step,
every cloth is owned by exactly one rank, the shards are balanced by constraint count, and timing is reduced as the
max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        w = bench.make_workload("c3", rank, world)
        ids = torch.tensor([s.meta["seed"] for s in w["specs"]], dtype=torch.int64)
        sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(sizes, torch.tensor([len(ids)]))
        gathered = [torch.zeros(int(sz.item()), dtype=torch.int64) for sz in sizes]
        dist.all_gather(gathered, ids)
        # max-over-ranks timing as bench.py reduces it (gloo has MAX too)
        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        out[rank] = dict(seeds=sorted(torch.cat(gathered).tolist()), n=w["n"], e=w["e"], total=w["total_cloths"],
                         tmax=float(t.item()), mine=len(ids))
    finally:
        dist.destroy_process_group()


def test_cloth_sharding_two_ranks():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    r0, r1 = out[0], out[1]
    assert r0["seeds"] == r1["seeds"]                       # both ranks see the same global set
    assert len(set(r0["seeds"])) == 256 == r0["total"]      # every cloth exactly once
    assert r0["mine"] + r1["mine"] == 256
    assert abs(r0["e"] - r1["e"]) / max(r0["e"], r1["e"]) < 0.05  # constraint balance of the shards
    assert r0["tmax"] == r1["tmax"] == 2.0


def test_shard_by_constraints_balances_and_covers():
    from bevy_xpbd_b200 import workloads as wl
    from bevy_xpbd_b200.sharding import shard_by_constraints
    counts = [s.num_constraints for s in wl.config3_batch()]
    for world in (1, 2, 4, 8):
        shards = shard_by_constraints(counts, world)
        assert sorted(k for s in shards for k in s) == list(range(len(counts)))
        loads = [sum(counts[k] for k in s) for s in shards]
        assert (max(loads) - min(loads)) / max(loads) < 0.05, (world, loads)
    assert shard_by_constraints([5, 3, 3, 1], 2) == [[0, 3], [1, 2]]
