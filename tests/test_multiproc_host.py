"""The multi-process paths of bench.py on CPU (gloo, world size 2): cost-balanced ensemble
sharding, the barrier, the max-over-ranks timing reduction, and the reference arm's
rank-0-only rule.  No GPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        inst = [{"n": n} for n, c in bench.ENSEMBLE_MIXED for _ in range(c)]
        shards = bench.shard_by_cost(inst, world)
        bench.barrier(world)
        t = bench.max_over_ranks(1.5 + rank, world)          # each rank's "time"
        args = type("A", (), {"gpus": world, "steps": 1, "warmup": 3})()
        ref_rc = bench.run_reference(args) if rank != 0 else None   # non-zero ranks return at once
        out.put((rank, [len(sh) for sh in shards], sum(len(sh) for sh in shards), t, ref_rc))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_timing():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    counts = {tuple(r[1]) for r in res}
    assert len(counts) == 1                      # every rank computes the same partition
    assert res[0][2] == 128 + 256 + 32           # all instances, each once
    assert all(r[3] == 2.5 for r in res)         # max over ranks
    assert res[1][4] == 0                        # the reference arm: only rank 0 works


def test_cost_balance():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import math
    import bench
    inst = [{"n": n, "id": k} for k, (n, c) in enumerate(bench.ENSEMBLE_MIXED) for _ in range(c)]
    for world in (2, 3, 4, 8):
        shards = bench.shard_by_cost(inst, world)
        assert sorted(id(i) for sh in shards for i in sh) == sorted(id(i) for i in inst)
        cost = [sum(i["n"] ** 2 * math.log2(i["n"]) for i in sh) for sh in shards]
        biggest = max(i["n"] ** 2 * math.log2(i["n"]) for i in inst)
        assert max(cost) - min(cost) <= biggest
