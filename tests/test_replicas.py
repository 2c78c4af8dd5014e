"""Multi-rank host logic on CPU (gloo, world size 2): request sharding,
replica seeds, the max-over-ranks timing reduction, and a rank that fails
before the collective (the survivor's collective ends with an error within
the process group's timeout instead of waiting forever)."""
import os
import socket
from datetime import timedelta

import pytest

from randomfield_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, mode, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
        costs = [5.0, 1.0, 3.0, 3.0, 2.0, 8.0, 1.0]
        shards = replicas.shard_by_cost(costs, world)
        mine = shards[rank]
        if mode == "fail" and rank == 1:
            raise RuntimeError("rank 1 fails before the collective")
        units = sum(costs[i] for i in mine)
        secs = 0.1 * (rank + 1)
        total, slowest = replicas.aggregate(units, secs, dist)
        q.put((rank, "ok", mine, replicas.replica_seed(7, rank), total, slowest))
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        q.put((rank, "error", type(e).__name__, str(e)[:200]))


def _run(mode):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = {}
    for _ in range(2):
        item = q.get(timeout=60)
        out[item[0]] = item
    for p in ps:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    return out


def test_shard_by_cost_is_balanced_and_complete():
    costs = [5.0, 1.0, 3.0, 3.0, 2.0, 8.0, 1.0]
    sh = replicas.shard_by_cost(costs, 2)
    assert sorted(sum(sh, [])) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in sh]
    assert max(loads) - min(loads) <= max(costs) and abs(loads[0] - loads[1]) <= 1.0


def test_two_rank_aggregate_over_gloo():
    out = _run("ok")
    assert out[0][1] == "ok" and out[1][1] == "ok", out
    mine0, mine1 = out[0][2], out[1][2]
    assert sorted(mine0 + mine1) == list(range(7)) and not set(mine0) & set(mine1)
    assert (out[0][3], out[1][3]) == (7, 8)
    assert out[0][4] == out[1][4] == 23.0          # total units: sum over ranks
    assert out[0][5] == out[1][5] == pytest.approx(0.2)  # slowest rank


def test_failed_rank_ends_the_survivors_collective_with_an_error():
    out = _run("fail")
    assert out[1][1] == "error"
    assert out[0][1] == "error", out[0]  # no hang: the collective fails within the timeout
