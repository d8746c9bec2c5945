"""The multi-rank host path on CPU: two gloo ranks (world size 2).

Checks what the bench and the batched engines rely on when run with one
process per GPU: every rank generates the same seeded instance list and takes
a disjoint shard, the shards cover the list, MAX over ranks is the slowest
rank's time, and the whole-job rate is all units over that time.  No GPU.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import torch.distributed as tdist

    from ruqu_b200 import dist, workloads
    assert dist.world() == (ws, rank, rank)
    dist.init("gloo", 30.0)
    try:
        inst = workloads.qaoa_instances(24, 2)
        mine = dist.shard(inst, rank, ws)
        keys = [(x["n"], tuple(map(tuple, x["edges"])), tuple(x["gammas"])) for x in mine]
        gathered = [None] * ws
        tdist.all_gather_object(gathered, keys)
        sets = workloads.vqe_parameter_sets(10, 8, 4)
        mine_sets = dist.shard(sets, rank, ws)
        all_sets = [None] * ws
        tdist.all_gather_object(all_sets, mine_sets.tolist())
        t = 10.0 * (rank + 1)
        mx = dist.max_over_ranks(t)
        rate = dist.whole_job_rate(len(inst), t)
        dist.barrier()
        if rank == 0:
            out.put({"gathered": gathered, "all_keys": [(x["n"], tuple(map(tuple, x["edges"])),
                                                          tuple(x["gammas"])) for x in inst],
                      "sets": all_sets, "all_sets": sets.tolist(), "max": mx, "rate": rate})
    finally:
        tdist.destroy_process_group()


def test_two_gloo_ranks_shard_and_time_like_the_bench():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = res["gathered"]
    assert not set(g[0]) & set(g[1])                       # disjoint
    assert sorted(g[0] + g[1]) == sorted(res["all_keys"])  # covering
    merged = [None] * len(res["all_sets"])
    for r in range(ws):
        merged[r::ws] = res["sets"][r]
    assert np.array_equal(np.array(merged), np.array(res["all_sets"]))
    assert res["max"] == 20.0
    assert res["rate"] == pytest.approx(24 / 0.020)


def test_shard_rejects_bad_rank():
    from ruqu_b200.dist import shard
    with pytest.raises(ValueError):
        shard([1, 2, 3], 2, 2)
    assert shard(list(range(7)), 1, 3) == [1, 4]
