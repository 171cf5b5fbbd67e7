"""The multi-GPU host logic (independent replicas) with two gloo ranks on
the CPU: the job split covers every job once, the cost-balanced split is
the same on every rank and balanced, and the max/sum over ranks and the
barrier behave as the bench uses them."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from vcl_b200 import replicas


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    n, r = replicas.init("gloo", timeout_s=60)
    assert (n, r) == (world, rank)
    rr = replicas.shard(len(costs), r, n)
    lpt = replicas.shard_by_cost(costs, r, n)
    replicas.barrier()
    mx = replicas.max_over_ranks(10.0 + r)            # per-rank "time"
    tot = replicas.sum_over_ranks(sum(costs[i] for i in lpt))
    out.put((r, rr, lpt, mx, tot))
    replicas.finish()


def test_two_gloo_ranks_split_jobs_and_reduce():
    world = 2
    costs = [5.0, 1.0, 3.0, 8.0, 2.0, 2.0, 7.0]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rr = [x[1] for x in res]
    lpt = [x[2] for x in res]
    assert sorted(rr[0] + rr[1]) == list(range(len(costs))) and not set(rr[0]) & set(rr[1])
    assert sorted(lpt[0] + lpt[1]) == list(range(len(costs))) and not set(lpt[0]) & set(lpt[1])
    loads = [sum(costs[i] for i in l) for l in lpt]
    assert max(loads) - min(loads) <= max(costs)
    assert all(x[3] == 11.0 for x in res)          # max over ranks
    assert all(x[4] == sum(costs) for x in res)    # sum over ranks


def test_single_process_helpers_need_no_group():
    assert replicas.shard(5, 0, 1) == [0, 1, 2, 3, 4]
    assert replicas.shard_by_cost([1.0, 2.0], 0, 1) == [0, 1]
    assert replicas.max_over_ranks(3.5) == 3.5
    replicas.barrier()
