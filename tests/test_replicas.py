"""Replica plumbing of the multi-GPU bench on CPU: two gloo ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from pdcs_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    r, w, _ = replicas.env()
    replicas.init(w, timeout_s=60)
    replicas.barrier(w)
    t = replicas.max_over_ranks(1.5 + r, w)          # rank times 1.5 s and 2.5 s
    work = replicas.sum_over_ranks(100 * (r + 1), w)  # 100 + 200 units
    mine = replicas.shard(list(range(7)), r, w)
    allsh = [None] * w
    import torch.distributed as dist
    dist.all_gather_object(allsh, mine)
    replicas.finalize(w)
    out.put((r, t, work, mine, allsh))


def test_two_rank_aggregation_and_shards():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, t, work, mine, allsh in res:
        assert t == 2.5            # the job's time is the slowest rank's
        assert work == 300.0       # work adds up over ranks
        assert mine == list(range(r, 7, 2))
        flat = sorted(i for s in allsh for i in s)
        assert flat == list(range(7))  # every instance on exactly one rank


def test_single_process_is_identity():
    assert replicas.max_over_ranks(3.0, 1) == 3.0
    assert replicas.sum_over_ranks(4.0, 1) == 4.0
    assert replicas.shard([1, 2, 3], 0, 1) == [1, 2, 3]
