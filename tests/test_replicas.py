"""Replica bookkeeping of the multi-GPU path, run as two gloo ranks on the CPU
(the physics itself has no collective)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mjb200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = replicas.reduce_over_ranks(1.5 + rank, "max")
        s = replicas.reduce_over_ranks(1.0 + rank, "sum")
        out.put((rank, t, s, replicas.rank_seeds(rank), replicas.shard(1001, world, rank)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.5, 2.5]           # max over ranks seen by every rank
    assert [r[2] for r in res] == [3.0, 3.0]
    assert res[0][3] != res[1][3]                       # replicas step different envs
    (o0, c0), (o1, c1) = res[0][4], res[1][4]
    assert (o0, c0, o1, c1) == (0, 501, 501, 500)


@pytest.mark.parametrize("total,world", [(16384, 8), (7, 3), (1, 4), (0, 2)])
def test_shards_cover_batch(total, world):
    seen = []
    for r in range(world):
        o, c = replicas.shard(total, world, r)
        seen += list(range(o, o + c))
    assert seen == list(range(total))


def test_single_process_identity():
    assert replicas.reduce_over_ranks(3.25) == 3.25
