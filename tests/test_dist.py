"""Replica plumbing on CPU: two gloo ranks agree on the max-over-ranks time and the
read shards tile the input exactly once."""
import os
import socket

import pytest

from phraya_b200 import dist as R


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world_size, port, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size, timeout=datetime.timedelta(seconds=60))
    try:
        R.barrier()
        got = R.max_over_ranks(10.0 + rank * 5.0)
        out.put((rank, got, R.world(), R.shard(1001, rank, world_size)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]
    assert [r[2] for r in res] == [2, 2]
    shards = [r[3] for r in res]
    assert shards[0][0] == 0 and shards[0][1] == shards[1][0] and shards[1][1] == 1001


@pytest.mark.parametrize("n,w", [(0, 1), (5, 2), (7, 3), (1000, 8), (3, 8)])
def test_shards_tile(n, w):
    covered = []
    for r in range(w):
        b, e = R.shard(n, r, w)
        assert 0 <= b <= e <= n
        covered += list(range(b, e))
    assert covered == list(range(n))


def test_single_process_is_identity():
    assert R.world() == 1
    assert R.max_over_ranks(3.5) == 3.5
