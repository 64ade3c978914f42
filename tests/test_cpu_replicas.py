"""The N > 1 path on CPU: two `gloo` ranks take disjoint shares of a request
stream, and the timing reduction gives every rank the slowest rank's time and
the units of all ranks (the only collective steps of a replica run)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT  # noqa: F401


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    from bem3_aw_qd2_b200 import replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mine = replicas.shard(11, rank, world)
        dist.barrier()
        # rank r "took" 10 + r ms for its units
        t, u = replicas.reduce_timing([10.0 + rank, 2.0 * rank], [len(mine)])
        q.put((rank, mine, t, u))
    finally:
        dist.destroy_process_group()


def test_shard_partitions_units():
    from bem3_aw_qd2_b200 import replicas
    for n in (0, 1, 7, 64):
        for world in (1, 2, 3, 8):
            parts = [replicas.shard(n, r, world) for r in range(world)]
            flat = sorted(i for p in parts for i in p)
            assert flat == list(range(n))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def test_reduce_timing_single_process():
    from bem3_aw_qd2_b200 import replicas
    assert replicas.reduce_timing([3.5], [7]) == ([3.5], [7.0])


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert res[0][1] == [0, 2, 4, 6, 8, 10] and res[1][1] == [1, 3, 5, 7, 9]
    for _, _, t, u in res:
        assert t == [11.0, 2.0]  # the slowest rank's time, per quantity
        assert u == [11.0]  # all units of the stream
