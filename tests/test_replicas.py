"""Replica placement and max-over-ranks timing, with world-size-2 gloo ranks
on the CPU (the multi-GPU path has no collective on the data path)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from lceqcd_b200.replicas import assign_chains, max_over_ranks, rank_loads


def test_assignment_covers_every_chain_once():
    vols = [16 ** 3] * 32 + [32 ** 3] * 32 + [48 ** 3] * 32
    for w in (1, 2, 3, 4, 8):
        parts = assign_chains(vols, w)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(vols)))
        loads = rank_loads(vols, w)
        assert max(loads) - min(loads) <= max(vols)


def test_assignment_rejects_empty_world():
    with pytest.raises(ValueError):
        assign_chains([1, 2], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        vols = [16 ** 3, 48 ** 3, 32 ** 3, 16 ** 3, 48 ** 3]
        mine = assign_chains(vols, world)[rank]
        t = max_over_ranks(1.0 + rank)          # rank-dependent "device time"
        q.put((rank, mine, t))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_partition_and_max():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert sorted(res[0][1] + res[1][1]) == [0, 1, 2, 3, 4]
    assert res[0][2] == res[1][2] == 2.0
