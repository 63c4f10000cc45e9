"""Multi-rank logic of the ensemble / benchmark on CPU: two gloo ranks."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fdm_cell_based_amr_cartesian_b200.ensemble import max_over_ranks, partition, sum_over_ranks


def test_partition_balances_and_covers():
    w = [5, 1, 1, 1, 1, 9, 2, 2, 3]
    owner = partition(w, 3)
    assert sorted(set(owner)) == [0, 1, 2]
    loads = [sum(wi for wi, o in zip(w, owner) if o == r) for r in range(3)]
    assert max(loads) - min(loads) <= max(w)
    assert partition(w, 3) == owner          # deterministic
    assert partition(w, 1) == [0] * len(w)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = [3, 7, 2, 2, 5, 1]
        owner = partition(w, world)
        mine = [i for i, o in enumerate(owner) if o == rank]
        local_updates = sum(w[i] for i in mine)
        elapsed = 10.0 + rank          # rank 1 is slower
        q.put((rank, mine, max_over_ranks(elapsed), sum_over_ranks(local_updates)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_without_overlap():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    owned = out[0][1] + out[1][1]
    assert sorted(owned) == list(range(6))
    assert not set(out[0][1]) & set(out[1][1])
    assert out[0][2] == out[1][2] == 11.0     # max over ranks
    assert out[0][3] == out[1][3] == 20.0     # all updates counted once
