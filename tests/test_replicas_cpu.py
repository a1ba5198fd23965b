"""The multi-rank layout on CPU: two gloo ranks split a disk sweep and agree
on the max-over-ranks timing, with no GPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from disco2_b200 import configs, replicas


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, cells, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        parts = replicas.partition(cells, world)
        mine = parts[rank]
        fake_ms = 10.0 + rank  # per-rank elapsed time
        m = replicas.max_over_ranks(fake_ms)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        q.put((rank, mine, m, gathered))
    finally:
        dist.destroy_process_group()


def test_partition_balances_and_covers():
    cells = [100, 90, 80, 10, 10, 5, 5]
    parts = replicas.partition(cells, 3)
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(cells)))
    loads = [sum(cells[k] for k in p) for p in parts]
    assert max(loads) - min(loads) <= 100
    assert replicas.partition(cells, 3) == parts  # deterministic


def test_two_gloo_ranks_split_sweep_and_reduce_max():
    from disco2_b200 import lib
    sweep = configs.circumbinary_sweep(8, seed=3)
    cells = [lib.Sim(p).num_cells for p in sweep]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, cells, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, m0, max0, g0), (r1, m1, max1, g1) = res
    assert max0 == max1 == 11.0
    assert g0 == g1 == [m0, m1]
    assert sorted(m0 + m1) == list(range(8)) and not set(m0) & set(m1)
