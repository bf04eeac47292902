"""CPU tests of the multi-process plumbing (gloo, world size 2): the
max-over-ranks timing reduction, the barrier, and the sharding of an ensemble
of independent members across ranks (no data-path collective)."""
import os
import socket

import torch.multiprocessing as mp

from astaroth_b200 import dist as adist


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    assert adist.init("gloo", timeout_s=60)
    adist.barrier()
    m = adist.max_over_ranks(10.0 * (rank + 1))
    s = adist.sum_over_ranks(rank + 1)
    sizes = [32, 48, 64, 96] * 16
    mine = adist.shard([n ** 3 for n in sizes], rank, world)
    out.put((rank, m, s, mine))
    adist.barrier()
    adist.destroy()


def test_gloo_two_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res.sort()
    assert all(r[1] == 20.0 for r in res)  # max over ranks
    assert all(r[2] == 3.0 for r in res)
    owned = sorted(res[0][3] + res[1][3])
    assert owned == list(range(64))  # every member exactly once
    assert not set(res[0][3]) & set(res[1][3])


def test_shard_balance_and_determinism():
    sizes = [32, 48, 64, 96] * 16
    costs = [n ** 3 for n in sizes]
    for world in (1, 2, 3, 4, 8):
        parts = [adist.shard(costs, r, world) for r in range(world)]
        assert sorted(sum(parts, [])) == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
        assert parts == [adist.shard(costs, r, world) for r in range(world)]


def test_single_process_defaults():
    assert not adist.init()  # WORLD_SIZE unset: no process group
    assert adist.max_over_ranks(3.5) == 3.5
    assert adist.sum_over_ranks(2.0) == 2.0
    adist.barrier()
