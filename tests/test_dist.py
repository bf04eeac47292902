"""CPU tests of the multi-process plumbing (gloo, world size 2): the
max-over-ranks timing reduction, the barrier, and the sharding of an ensemble
of independent members across ranks (no data-path collective)."""
import os
import socket

import pytest
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


def _exchange_worker(rank, world, port, out):
    import torch

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    assert adist.init("gloo", timeout_s=60)
    from astaroth_b200.grid import DistTransport

    t = DistTransport()
    n = 64
    sb = torch.full((n,), 10 * rank + 1, dtype=torch.uint8)
    st = torch.full((n,), 10 * rank + 2, dtype=torch.uint8)
    rb = torch.zeros(n, dtype=torch.uint8)
    rt = torch.zeros(n, dtype=torch.uint8)
    for _ in range(3):  # repeated exchanges keep matching in order
        t.exchange([sb], [st], [rb], [rt])
    res = (rank, int(rb[0]), int(rb[-1]), int(rt[0]), int(rt[-1]),
           t.combine([float(rank + 1)], "max"), t.combine([float(rank + 1)], "min"),
           t.combine([float(rank + 1)], "sum"))
    out.put(res)
    adist.barrier()
    adist.destroy()


@pytest.mark.parametrize("world", [2, 3])
def test_grid_halo_exchange_gloo(world):
    """Each rank's bottom ghost receives the top planes of the rank below and
    its top ghost the bottom planes of the rank above, periodically; the
    reductions combine over the ranks."""
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_exchange_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, rb0, rb1, rt0, rt1, mx, mn, sm in res:
        below, above = (rank - 1) % world, (rank + 1) % world
        assert rb0 == rb1 == 10 * below + 2
        assert rt0 == rt1 == 10 * above + 1
        assert (mx, mn, sm) == (world, 1, world * (world + 1) / 2)


def _grid_exchange_worker(rank, world, port, dims, mapping, out):
    import torch

    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    assert adist.init("gloo", timeout_s=60)
    from astaroth_b200.grid import DistTransport, ProcessGrid

    t = DistTransport()
    pg = ProcessGrid((24, 24, 24), dims, mapping)
    res = []
    for _ in range(2):  # repeated rounds keep matching in order
        for axis in range(3):
            sb = torch.full((16,), 100 * rank + 10 * axis + 1, dtype=torch.int32)
            st = torch.full((16,), 100 * rank + 10 * axis + 2, dtype=torch.int32)
            rb = torch.zeros(16, dtype=torch.int32)
            rt = torch.zeros(16, dtype=torch.int32)
            t.exchange([sb], [st], [rb], [rt], lo=[pg.neighbour(rank, axis, -1)],
                       hi=[pg.neighbour(rank, axis, +1)], tag=axis)
            res.append((axis, int(rb[0]), int(rb[-1]), int(rt[0]), int(rt[-1])))
    out.put((rank, res))
    adist.barrier()
    adist.destroy()


@pytest.mark.parametrize("dims,mapping", [((2, 2, 1), "linear"), ((1, 2, 2), "morton"),
                                          ((2, 1, 2), "linear")])
def test_process_grid_exchange_gloo(dims, mapping):
    """Along each axis of a 4-rank process grid, a rank's low ghost receives
    the high cells of its neighbour below and its high ghost the low cells of
    the one above; an axis that is not split exchanges with itself; the tags
    keep the three axes apart."""
    from astaroth_b200.grid import ProcessGrid

    world = 4
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_grid_exchange_worker, args=(r, world, port, dims, mapping, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    pg = ProcessGrid((24, 24, 24), dims, mapping)
    for rank, rows in res.items():
        for axis, rb0, rb1, rt0, rt1 in rows:
            below, above = pg.neighbour(rank, axis, -1), pg.neighbour(rank, axis, +1)
            assert rb0 == rb1 == 100 * below + 10 * axis + 2
            assert rt0 == rt1 == 100 * above + 10 * axis + 1


def test_decompose_covers_the_planes():
    from astaroth_b200.grid import decompose

    for nz, parts in ((48, 2), (20, 3), (16, 5), (9, 3)):
        r = decompose(nz, parts)
        assert r[0][0] == 0 and sum(n for _, n in r) == nz
        assert all(r[i][0] + r[i][1] == r[i + 1][0] for i in range(parts - 1))
        assert max(n for _, n in r) - min(n for _, n in r) <= 1
        assert min(n for _, n in r) >= 3
    with pytest.raises(ValueError):
        decompose(8, 3)  # slabs thinner than the 3-plane halo
