"""CPU tests of the process grids of astaroth_b200.grid: the reference's Morton
order and default grids (src/core/decomposition/decomposition.cc:502-663), the
tiling of the mesh by sub-domains, and the three-pass halo exchange plan
(face_boxes along x, y, z with the neighbours of ProcessGrid), applied with
numpy to every sub-domain of a random mesh: every ghost cell must equal the
global periodic wrap.  Also the Grid's clean-up when a sub-domain's Device
cannot be made."""
import numpy as np
import pytest

from astaroth_b200.grid import (HALO, ProcessGrid, face_boxes, morton_coords,
                                morton_decomposition, morton_rank)


def test_morton_default_grids():
    # the reference's morton_decompose: Morton coordinates of nprocs - 1, plus one
    assert [morton_decomposition(n) for n in (1, 2, 4, 8, 16, 32, 64)] == [
        (1, 1, 1), (1, 1, 2), (1, 2, 2), (2, 2, 2), (2, 2, 4), (2, 4, 4), (4, 4, 4)]
    for n in (3, 6, 12):
        with pytest.raises(ValueError):
            morton_decomposition(n)


def test_morton_order_is_a_bijection():
    assert [morton_coords(p) for p in range(8)] == [
        (0, 0, 0), (0, 0, 1), (0, 1, 0), (0, 1, 1), (1, 0, 0), (1, 0, 1), (1, 1, 0), (1, 1, 1)]
    for p in range(4096):
        assert morton_rank(*morton_coords(p)) == p
    # bits interleave with z lowest: rank 9 = 0b001001 -> k = 0b11
    assert morton_coords(9) == (0, 0, 3)


@pytest.mark.parametrize("dims,mapping", [((2, 1, 1), "linear"), ((1, 3, 2), "linear"),
                                          ((2, 2, 2), "morton"), ((1, 2, 2), "morton"),
                                          ((3, 2, 2), "linear")])
def test_process_grid_tiles_the_mesh(dims, mapping):
    n = (13, 11, 12)
    pg = ProcessGrid(n, dims, mapping)
    cover = np.zeros(n[::-1], dtype=int)
    for r in range(pg.size):
        (ox, oy, oz), (nx, ny, nz) = pg.box(r)
        cover[oz:oz + nz, oy:oy + ny, ox:ox + nx] += 1
        assert pg.rank(pg.coords(r)) == r
        for axis in range(3):
            assert pg.neighbour(pg.neighbour(r, axis, +1), axis, -1) == r
            # the neighbour along an axis shares the other two coordinates
            c, cn = pg.coords(r), pg.coords(pg.neighbour(r, axis, +1))
            assert [c[b] for b in range(3) if b != axis] == [cn[b] for b in range(3) if b != axis]
    assert (cover == 1).all()


def test_process_grid_refusals():
    with pytest.raises(ValueError):
        ProcessGrid((12, 12, 12), (2, 1, 1), "morton")  # Morton order leaves this grid
    with pytest.raises(ValueError):
        ProcessGrid((8, 12, 12), (3, 1, 1))  # parts thinner than the halo
    with pytest.raises(ValueError):
        ProcessGrid((12, 12, 12), (0, 1, 1))


def _exchange_numpy(pg, local):
    """The three passes of Grid._exchange_axis on numpy sub-domains (axis order
    x, y, z; arrays indexed [z, y, x])."""
    for axis in range(3):
        packed = []
        for r in range(pg.size):
            n = pg.box(r)[1]
            send_lo, send_hi, _, _ = face_boxes(axis, n)
            packed.append([_take(local[r], b) for b in (send_lo, send_hi)])
        for r in range(pg.size):
            n = pg.box(r)[1]
            _, _, recv_lo, recv_hi = face_boxes(axis, n)
            below, above = pg.neighbour(r, axis, -1), pg.neighbour(r, axis, +1)
            _put(local[r], recv_lo, packed[below][1])  # the high cells of the one below
            _put(local[r], recv_hi, packed[above][0])  # the low cells of the one above


def _sl(box):
    (x, y, z), (dx, dy, dz) = box
    return np.s_[z:z + dz, y:y + dy, x:x + dx]


def _take(a, box):
    return a[_sl(box)].copy()


def _put(a, box, v):
    assert a[_sl(box)].shape == v.shape
    a[_sl(box)] = v


@pytest.mark.parametrize("dims,mapping", [((2, 1, 1), "linear"), ((1, 2, 1), "linear"),
                                          ((1, 1, 3), "linear"), ((2, 2, 1), "linear"),
                                          ((2, 2, 2), "morton"), ((3, 2, 2), "linear"),
                                          ((1, 1, 1), "linear"), ((2, 3, 2), "linear")])
def test_three_pass_exchange_fills_every_ghost(dims, mapping):
    n = (13, 11, 12)
    rng = np.random.default_rng(7)
    interior = rng.standard_normal(n[::-1])
    wrapped = np.pad(interior, HALO, mode="wrap")  # the global periodic fill
    pg = ProcessGrid(n, dims, mapping)
    local = []
    for r in range(pg.size):
        (ox, oy, oz), (nx, ny, nz) = pg.box(r)
        a = np.full((nz + 2 * HALO, ny + 2 * HALO, nx + 2 * HALO), np.nan)
        a[HALO:-HALO, HALO:-HALO, HALO:-HALO] = interior[oz:oz + nz, oy:oy + ny, ox:ox + nx]
        local.append(a)
    _exchange_numpy(pg, local)
    for r in range(pg.size):
        (ox, oy, oz), (nx, ny, nz) = pg.box(r)
        want = wrapped[oz:oz + nz + 2 * HALO, oy:oy + ny + 2 * HALO, ox:ox + nx + 2 * HALO]
        assert np.array_equal(local[r], want), r


def test_face_boxes_shapes():
    n = (10, 8, 6)
    m = [v + 2 * HALO for v in n]
    x = face_boxes(0, n)
    assert x == (((3, 3, 3), (3, 8, 6)), ((10, 3, 3), (3, 8, 6)), ((0, 3, 3), (3, 8, 6)),
                 ((13, 3, 3), (3, 8, 6)))
    y = face_boxes(1, n)
    assert all(b[1] == (m[0], 3, n[2]) for b in y)
    z = face_boxes(2, n)
    assert all(b[1] == (m[0], m[1], 3) for b in z)  # whole planes
    assert [b[0][2] for b in z] == [3, 6, 0, 9]


def test_grid_releases_devices_when_one_fails(monkeypatch):
    """A sub-domain whose Device cannot be made releases the ones made before it."""
    import astaroth_b200.grid as grid
    from astaroth_b200.device import make_info

    made, destroyed = [], []

    class FakeDevice:
        def __init__(self, info, device_id=0):
            if len(made) == 1:
                raise RuntimeError("no device")
            made.append(self)

        def destroy(self):
            destroyed.append(self)

    monkeypatch.setattr(grid, "Device", FakeDevice)
    with pytest.raises(RuntimeError):
        grid.Grid(make_info((32, 32, 24)), decomp=(2, 1, 1))
    assert len(made) == 1 and destroyed == made
