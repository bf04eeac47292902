"""A periodic mesh decomposed into sub-domains, one Device per sub-domain: the
grid layer of the reference (acGridInit / acGridIntegrate /
acGridPeriodicBoundconds / acGridReduceScal, src/core/grid.cc:3086-3110,
3170-3230; halo exchange src/core/task.cc:1933-1993; CFL allreduce
task.cc:2865-2882; process grids src/core/decomposition/decomposition.cc).

The default splits z into slabs.  A process grid (px, py, pz) splits x, y and z
(pencils and blocks), with the ranks placed linearly or in the reference's
Morton order.

One RK3 substep of a slab grid is, on every slab:

1. the periodic fill of the x and y ghost zones of the interior z planes
   (acDevicePeriodicBoundconds on the box [0, mx) x [0, my) x [3, nz + 3));
2. the exchange of the three bottom and three top interior planes of every
   field with the slabs below and above (whole xy planes, halo rows and columns
   included, so edges and corners are right): acDevicePackPlanes into a send
   buffer, a transport, acDeviceUnpackPlanes into the ghost planes;
3. acDeviceIntegrateSubstep and the buffer swap.

With ``overlap`` and every slab at least 7 planes deep, step 3 overlaps step
2, as the reference's task graph does (src/core/task.cc:1933-1993): each slab
solves its interior planes [3, n - 3), which read no ghost plane, on its second
library stream as soon as the x/y fill is done, while the planes travel on the
first; after the unpack the first stream waits for that solve and solves the
three planes at each end (acDeviceIntegrateSubstep on z boxes).  The default
overlaps where the planes cross between GPUs (DistTransport with more than one
rank).  With every slab on one GPU (LocalTransport) the exchange is a copy in
the same HBM and there is nothing to hide: measured on one B200, the split
substep is 3-9% slower than the serial one (two more launches per substep and
slab, and the end boxes load 9 planes for 3).

A grid split in x or y fills its ghost zones in three passes, x, y, then z:
each pass packs the three interior cells at both ends of the axis
(acDevicePackBox), exchanges them with the two neighbours along the axis
(itself where the axis is not split) and unpacks them into the ghost cells.
The x pass covers the interior y and z range, the y pass every x (the x ghosts
are filled by then) and the interior z, the z pass whole planes, so the edges
and corners arrive with the faces, as in the reference's packed segments.  Its
substeps are serial.

Transports:

* ``LocalTransport`` -- every sub-domain in this process, on one GPU; the
  exchange is device-to-device copies.  It exercises the decomposition on one
  GPU and gives the same bits as an undecomposed Device.
* ``DistTransport`` -- one sub-domain per rank of a torch.distributed process
  group (NCCL between GPUs, gloo on CPU tensors): the packed faces go to the
  neighbouring ranks as one batch of point-to-point operations per exchange.

Reductions combine the sub-domains' unprocessed results (max, min, sum) and
apply the RMS post-processing with the global cell count; the CFL maxima are
combined with max before the timestep formula.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import capi
from .capi import AcMeshInfo, Int3Param, Volume
from .device import AstarothError, Device, _check, dims, make_info

HALO = capi.NGHOST


def decompose(nz: int, parts: int) -> list[tuple[int, int]]:
    """(z0, nz) of each of `parts` parts covering nz cells along one axis, sizes
    differing by at most one (the first nz % parts parts one cell larger)."""
    if parts < 1 or nz < parts * HALO:
        raise ValueError(f"{nz} cells cannot be split into {parts} parts of >= {HALO} cells")
    base, extra = divmod(nz, parts)
    out, z0 = [], 0
    for p in range(parts):
        n = base + (1 if p < extra else 0)
        out.append((z0, n))
        z0 += n
    return out


def morton_coords(pid: int) -> tuple[int, int, int]:
    """(i, j, k) of rank `pid` in Morton (z) order over three axes, as the
    reference's morton3D (src/core/decomposition/decomposition.cc:502-517):
    bit 3b of pid is bit b of k, bit 3b + 1 bit b of j, bit 3b + 2 bit b of i."""
    if pid < 0:
        raise ValueError("negative rank")
    c = [0, 0, 0]  # k, j, i
    b = 0
    while pid >> (3 * b):
        for a in range(3):
            c[a] |= ((pid >> (3 * b + a)) & 1) << b
        b += 1
    return c[2], c[1], c[0]


def morton_rank(i: int, j: int, k: int) -> int:
    """The inverse of morton_coords (the reference's morton1D,
    decomposition.cc:546-557)."""
    pid = 0
    for b in range(max(i, j, k).bit_length()):
        pid |= ((k >> b) & 1) << (3 * b)
        pid |= ((j >> b) & 1) << (3 * b + 1)
        pid |= ((i >> b) & 1) << (3 * b + 2)
    return pid


def morton_decomposition(nprocs: int) -> tuple[int, int, int]:
    """The reference's default process grid (morton_decompose,
    decomposition.cc:654-663): the Morton coordinates of rank nprocs - 1 plus
    one, so 2 -> (1, 1, 2), 4 -> (1, 2, 2), 8 -> (2, 2, 2), 16 -> (2, 2, 4).
    Only a power of two fills such a grid exactly; other counts are refused, as
    the reference refuses them."""
    if nprocs < 1:
        raise ValueError("no ranks")
    i, j, k = morton_coords(nprocs - 1)
    dims = (i + 1, j + 1, k + 1)
    if dims[0] * dims[1] * dims[2] != nprocs:
        raise ValueError(f"{nprocs} ranks do not fill a Morton process grid (a power of two does)")
    return dims


class ProcessGrid:
    """A process grid `dims` = (px, py, pz) over a global interior `n` = (nx,
    ny, nz): per rank its coordinates, offset and size, and its neighbours
    along each axis (periodic).  `mapping` places the ranks: "linear" (x
    fastest, the reference's linear_getPid / linear_getPid3D,
    decomposition.cc:606-623) or "morton" (morton_getPid / morton_getPid3D,
    decomposition.cc:599-617)."""

    def __init__(self, n, dims, mapping: str = "linear"):
        self.n = tuple(int(v) for v in n)
        self.dims = tuple(int(v) for v in dims)
        if len(self.dims) != 3 or min(self.dims) < 1:
            raise ValueError(f"bad process grid {dims}")
        if mapping not in ("linear", "morton"):
            raise ValueError(f"unknown rank mapping {mapping!r}")
        self.mapping = mapping
        self.size = self.dims[0] * self.dims[1] * self.dims[2]
        self.splits = [decompose(self.n[a], self.dims[a]) for a in range(3)]
        if mapping == "morton":
            seen = {self.rank(self.coords(r)) for r in range(self.size)}
            if seen != set(range(self.size)) or any(
                    c >= d for r in range(self.size) for c, d in zip(self.coords(r), self.dims)):
                raise ValueError(f"Morton order does not fill the process grid {self.dims}")

    def coords(self, rank: int) -> tuple[int, int, int]:
        if self.mapping == "morton":
            return morton_coords(rank)
        px, py, _ = self.dims
        return rank % px, (rank // px) % py, rank // (px * py)

    def rank(self, c) -> int:
        c = [c[a] % self.dims[a] for a in range(3)]
        if self.mapping == "morton":
            return morton_rank(*c)
        return c[0] + self.dims[0] * (c[1] + self.dims[1] * c[2])

    def box(self, rank: int) -> tuple[tuple[int, int, int], tuple[int, int, int]]:
        """(offset, size) of rank's interior in the global interior."""
        c = self.coords(rank)
        return (tuple(self.splits[a][c[a]][0] for a in range(3)),
                tuple(self.splits[a][c[a]][1] for a in range(3)))

    def neighbour(self, rank: int, axis: int, d: int) -> int:
        c = list(self.coords(rank))
        c[axis] += d
        return self.rank(c)


def face_boxes(axis: int, n) -> tuple:
    """The (start, dims) boxes, in padded local indices, of the exchange along
    `axis` of a sub-domain with interior `n`: (send_lo, send_hi, recv_lo,
    recv_hi).  The three interior cells at each end go to the neighbour on that
    side; the ghost cells at each end come from it.  Axes before `axis` span
    every cell (their ghosts are filled by then), axes after it their interior."""
    m = [v + 2 * HALO for v in n]
    start, dims = [0, 0, 0], [0, 0, 0]
    for b in range(3):
        if b < axis:
            start[b], dims[b] = 0, m[b]
        elif b > axis:
            start[b], dims[b] = HALO, n[b]
    boxes = []
    for lo in (HALO, n[axis], 0, n[axis] + HALO):
        s = list(start)
        s[axis] = lo
        d = list(dims)
        d[axis] = HALO
        boxes.append((tuple(s), tuple(d)))
    return tuple(boxes)


def subdomain_info(info: AcMeshInfo, offset, n) -> AcMeshInfo:
    """The AcMeshInfo of one sub-domain: AC_nlocal = n with the global AC_ngrid
    and AC_ds, AC_multigpu_offset = offset."""
    s = AcMeshInfo()
    C.memmove(C.byref(s), C.byref(info), C.sizeof(AcMeshInfo))
    s.int3_params[Int3Param.AC_nlocal] = capi.Int3(*n)
    s.int3_params[Int3Param.AC_multigpu_offset] = capi.Int3(*offset)
    _check(capi.load().acHostUpdateParams(C.byref(s)), "acHostUpdateParams")
    return s


def slab_info(info: AcMeshInfo, z0: int, nz: int) -> AcMeshInfo:
    """The AcMeshInfo of one z slab: AC_nlocal = (nx, ny, nz) with the global
    AC_ngrid and AC_ds, AC_multigpu_offset = (0, 0, z0)."""
    n = info.int3_params[Int3Param.AC_ngrid]
    return subdomain_info(info, (0, 0, z0), (n.x, n.y, nz))


class LocalTransport:
    """All sub-domains in this process: sub-domain i's low ghost cells come from
    the high interior cells of its neighbour below, lo[i], and its high ghost
    cells from the low interior cells of its neighbour above, hi[i]
    (periodically; by default the ring of z slabs i - 1 and i + 1).

    With `streams` (the sub-domains' library streams, as torch streams) the
    copies are stream-ordered, with no host synchronisation: they run on
    streams[0] after every sub-domain's pack, and every sub-domain's stream then
    waits for them, so that the unpack follows the copies and the next pack into
    a send buffer follows every read of it."""

    def exchange(self, send_bottom, send_top, recv_bottom, recv_top, streams=None, lo=None,
                 hi=None, tag=0):
        k = len(send_bottom)
        lo = lo if lo is not None else [(i - 1) % k for i in range(k)]
        hi = hi if hi is not None else [(i + 1) % k for i in range(k)]
        if streams is None:
            for i in range(k):
                recv_bottom[i].copy_(send_top[lo[i]])
                recv_top[i].copy_(send_bottom[hi[i]])
            return
        import torch

        s0 = streams[0]
        for s in streams[1:]:
            s0.wait_stream(s)  # every sub-domain packed
        with torch.cuda.stream(s0):
            for i in range(k):
                recv_bottom[i].copy_(send_top[lo[i]])
                recv_top[i].copy_(send_bottom[hi[i]])
        for s in streams[1:]:
            s.wait_stream(s0)  # copies done before unpack and the next pack

    def combine(self, values, op):
        return {"max": max, "min": min, "sum": math.fsum}[op](values)


class DistTransport:
    """One sub-domain per rank: the high cells go to the neighbour above (its
    low ghost cells), the low cells to the neighbour below (its high ghost
    cells), periodically; by default the ranks rank + 1 and rank - 1 of a ring
    of z slabs.  Sends and receives are posted in the same order on every rank,
    with a tag per direction and axis, so messages between the same two ranks
    match in order (two ranks along an axis are each other's neighbour on both
    sides).  A rank that is its own neighbour (an axis that is not split) copies.

    With `streams` (NCCL, device buffers) the point-to-point operations are
    enqueued behind the pack on the sub-domain's library stream and waited for
    on that stream (Work.wait orders the current stream, the host does not
    block), so the unpack that follows on the same stream sees the cells."""

    def __init__(self):
        import torch.distributed as dist

        self.dist = dist
        self.rank = dist.get_rank()
        self.world = dist.get_world_size()
        # every rank takes part in the group's first collective, so that the
        # exchanges, which involve neighbours only, are never the first
        dist.barrier()

    def exchange(self, send_bottom, send_top, recv_bottom, recv_top, streams=None, lo=None,
                 hi=None, tag=0):
        (sb,), (st,), (rb,), (rt,) = send_bottom, send_top, recv_bottom, recv_top
        down = lo[0] if lo is not None else (self.rank - 1) % self.world
        up = hi[0] if hi is not None else (self.rank + 1) % self.world
        if streams is None:
            self._exchange(sb, st, rb, rt, down, up, tag)
            return
        import torch

        with torch.cuda.stream(streams[0]):
            self._exchange(sb, st, rb, rt, down, up, tag)

    def _exchange(self, sb, st, rb, rt, down, up, tag):
        if down == self.rank and up == self.rank:
            rb.copy_(st)
            rt.copy_(sb)
            return
        d = self.dist
        t_up, t_down = 2 * tag + 1, 2 * tag + 2
        # one batch: a single NCCL group (ncclGroupStart / ncclSend, ncclRecv /
        # ncclGroupEnd) for the four transfers
        ops = [d.P2POp(d.isend, st, up, tag=t_up), d.P2POp(d.irecv, rb, down, tag=t_up),
               d.P2POp(d.isend, sb, down, tag=t_down), d.P2POp(d.irecv, rt, up, tag=t_down)]
        for r in d.batch_isend_irecv(ops):
            r.wait()

    def combine(self, values, op):
        import torch

        (v,) = values
        t = torch.tensor([v], dtype=torch.float64,
                         device="cuda" if self.dist.get_backend() == "nccl" else "cpu")
        red = {"max": self.dist.ReduceOp.MAX, "min": self.dist.ReduceOp.MIN,
               "sum": self.dist.ReduceOp.SUM}[op]
        self.dist.all_reduce(t, op=red)
        return float(t.item())


class Grid:
    """A periodic mesh of global size AC_ngrid split into sub-domains.

    info: the global AcMeshInfo.  With ``transport=None`` every sub-domain is
    held in this process (LocalTransport); with a DistTransport this process
    holds its rank's sub-domain.

    decomp: the process grid.  None splits z only, into ``slabs`` slabs here or
    one per rank; (px, py, pz) splits each axis (the product is the number of
    sub-domains); "morton" takes the reference's default grid for that many
    sub-domains (``slabs`` here, the world size with a DistTransport), ranks in
    Morton order.  mapping: the rank order of a tuple ``decomp`` ("linear",
    x fastest, or "morton").
    """

    def __init__(self, info: AcMeshInfo, slabs: int = 1, transport=None, device_id: int = 0,
                 overlap: bool | None = None, decomp=None, mapping: str = "linear"):
        import torch

        self.lib = capi.load()
        self.info = info
        self.n = dims(info)
        dist = isinstance(transport, DistTransport)
        count = transport.world if dist else slabs
        if decomp is None:
            decomp = (1, 1, count)
        elif decomp == "morton":
            decomp, mapping = morton_decomposition(count), "morton"
        self.pgrid = ProcessGrid(self.n, decomp, mapping)
        if dist and self.pgrid.size != transport.world:
            raise ValueError(f"process grid {self.pgrid.dims} does not have "
                             f"{transport.world} ranks")
        self.ranks = [transport.rank] if dist else list(range(self.pgrid.size))
        self.transport = transport if dist else (transport or LocalTransport())
        self.boxes = [self.pgrid.box(r) for r in self.ranks]
        self.slabs_only = self.pgrid.dims[0] == self.pgrid.dims[1] == 1
        # (z0, nz) of each local sub-domain
        self.ranges = [(off[2], n[2]) for off, n in self.boxes]
        self.devs = []
        try:
            for off, n in self.boxes:
                self.devs.append(Device(subdomain_info(info, off, n), device_id))
        except BaseException:
            self.destroy()  # the sub-domains made so far
            raise
        self.plane_bytes = self.lib.acDevicePlaneBytes(self.devs[0].handle)
        dev = torch.device("cuda", device_id)
        self._dev = dev
        self._streams = [torch.cuda.ExternalStream(d.stream_handle(0), device=dev)
                         for d in self.devs]
        # the interior solve of the overlapped substep runs on library stream 1
        self._streams1 = [torch.cuda.ExternalStream(d.stream_handle(1), device=dev)
                          for d in self.devs]
        if overlap is None:
            overlap = dist and transport.world > 1
        self.overlap = (overlap and self.slabs_only and
                        min(n for _, n in self.ranges) >= 2 * HALO + 1)
        if self.slabs_only:
            self._buf = {k: [torch.empty(HALO * self.plane_bytes, dtype=torch.uint8, device=dev)
                             for _ in self.devs] for k in ("sb", "st", "rb", "rt")}
        else:
            self._faces = [self._face_buffers(axis) for axis in range(3)]
        self.cells = self.n[0] * self.n[1] * self.n[2]

    def _face_buffers(self, axis: int) -> dict:
        """Send and receive buffers of the exchange along `axis`, per local
        sub-domain."""
        import torch

        out = {k: [] for k in ("sb", "st", "rb", "rt")}
        for d, (_, n) in zip(self.devs, self.boxes):
            size = self.lib.acDeviceBoxBytes(d.handle, capi.Int3(*face_boxes(axis, n)[0][1]))
            for k in out:
                out[k].append(torch.empty(size, dtype=torch.uint8, device=self._dev))
        return out

    def destroy(self):
        for d in self.devs:
            d.destroy()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    # ---- data ----
    def load_mesh(self, fields: np.ndarray) -> None:
        """Loads this process's sub-domains from a global (8, mz, my, mx) mesh."""
        for d, (o, n) in zip(self.devs, self.boxes):
            d.load_mesh(np.ascontiguousarray(
                fields[:, o[2]:o[2] + n[2] + 2 * HALO, o[1]:o[1] + n[1] + 2 * HALO,
                       o[0]:o[0] + n[0] + 2 * HALO]))

    def store_mesh(self, out: np.ndarray | None = None) -> np.ndarray:
        """The interiors of this process's sub-domains in a global (8, mz, my, mx)
        array (cells of other ranks' sub-domains and ghost cells are left as they
        are)."""
        nx, ny, nz = self.n
        if out is None:
            out = np.zeros((capi.NUM_FIELDS, nz + 2 * HALO, ny + 2 * HALO, nx + 2 * HALO))
        H = HALO
        for d, (o, n) in zip(self.devs, self.boxes):
            s = d.store_mesh()
            out[:, H + o[2]:H + o[2] + n[2], H + o[1]:H + o[1] + n[1], H + o[0]:H + o[0] + n[0]] = \
                s[:, H:H + n[2], H:H + n[1], H:H + n[0]]
        return out

    # ---- boundary conditions ----
    def periodic_boundconds(self, interior_step=None) -> None:
        """Fills every ghost cell of every sub-domain.  Slabs: x and y by local
        wrap, z by the exchange with the neighbouring slabs.  Otherwise: the
        exchanges along x, y and z in turn.  Everything is ordered on the
        sub-domains' library streams (stream 0); the host does not wait.

        interior_step: (step, dt) of a substep whose interior planes each slab
        solves on its stream 1 once its x/y fill is done, while the planes
        travel (the overlapped substep; slabs only)."""
        if not self.slabs_only:
            if interior_step is not None:
                raise ValueError("the overlapped substep needs a slab decomposition")
            for axis in range(3):
                self._exchange_axis(axis)
            return
        b = self._buf
        nx, ny, _ = self.n
        for i, (d, (_, n)) in enumerate(zip(self.devs, self.ranges)):
            _check(self.lib.acDevicePeriodicBoundconds(
                d.handle, 0, Volume(0, 0, HALO), Volume(nx + 2 * HALO, ny + 2 * HALO, n + HALO)),
                "acDevicePeriodicBoundconds")
            if interior_step is not None:
                self._streams1[i].wait_stream(self._streams[i])
                self._solve_box(d, 1, interior_step, 2 * HALO, n)
            _check(self.lib.acDevicePackPlanes(d.handle, 0, HALO, HALO, b["sb"][i].data_ptr()),
                   "acDevicePackPlanes")
            _check(self.lib.acDevicePackPlanes(d.handle, 0, n, HALO, b["st"][i].data_ptr()),
                   "acDevicePackPlanes")
        self.transport.exchange(b["sb"], b["st"], b["rb"], b["rt"], streams=self._streams)
        for i, (d, (_, n)) in enumerate(zip(self.devs, self.ranges)):
            _check(self.lib.acDeviceUnpackPlanes(d.handle, 0, 0, HALO, b["rb"][i].data_ptr()),
                   "acDeviceUnpackPlanes")
            _check(self.lib.acDeviceUnpackPlanes(d.handle, 0, n + HALO, HALO,
                                                 b["rt"][i].data_ptr()), "acDeviceUnpackPlanes")

    def _exchange_axis(self, axis: int) -> None:
        """The exchange along `axis`: pack the three interior cells at each end,
        swap them with the neighbours along the axis, unpack into the ghosts."""
        b = self._faces[axis]
        lib = self.lib
        for i, (d, (_, n)) in enumerate(zip(self.devs, self.boxes)):
            send_lo, send_hi, _, _ = face_boxes(axis, n)
            for box, k in ((send_lo, "sb"), (send_hi, "st")):
                _check(lib.acDevicePackBox(d.handle, 0, capi.Int3(*box[0]), capi.Int3(*box[1]),
                                           b[k][i].data_ptr()), "acDevicePackBox")
        # the neighbours' ranks (with every sub-domain here, rank = local index)
        lo = [self.pgrid.neighbour(r, axis, -1) for r in self.ranks]
        hi = [self.pgrid.neighbour(r, axis, +1) for r in self.ranks]
        self.transport.exchange(b["sb"], b["st"], b["rb"], b["rt"], streams=self._streams, lo=lo,
                                hi=hi, tag=axis)
        for i, (d, (_, n)) in enumerate(zip(self.devs, self.boxes)):
            _, _, recv_lo, recv_hi = face_boxes(axis, n)
            for box, k in ((recv_lo, "rb"), (recv_hi, "rt")):
                _check(lib.acDeviceUnpackBox(d.handle, 0, capi.Int3(*box[0]), capi.Int3(*box[1]),
                                             b[k][i].data_ptr()), "acDeviceUnpackBox")

    def _solve_box(self, d, stream: int, step_dt, z0: int, z1: int) -> None:
        """acDeviceIntegrateSubstep on the interior x-y planes [z0, z1) (padded
        z indices) of slab device d."""
        nx, ny, _ = self.n
        step, dt = step_dt
        _check(self.lib.acDeviceIntegrateSubstep(d.handle, stream, step, Volume(HALO, HALO, z0),
                                                 Volume(nx + HALO, ny + HALO, z1), dt),
               "acDeviceIntegrateSubstep")

    # ---- integration ----
    def integrate_substep(self, step: int, dt: float) -> None:
        if not self.overlap:
            self.periodic_boundconds()
            for d in self.devs:
                d.integrate_substep(step, dt)
            for d in self.devs:
                d.swap_buffers()
            return
        # interior planes while the boundary planes travel; then, after the
        # unpack and the interior solve (whose first box also clears the CFL
        # maxima of substep 2), the three planes at each end
        self.periodic_boundconds(interior_step=(step, dt))
        for i, (d, (_, n)) in enumerate(zip(self.devs, self.ranges)):
            self._streams[i].wait_stream(self._streams1[i])
            self._solve_box(d, 0, (step, dt), HALO, 2 * HALO)
            self._solve_box(d, 0, (step, dt), n, n + HALO)
        for d in self.devs:
            d.swap_buffers()

    def integrate_step(self, dt: float) -> None:
        for s in range(3):
            self.integrate_substep(s, dt)

    def synchronize(self) -> None:
        for d in self.devs:
            d.synchronize()

    # ---- reductions over the whole grid ----
    def _post(self, rtype: str, v: float) -> float:
        r = capi.RTYPES[rtype]
        if r.post_processing_op == 1:  # AC_RMS: sqrt(sum / cells) over the global grid
            return math.sqrt(v / self.cells)
        return v

    def _op(self, rtype: str) -> str:
        return {capi.ReduceOp.AC_REDUCE_OP_MAX: "max", capi.ReduceOp.AC_REDUCE_OP_MIN: "min",
                capi.ReduceOp.AC_REDUCE_OP_SUM: "sum"}[capi.RTYPES[rtype].reduce_op]

    def reduce_scal(self, rtype: str, field: int) -> float:
        vals = [d.reduce_scal(rtype, field, post=False) for d in self.devs]
        return self._post(rtype, self.transport.combine([self._local(vals, rtype)],
                                                        self._op(rtype)))

    def reduce_vec(self, rtype: str, a: int, b: int, c: int) -> float:
        vals = [d.reduce_vec(rtype, a, b, c, post=False) for d in self.devs]
        return self._post(rtype, self.transport.combine([self._local(vals, rtype)],
                                                        self._op(rtype)))

    def _local(self, vals, rtype):
        op = self._op(rtype)
        return {"max": max, "min": min, "sum": math.fsum}[op](vals)

    # ---- CFL timestep ----
    def calc_timestep(self) -> None:
        for d in self.devs:
            d.calc_timestep()

    def timestep(self) -> float:
        """dt from the CFL outputs of all slabs (the last substep 2, or
        calc_timestep): each output finished on every slab, combined with its
        own operation (max, or min for AC_dt_min) and set back on the slabs,
        as acGridFinalizeReduce (src/core/grid.cc:3004-3024); then the dt of
        the maximum or the additive form (AC_additive_timestep)."""
        out = capi.RealOutputParam
        for p, op in ((out.UU_MAX_ADVEC, "max"), (out.ALFVEN_SPEED_MAX, "max"),
                      (out.AC_dt_min, "min")):
            vals = [d.finish_reduce(p) for d in self.devs]
            v = self.transport.combine([{"max": max, "min": min}[op](vals)], op)
            for d in self.devs:
                d.set_output(p, v)
        return self.devs[0].timestep()


__all__ = ["Grid", "LocalTransport", "DistTransport", "ProcessGrid", "decompose", "face_boxes",
           "morton_coords", "morton_decomposition", "morton_rank", "slab_info", "subdomain_info"]
