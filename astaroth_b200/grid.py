"""A periodic mesh decomposed along z into slabs, one Device per slab: the
grid layer of the reference (acGridInit / acGridIntegrate /
acGridPeriodicBoundconds / acGridReduceScal, src/core/grid.cc:3086-3110,
3170-3230; halo exchange src/core/task.cc:1933-1993; CFL allreduce
task.cc:2865-2882) for slab decompositions.

One RK3 substep of the grid is, on every slab:

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

Transports:

* ``LocalTransport`` -- every slab in this process, on one GPU; the exchange
  is device-to-device copies.  It exercises the decomposition on one GPU and
  gives the same bits as an undecomposed Device.
* ``DistTransport`` -- one slab per rank of a torch.distributed process group
  (NCCL between GPUs, gloo on CPU tensors): point-to-point sends of the packed
  planes to the ranks below and above.

Reductions combine the slabs' unprocessed results (max, min, sum) and apply the
RMS post-processing with the global cell count; the CFL maxima are combined
with max before the timestep formula.
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
    """(z0, nz) of each of `parts` slabs covering nz planes, sizes differing by
    at most one (the first nz % parts slabs one plane larger)."""
    if parts < 1 or nz < parts * HALO:
        raise ValueError(f"{nz} planes cannot be split into {parts} slabs of >= {HALO} planes")
    base, extra = divmod(nz, parts)
    out, z0 = [], 0
    for p in range(parts):
        n = base + (1 if p < extra else 0)
        out.append((z0, n))
        z0 += n
    return out


def slab_info(info: AcMeshInfo, z0: int, nz: int) -> AcMeshInfo:
    """The AcMeshInfo of one slab: AC_nlocal = (nx, ny, nz) with the global
    AC_ngrid and AC_ds, AC_multigpu_offset = (0, 0, z0)."""
    s = AcMeshInfo()
    C.memmove(C.byref(s), C.byref(info), C.sizeof(AcMeshInfo))
    n = s.int3_params[Int3Param.AC_ngrid]
    s.int3_params[Int3Param.AC_nlocal] = capi.Int3(n.x, n.y, nz)
    s.int3_params[Int3Param.AC_multigpu_offset] = capi.Int3(0, 0, z0)
    _check(capi.load().acHostUpdateParams(C.byref(s)), "acHostUpdateParams")
    return s


class LocalTransport:
    """All slabs in this process: slab i's bottom ghost planes come from slab
    i - 1's top interior planes and its top ghost planes from slab i + 1's
    bottom interior planes (periodically).

    With `streams` (the slabs' library streams, as torch streams) the copies
    are stream-ordered, with no host synchronisation: they run on streams[0]
    after every slab's pack, and every slab's stream then waits for them, so
    that the unpack follows the copies and the next pack into a send buffer
    follows every read of it."""

    def exchange(self, send_bottom, send_top, recv_bottom, recv_top, streams=None):
        k = len(send_bottom)
        if streams is None:
            for i in range(k):
                recv_bottom[i].copy_(send_top[(i - 1) % k])
                recv_top[i].copy_(send_bottom[(i + 1) % k])
            return
        import torch

        s0 = streams[0]
        for s in streams[1:]:
            s0.wait_stream(s)  # every slab packed
        with torch.cuda.stream(s0):
            for i in range(k):
                recv_bottom[i].copy_(send_top[(i - 1) % k])
                recv_top[i].copy_(send_bottom[(i + 1) % k])
        for s in streams[1:]:
            s.wait_stream(s0)  # copies done before unpack and the next pack

    def combine(self, values, op):
        return {"max": max, "min": min, "sum": math.fsum}[op](values)


class DistTransport:
    """One slab per rank: the top planes go to rank + 1 (its bottom ghost), the
    bottom planes to rank - 1 (its top ghost), periodically.  Sends and
    receives are posted in the same order on every rank, so messages between
    the same two ranks match in order (world size 2 has one neighbour on both
    sides).

    With `streams` (NCCL, device buffers) the point-to-point operations are
    enqueued behind the pack on the slab's library stream and waited for on
    that stream (Work.wait orders the current stream, the host does not
    block), so the unpack that follows on the same stream sees the planes."""

    def __init__(self):
        import torch.distributed as dist

        self.dist = dist
        self.rank = dist.get_rank()
        self.world = dist.get_world_size()

    def exchange(self, send_bottom, send_top, recv_bottom, recv_top, streams=None):
        (sb,), (st,), (rb,), (rt,) = send_bottom, send_top, recv_bottom, recv_top
        if streams is None:
            self._exchange(sb, st, rb, rt)
            return
        import torch

        with torch.cuda.stream(streams[0]):
            self._exchange(sb, st, rb, rt)

    def _exchange(self, sb, st, rb, rt):
        if self.world == 1:
            rb.copy_(st)
            rt.copy_(sb)
            return
        d = self.dist
        up, down = (self.rank + 1) % self.world, (self.rank - 1) % self.world
        reqs = [d.isend(st, up, tag=1), d.irecv(rb, down, tag=1),
                d.isend(sb, down, tag=2), d.irecv(rt, up, tag=2)]
        for r in reqs:
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
    """A periodic mesh of global size AC_ngrid split into z slabs.

    info: the global AcMeshInfo.  With ``transport=None`` the mesh is split into
    ``slabs`` slabs held in this process (LocalTransport); with a DistTransport
    this process holds its rank's slab of ``world`` slabs.
    """

    def __init__(self, info: AcMeshInfo, slabs: int = 1, transport=None, device_id: int = 0,
                 overlap: bool | None = None):
        import torch

        self.lib = capi.load()
        self.info = info
        self.n = dims(info)
        nz = self.n[2]
        if isinstance(transport, DistTransport):
            self.ranges = [decompose(nz, transport.world)[transport.rank]]
        else:
            transport = transport or LocalTransport()
            self.ranges = decompose(nz, slabs)
        self.transport = transport
        self.devs = [Device(slab_info(info, z0, n), device_id) for z0, n in self.ranges]
        self.plane_bytes = self.lib.acDevicePlaneBytes(self.devs[0].handle)
        dev = torch.device("cuda", device_id)
        self._streams = [torch.cuda.ExternalStream(d.stream_handle(0), device=dev)
                         for d in self.devs]
        # the interior solve of the overlapped substep runs on library stream 1
        self._streams1 = [torch.cuda.ExternalStream(d.stream_handle(1), device=dev)
                          for d in self.devs]
        if overlap is None:
            overlap = isinstance(transport, DistTransport) and transport.world > 1
        self.overlap = overlap and min(n for _, n in self.ranges) >= 2 * HALO + 1
        self._buf = {k: [torch.empty(HALO * self.plane_bytes, dtype=torch.uint8, device=dev)
                         for _ in self.devs] for k in ("sb", "st", "rb", "rt")}
        self.cells = self.n[0] * self.n[1] * self.n[2]

    def destroy(self):
        for d in self.devs:
            d.destroy()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    # ---- data ----
    def load_mesh(self, fields: np.ndarray) -> None:
        """Loads this process's slabs from a global (8, mz, my, mx) mesh."""
        for d, (z0, n) in zip(self.devs, self.ranges):
            d.load_mesh(np.ascontiguousarray(fields[:, z0:z0 + n + 2 * HALO]))

    def store_mesh(self, out: np.ndarray | None = None) -> np.ndarray:
        """The interior planes of this process's slabs in a global (8, mz, my, mx)
        array (cells of other ranks' slabs and ghost planes are left as they are)."""
        nx, ny, nz = self.n
        if out is None:
            out = np.zeros((capi.NUM_FIELDS, nz + 2 * HALO, ny + 2 * HALO, nx + 2 * HALO))
        for d, (z0, n) in zip(self.devs, self.ranges):
            s = d.store_mesh()
            out[:, HALO + z0:HALO + z0 + n] = s[:, HALO:HALO + n]
        return out

    # ---- boundary conditions ----
    def periodic_boundconds(self, interior_step=None) -> None:
        """Fills every ghost cell of every slab: x and y by local wrap, z by the
        exchange with the neighbouring slabs.  Everything is ordered on the
        slabs' library streams (stream 0); the host does not wait.

        interior_step: (step, dt) of a substep whose interior planes each slab
        solves on its stream 1 once its x/y fill is done, while the planes
        travel (the overlapped substep)."""
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


__all__ = ["Grid", "LocalTransport", "DistTransport", "decompose", "slab_info"]
