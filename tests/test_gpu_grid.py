"""The z-slab grid (astaroth_b200.grid) on one GPU: the mesh split into 1-4
slabs in one process (LocalTransport), or one slab in a process group of one
rank (DistTransport over NCCL), gives the same bits as one undecomposed Device
after whole RK3 steps; global reductions and the CFL timestep agree."""
import ctypes as C
import os
import socket

import numpy as np
import pytest

from astaroth_b200 import capi
from astaroth_b200.capi import IntParam, Real3
from astaroth_b200.device import CONFIG_PARAMS, Device, make_info, seeded_mesh
from astaroth_b200.grid import DistTransport, Grid

pytestmark = pytest.mark.gpu

DT = 1e-3


def _device(info, f, steps):
    with Device(info) as d:
        d.load_mesh(f)
        for _ in range(steps):
            d.integrate_step(DT)
        d.synchronize()
        return d.store_mesh()


def _interior(a):
    return a[:, 3:-3, 3:-3, 3:-3]


# overlap: the interior planes solved while the planes travel, then the ends
@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("kernel", [0, 3])  # the default choice; the leading-plane kernel
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("shape,slabs", [((40, 36, 48), 2), ((32, 32, 20), 3), ((40, 36, 48), 4),
                                         ((33, 24, 16), 1)])
def test_slabs_equal_one_device(shape, slabs, precision, kernel, overlap):
    if kernel == 3 and (precision == 0 and shape[0] % 2):
        pytest.skip("odd nx in FP64 takes the plain kernel")
    info = make_info(shape, precision=precision)
    info.int_params[IntParam.AC_debug_plain_kernel] = kernel
    f = seeded_mesh(info, 81)
    with Grid(info, slabs=slabs, overlap=overlap) as g:
        # slabs of fewer than 7 planes have no interior box: the serial substep
        assert g.overlap == (overlap and min(n for _, n in g.ranges) >= 7)
        g.load_mesh(f)
        for _ in range(3):
            g.integrate_step(DT)
        g.synchronize()
        got = g.store_mesh()
    assert np.array_equal(_interior(got), _interior(_device(info, f, 3)))


def _boxes_run(info, f, boxes, forcing=False):
    """Three RK3 steps, each substep as acDeviceIntegrateSubstep on the z boxes
    (padded z ranges) in order; the final mesh and the CFL timestep."""
    lib = capi.load()
    n = info.int3_params[capi.Int3Param.AC_nlocal]
    nx, ny = n.x, n.y
    h = capi.NGHOST
    with Device(info) as d:
        d.load_mesh(f)
        for _ in range(3):
            for s in range(3):
                d.periodic_boundconds()
                for z0, z1 in boxes:
                    assert lib.acDeviceIntegrateSubstep(d.handle, 0, s, capi.Volume(h, h, z0),
                                                        capi.Volume(nx + h, ny + h, z1),
                                                        DT) == capi.AC_SUCCESS
                d.swap_buffers()
        d.synchronize()
        return d.store_mesh(), d.timestep()


@pytest.mark.parametrize("kernel", [0, 1, 2, 3])
@pytest.mark.parametrize("precision", [0, 1])
def test_substep_in_z_boxes_equals_whole(precision, kernel):
    """acDeviceIntegrateSubstep on z boxes -- the interior planes, then the three
    at each end, as the overlapped grid substep calls it -- gives the bits of the
    whole-interior call with every kernel, and substep 2's CFL maxima cover all
    boxes (the first box clears them)."""
    shape = (64, 40, 72)
    info = make_info(shape, precision=precision)
    info.int_params[IntParam.AC_debug_plain_kernel] = kernel
    f = seeded_mesh(info, 86, sigma_uu=1e-2)
    h, nz = capi.NGHOST, shape[2]
    whole, whole_dt = _boxes_run(info, f, [(h, nz + h)])
    split, split_dt = _boxes_run(info, f, [(2 * h, nz), (h, 2 * h), (nz, nz + h)])
    assert np.array_equal(split, whole)
    assert split_dt == whole_dt
    # the boxes may come in any order (here the top first)
    split2, split2_dt = _boxes_run(info, f, [(nz, nz + h), (2 * h, nz), (h, 2 * h)])
    assert np.array_equal(split2, whole)
    assert split2_dt == whole_dt


def test_substep_z_boxes_with_forcing():
    """With helical forcing on, each box forces its own planes once."""
    info = make_info((32, 32, 24), **dict(CONFIG_PARAMS, relhel=0.5, forcing_magnitude=0.5,
                                           kmin=0.8, kmax=2.2, current_time=1.0))
    info.int_params[IntParam.AC_lforcing] = 1
    assert capi.load().acHostForcingParams(Real3(1, 0, 1), 0.4, 0.7, C.byref(info)) == 0
    f = seeded_mesh(info, 88)
    h, nz = capi.NGHOST, 24
    whole, _ = _boxes_run(info, f, [(h, nz + h)])
    split, _ = _boxes_run(info, f, [(2 * h, nz), (h, 2 * h), (nz, nz + h)])
    assert np.array_equal(split, whole)


def test_substep_rejects_partial_xy_boxes():
    info = make_info((32, 32, 24))
    lib = capi.load()
    h = capi.NGHOST
    with Device(info) as d:
        for start, end in (((h + 1, h, h), (32 + h, 32 + h, 24 + h)),
                           ((h, h, h), (32 + h, 31 + h, 24 + h)),
                           ((h, h, h - 1), (32 + h, 32 + h, 24 + h)),
                           ((h, h, 10), (32 + h, 32 + h, 10)),
                           ((h, h, h), (32 + h, 32 + h, 25 + h))):
            assert lib.acDeviceIntegrateSubstep(d.handle, 0, 0, capi.Volume(*start),
                                                capi.Volume(*end), DT) == capi.AC_FAILURE


@pytest.mark.parametrize("precision", [0, 1])
def test_slabs_with_upwinding(precision):
    """The upwinding terms (AC_upwind) are per-cell stencils too: slabs give the
    bits of one device."""
    info = make_info((40, 36, 30), precision=precision, upwind=1)
    f = seeded_mesh(info, 85, sigma_uu=1e-2)
    with Grid(info, slabs=3) as g:
        g.load_mesh(f)
        for _ in range(2):
            g.integrate_step(DT)
        g.synchronize()
        got = g.store_mesh()
    assert np.array_equal(_interior(got), _interior(_device(info, f, 2)))


def test_reductions_and_timestep():
    info = make_info((40, 36, 30))
    f = seeded_mesh(info, 82, sigma_uu=1e-2)
    with Grid(info, slabs=3, overlap=True) as g, Device(info) as d:
        assert g.overlap
        g.load_mesh(f)
        d.load_mesh(f)
        g.integrate_step(DT)
        d.integrate_step(DT)
        for rt in ("RTYPE_MAX", "RTYPE_MIN"):
            assert g.reduce_scal(rt, 2) == d.reduce_scal(rt, 2)
            assert g.reduce_vec(rt, 1, 2, 3) == d.reduce_vec(rt, 1, 2, 3)
        for rt in ("RTYPE_RMS", "RTYPE_SUM", "RTYPE_RMS_EXP"):
            assert g.reduce_scal(rt, 0) == pytest.approx(d.reduce_scal(rt, 0), rel=1e-13)
        # the maxima of the last substep 2, combined over the slabs with max
        assert g.timestep() == d.timestep()


def test_forcing_across_slabs():
    """The forcing phase of each slab is shifted by its z offset."""
    info = make_info((32, 32, 24), **dict(CONFIG_PARAMS, relhel=0.5, forcing_magnitude=0.5,
                                           kmin=0.8, kmax=2.2, current_time=1.0))
    info.int_params[IntParam.AC_lforcing] = 1
    assert capi.load().acHostForcingParams(Real3(1, 0, 1), 0.4, 0.7, C.byref(info)) == 0
    f = seeded_mesh(info, 83)
    with Grid(info, slabs=3, overlap=True) as g:
        assert g.overlap
        g.load_mesh(f)
        g.integrate_step(DT)
        g.synchronize()
        got = g.store_mesh()
    ref = _device(info, f, 1)
    err = np.abs(_interior(got) - _interior(ref)).max() / np.abs(_interior(ref)).max()
    assert err <= 1e-13


@pytest.mark.parametrize("precision", [0, 1])
def test_pack_unpack_box(precision):
    """acDevicePackBox gathers a box of every array (x fastest), acDeviceUnpackBox
    scatters it into another device at the same place and nowhere else; boxes
    outside the padded mesh are refused."""
    import torch

    lib = capi.load()
    info = make_info((20, 16, 12), precision=precision)
    f = seeded_mesh(info, 90)
    start, size = capi.Int3(2, 5, 4), capi.Int3(7, 3, 9)
    with Device(info) as a, Device(info) as b:
        a.load_mesh(f)
        b.load_mesh(np.zeros_like(f))
        nbytes = lib.acDeviceBoxBytes(a.handle, size)
        assert nbytes == 7 * 3 * 9 * 8 * 8  # 8 fields of 8 B, or 16 arrays of 4 B
        buf = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        assert lib.acDevicePackBox(a.handle, 0, start, size, buf.data_ptr()) == capi.AC_SUCCESS
        assert lib.acDeviceUnpackBox(b.handle, 0, start, size, buf.data_ptr()) == capi.AC_SUCCESS
        a.synchronize()
        b.synchronize()
        got = b.store_mesh()
        if precision == 0:
            packed = buf.cpu().numpy().view(np.float64).reshape(8, 9, 3, 7)
            assert np.array_equal(packed, f[:, 4:13, 5:8, 2:9])
        box = np.zeros(got.shape, dtype=bool)
        box[:, 4:13, 5:8, 2:9] = True
        assert np.array_equal(got[box], a.store_mesh()[box])
        assert not got[~box].any()
        for st, sz in (((-1, 0, 0), (3, 3, 3)), ((0, 0, 0), (27, 1, 1)), ((0, 20, 0), (1, 3, 1)),
                       ((0, 0, 0), (0, 1, 1))):
            assert lib.acDevicePackBox(a.handle, 0, capi.Int3(*st), capi.Int3(*sz),
                                       buf.data_ptr()) == capi.AC_FAILURE
        assert lib.acDeviceBoxBytes(a.handle, capi.Int3(0, 4, 4)) == 0


# process grids: x, y and z split, ranks linear or in the reference's Morton order
PENCILS = [((2, 1, 1), "linear"), ((1, 2, 1), "linear"), ((2, 2, 1), "linear"),
           ((2, 2, 2), "morton"), ((1, 3, 2), "linear"), ("morton", None)]


@pytest.mark.parametrize("kernel", [0, 3])
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("decomp,mapping", PENCILS)
def test_pencils_equal_one_device(decomp, mapping, precision, kernel):
    """A mesh split in x, y and z (the three-pass exchange of acDevicePackBox /
    acDeviceUnpackBox) gives the bits of one undecomposed Device.  Every
    sub-domain is at least one 32-cell tile wide, so the kernel of the whole
    mesh runs on every sub-domain too (narrower meshes take the plain kernel)."""
    info = make_info((64, 40, 30), precision=precision)
    info.int_params[IntParam.AC_debug_plain_kernel] = kernel
    f = seeded_mesh(info, 91, sigma_uu=1e-2)
    kw = dict(decomp=decomp, slabs=4) if mapping is None else dict(decomp=decomp, mapping=mapping)
    with Grid(info, **kw) as g:
        assert not g.slabs_only and not g.overlap
        g.load_mesh(f)
        for _ in range(3):
            g.integrate_step(DT)
        g.synchronize()
        got = g.store_mesh()
    assert np.array_equal(_interior(got), _interior(_device(info, f, 3)))


def test_pencils_reductions_timestep_and_forcing():
    """Reductions and the CFL timestep of a (2, 2, 2) grid equal one Device's;
    with forcing on, the phase of each block is shifted by its x, y and z
    offsets."""
    info = make_info((64, 40, 30))
    f = seeded_mesh(info, 92, sigma_uu=1e-2)
    with Grid(info, decomp=(2, 2, 2)) as g, Device(info) as d:
        g.load_mesh(f)
        d.load_mesh(f)
        g.integrate_step(DT)
        d.integrate_step(DT)
        for rt in ("RTYPE_MAX", "RTYPE_MIN"):
            assert g.reduce_scal(rt, 2) == d.reduce_scal(rt, 2)
            assert g.reduce_vec(rt, 1, 2, 3) == d.reduce_vec(rt, 1, 2, 3)
        for rt in ("RTYPE_RMS", "RTYPE_SUM", "RTYPE_RMS_EXP"):
            assert g.reduce_scal(rt, 0) == pytest.approx(d.reduce_scal(rt, 0), rel=1e-13)
        assert g.timestep() == d.timestep()
    info = make_info((32, 32, 24), **dict(CONFIG_PARAMS, relhel=0.5, forcing_magnitude=0.5,
                                           kmin=0.8, kmax=2.2, current_time=1.0))
    info.int_params[IntParam.AC_lforcing] = 1
    assert capi.load().acHostForcingParams(Real3(1, 0, 1), 0.4, 0.7, C.byref(info)) == 0
    f = seeded_mesh(info, 93)
    with Grid(info, decomp=(2, 2, 1)) as g:
        g.load_mesh(f)
        g.integrate_step(DT)
        g.synchronize()
        got = g.store_mesh()
    ref = _device(info, f, 1)
    err = np.abs(_interior(got) - _interior(ref)).max() / np.abs(_interior(ref)).max()
    assert err <= 1e-13


def test_dist_transport_one_rank():
    import torch.distributed as dist

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("nccl", rank=0, world_size=1)
    try:
        info = make_info((32, 28, 24))
        f = seeded_mesh(info, 84)
        with Grid(info, transport=DistTransport(), overlap=True) as g:
            assert g.overlap
            g.load_mesh(f)
            for _ in range(2):
                g.integrate_step(DT)
            g.synchronize()
            got = g.store_mesh()
            assert g.reduce_scal("RTYPE_MAX", 1) == _device_max(info, f)
        assert np.array_equal(_interior(got), _interior(_device(info, f, 2)))
    finally:
        dist.destroy_process_group()


def _device_max(info, f):
    with Device(info) as d:
        d.load_mesh(f)
        for _ in range(2):
            d.integrate_step(DT)
        return d.reduce_scal("RTYPE_MAX", 1)
