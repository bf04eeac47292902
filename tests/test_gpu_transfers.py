"""The linear-range transfers of the device layer (the reference's
acDevice{Load,Store,Transfer}{VertexBuffer,Mesh}WithOffset, acDeviceTransfer*,
include/astaroth_device.h:67-131), acDeviceUpdate / acDeviceGetLocalConfig,
and acDeviceVolumeCopy, in FP64 and FP32-compensated precision."""
import ctypes as C

import numpy as np
import pytest

import astaroth_b200 as ab
from astaroth_b200 import capi
from astaroth_b200.capi import Int3, Volume
from astaroth_b200.device import mesh_struct

pytestmark = pytest.mark.gpu

SHAPE = (20, 14, 12)


def _held(f, precision):
    """What a device of this precision holds for doubles f."""
    if precision == 0:
        return f
    hi = f.astype(np.float32)
    lo = (f - hi.astype(np.float64)).astype(np.float32)
    return hi.astype(np.float64) + lo.astype(np.float64)


def _lin(p, shape_zyx):
    mz, my, mx = shape_zyx
    return p[0] + mx * (p[1] + my * p[2])


@pytest.mark.parametrize("precision", [0, 1])
def test_load_and_store_with_offset(precision):
    info = ab.make_info(SHAPE, precision=precision)
    lib = capi.load()
    f = ab.seeded_mesh(info, 51)
    m = f.shape[1:]
    src, dst, n = (2, 3, 4), (5, 1, 2), 1234
    s0, d0 = _lin(src, m), _lin(dst, m)
    with ab.Device(info) as d:
        hm = mesh_struct(f, info)
        assert lib.acDeviceLoadVertexBufferWithOffset(d.handle, 0, hm, 3, Int3(*src), Int3(*dst),
                                                      n) == 0
        assert lib.acDeviceLoadMeshWithOffset(d.handle, 0, hm, Int3(*src), Int3(*dst), 77) == 0
        got = d.store_mesh().reshape(8, -1)
        want = np.zeros_like(got)
        flat = _held(f, precision).reshape(8, -1)
        want[:, d0:d0 + 77] = flat[:, s0:s0 + 77]
        want[3, d0:d0 + n] = flat[3, s0:s0 + n]
        assert np.array_equal(got, want)

        d.load_mesh(f)
        back = np.zeros_like(f)
        bm = mesh_struct(back, info)
        assert lib.acDeviceStoreVertexBufferWithOffset(d.handle, 0, 6, Int3(*src), Int3(*dst), n,
                                                       C.byref(bm)) == 0
        assert lib.acDeviceStoreMeshWithOffset(d.handle, 0, Int3(*dst), Int3(*src), 55,
                                               C.byref(bm)) == 0
        want = np.zeros_like(back).reshape(8, -1)
        want[6, d0:d0 + n] = flat[6, s0:s0 + n]
        want[:, s0:s0 + 55] = flat[:, d0:d0 + 55]
        assert np.array_equal(back.reshape(8, -1), want)

        # ranges past the mesh, a point outside it, a NULL host field
        total = int(np.prod(m))
        assert lib.acDeviceLoadVertexBufferWithOffset(d.handle, 0, hm, 0, Int3(0, 0, 0),
                                                      Int3(*dst), total) == capi.AC_FAILURE
        assert lib.acDeviceLoadVertexBufferWithOffset(d.handle, 0, hm, 0, Int3(m[2], 0, 0),
                                                      Int3(0, 0, 0), 1) == capi.AC_FAILURE
        hm.vertex_buffer[2] = None
        assert lib.acDeviceLoadVertexBufferWithOffset(d.handle, 0, hm, 2, Int3(0, 0, 0),
                                                      Int3(0, 0, 0), 5) == capi.AC_NOT_ALLOCATED


@pytest.mark.parametrize("precision", [0, 1])
def test_transfers_between_devices(precision):
    info = ab.make_info(SHAPE, precision=precision)
    lib = capi.load()
    f = ab.seeded_mesh(info, 52)
    flat = _held(f, precision).reshape(8, -1)
    m = f.shape[1:]
    src, dst, n = (1, 2, 3), (4, 0, 5), 999
    s0, d0 = _lin(src, m), _lin(dst, m)
    with ab.Device(info) as a, ab.Device(info) as b:
        a.load_mesh(f)
        assert lib.acDeviceTransferVertexBufferWithOffset(a.handle, 0, 5, Int3(*src), Int3(*dst),
                                                          n, b.handle) == 0
        a.synchronize()
        got = b.store_mesh().reshape(8, -1)
        want = np.zeros_like(got)
        want[5, d0:d0 + n] = flat[5, s0:s0 + n]
        assert np.array_equal(got, want)
        assert lib.acDeviceTransferMeshWithOffset(a.handle, 0, Int3(*src), Int3(*dst), 10,
                                                  b.handle) == 0
        a.synchronize()
        want[:, d0:d0 + 10] = flat[:, s0:s0 + 10]
        assert np.array_equal(b.store_mesh().reshape(8, -1), want)
        assert lib.acDeviceTransferMesh(a.handle, 0, b.handle) == 0
        a.synchronize()
        assert np.array_equal(b.store_mesh(), a.store_mesh())
        # other dims or another precision
        with ab.Device(ab.make_info((20, 14, 13), precision=precision)) as c:
            assert lib.acDeviceTransferVertexBuffer(a.handle, 0, 0, c.handle) == capi.AC_FAILURE
        with ab.Device(ab.make_info(SHAPE, precision=1 - precision)) as c:
            assert lib.acDeviceTransferMesh(a.handle, 0, c.handle) == capi.AC_FAILURE


def test_update_and_local_config():
    info = ab.make_info(SHAPE)
    lib = capi.load()
    with ab.Device(info) as d:
        cfg = lib.acDeviceGetLocalConfig(d.handle)
        cfg.real_params[capi.RealParam.AC_nu_visc] = 3e-3
        assert lib.acDeviceUpdate(d.handle, cfg) == 0
        assert lib.acDeviceGetConfig(d.handle).real_params[capi.RealParam.AC_nu_visc] == 3e-3
        assert lib.acDeviceGetLocalConfig(d.handle).real_params[capi.RealParam.AC_nu_visc] == 3e-3
        ds, iv, n3 = capi.Real3(), C.c_int(), Int3()
        assert lib.acDeviceStoreVectorUniform(d.handle, 0, capi.Real3Param.AC_ds, C.byref(ds)) == 0
        assert ds.x == info.real3_params[capi.Real3Param.AC_ds].x
        assert lib.acDeviceStoreIntUniform(d.handle, 0, capi.IntParam.AC_precision,
                                           C.byref(iv)) == 0 and iv.value == 0
        assert lib.acDeviceStoreInt3Uniform(d.handle, 0, capi.Int3Param.AC_nlocal,
                                            C.byref(n3)) == 0
        assert (n3.x, n3.y, n3.z) == SHAPE
        # the offset may be reloaded; the dimensions may not change
        assert lib.acDeviceLoadInt3Uniform(d.handle, 0, capi.Int3Param.AC_multigpu_offset,
                                           Int3(0, 0, 0)) == 0
        assert lib.acDeviceLoadInt3Uniform(d.handle, 0, capi.Int3Param.AC_nlocal,
                                           Int3(20, 14, 13)) == capi.AC_FAILURE
        assert lib.acDeviceStoreIntUniform(d.handle, 0, 99, C.byref(iv)) == capi.AC_FAILURE


def test_volume_copy():
    import torch

    info = ab.make_info(16)
    lib = capi.load()
    src = torch.randn((10, 12, 16), dtype=torch.float64, device="cuda")  # (z, y, x)
    out = torch.zeros((5, 6, 8), dtype=torch.float64, device="cuda")
    with ab.Device(info) as d:
        torch.cuda.synchronize()
        assert lib.acDeviceVolumeCopy(d.handle, 0, src.data_ptr(), Volume(3, 4, 2),
                                      Volume(16, 12, 10), out.data_ptr(), Volume(0, 0, 0),
                                      Volume(8, 6, 5)) == 0
        d.synchronize()
        assert torch.equal(out, src[2:7, 4:10, 3:11])
        # into a larger array at an offset: the box is min(in, out) = the input
        big = torch.zeros((7, 9, 10), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert lib.acDeviceVolumeCopy(d.handle, 0, out.data_ptr(), Volume(0, 0, 0),
                                      Volume(8, 6, 5), big.data_ptr(), Volume(1, 2, 1),
                                      Volume(10, 9, 7)) == 0
        d.synchronize()
        assert torch.equal(big[1:6, 2:8, 1:9], out)
        rest = big.clone()
        rest[1:6, 2:8, 1:9] = 0
        assert not rest.any()  # nothing written outside the box
        # a box that reaches past the input
        assert lib.acDeviceVolumeCopy(d.handle, 0, src.data_ptr(), Volume(9, 0, 0),
                                      Volume(16, 12, 10), out.data_ptr(), Volume(0, 0, 0),
                                      Volume(8, 6, 5)) == capi.AC_FAILURE


@pytest.mark.parametrize("precision", [0, 1])
def test_staged_loads_overlap_and_equal_direct_loads(precision):
    """acDeviceLoadMeshStaged / acDeviceCommitStagedMesh: the next input staged
    on stream 1 while stream 0 integrates the current one gives the same bits
    as loading each input directly before its steps."""
    import torch

    info = ab.make_info(SHAPE, precision=precision)
    lib = capi.load()
    inputs = [ab.seeded_mesh(info, 60 + i) for i in range(3)]
    pinned = [torch.from_numpy(f).pin_memory() for f in inputs]
    meshes = [mesh_struct(p.numpy(), info) for p in pinned]
    direct = []
    with ab.Device(info) as d:
        for f in inputs:
            d.load_mesh(f)
            d.integrate_step(1e-3)
            d.synchronize()
            direct.append(d.store_mesh())
    staged = []
    with ab.Device(info) as d:
        assert lib.acDeviceCommitStagedMesh(d.handle, 0) == capi.AC_FAILURE  # nothing staged
        assert lib.acDeviceLoadMeshStaged(d.handle, 1, meshes[0]) == 0
        for i in range(3):
            assert lib.acDeviceCommitStagedMesh(d.handle, 0) == 0
            if i + 1 < 3:
                assert lib.acDeviceLoadMeshStaged(d.handle, 1, meshes[i + 1]) == 0
            d.integrate_step(1e-3)
            d.synchronize()
            staged.append(d.store_mesh())
        bad = mesh_struct(pinned[0].numpy(), info)
        bad.vertex_buffer[4] = None
        assert lib.acDeviceLoadMeshStaged(d.handle, 1, bad) == capi.AC_NOT_ALLOCATED
    for a, b in zip(direct, staged):
        assert np.array_equal(a, b)

    # the same through the Python wrappers
    with ab.Device(info) as d, ab.Device(info) as e:
        d.load_mesh_staged(pinned[1].numpy())
        d.commit_staged()
        d.integrate_step(1e-3)
        d.synchronize()
        d.transfer_mesh(e)
        d.synchronize()
        assert np.array_equal(e.store_mesh(), direct[1])
