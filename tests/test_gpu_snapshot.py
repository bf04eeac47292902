"""Device snapshots (acDeviceWriteMeshToDisk / acDeviceReadMeshFromDisk) on
the GPU: the files hold exactly the interior of the in-buffers, the restored
state is bit-identical with its halos as the periodic fill, and a restart
continues bit for bit in FP64 (within FP32 rounding for FP32-compensated
meshes, whose (hi, lo) pairs are re-split from the stored doubles)."""
import numpy as np
import pytest

from astaroth_b200 import capi
from astaroth_b200 import snapshot as snap
from astaroth_b200.device import Device, dims, make_info, seeded_mesh
from oracle import oracle

pytestmark = pytest.mark.gpu

SHAPE = (40, 36, 32)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("segmented", [0, 1])
def test_write_read_restart(tmp_path, precision, segmented):
    info = make_info(SHAPE, precision=precision)
    lib = capi.load()
    d = str(tmp_path / "snap").encode()
    with Device(info) as a:
        a.load_mesh(seeded_mesh(info, 31))
        a.integrate_step(1e-3)
        a.synchronize()
        state = a.store_mesh()
        assert lib.acDeviceWriteMeshToDisk(a.handle, d, b"step-1", segmented) == capi.AC_SUCCESS
        seg = {(0, 0, 0): SHAPE} if segmented else None
        on_disk = snap.read_mesh(tmp_path / "snap", "step-1", dims(info), segments=seg)
        assert np.array_equal(on_disk, state[:, 3:-3, 3:-3, 3:-3])
        a.integrate_step(1e-3)
        a.synchronize()
        want = a.store_mesh()
    with Device(info) as b:
        assert lib.acDeviceReadMeshFromDisk(b.handle, d, b"step-1", segmented) == capi.AC_SUCCESS
        restored = b.store_mesh()
        assert np.array_equal(restored[:, 3:-3, 3:-3, 3:-3], state[:, 3:-3, 3:-3, 3:-3])
        filled = state.copy()
        oracle.periodic_bounds(filled, "port")
        assert np.array_equal(restored, filled)  # halos: the periodic fill
        b.integrate_step(1e-3)
        b.synchronize()
        got = b.store_mesh()
    if precision == 0:
        assert np.array_equal(got[:, 3:-3, 3:-3, 3:-3], want[:, 3:-3, 3:-3, 3:-3])
    else:
        # The file holds hi + lo as a double.  Splitting it again gives the same
        # pair except where lo was exactly half an ulp of hi (a rounding tie):
        # the same value, but the stencils read hi, so the next step may differ
        # at FP32 rounding level.
        assert oracle.rel_linf(got, want).max() <= 1e-6


def test_read_errors(tmp_path):
    info = make_info(SHAPE)
    lib = capi.load()
    with Device(info) as a:
        a.load_mesh(seeded_mesh(info, 32))
        assert lib.acDeviceReadMeshFromDisk(a.handle, str(tmp_path / "none").encode(), b"x",
                                            0) != capi.AC_SUCCESS
        d = str(tmp_path / "s").encode()
        assert lib.acDeviceWriteMeshToDisk(a.handle, d, b"x", 0) == capi.AC_SUCCESS
        # a field file one value short is rejected
        p = snap.mesh_path(tmp_path / "s", 2, "x")
        p.write_bytes(p.read_bytes()[:-8])
        assert lib.acDeviceReadMeshFromDisk(a.handle, d, b"x", 0) != capi.AC_SUCCESS
    # a snapshot of another mesh size is rejected (the files are too long)
    big = make_info((40, 36, 33))
    with Device(big) as c:
        c.load_mesh(seeded_mesh(big, 33))
        d2 = str(tmp_path / "t").encode()
        assert lib.acDeviceWriteMeshToDisk(c.handle, d2, b"y", 0) == capi.AC_SUCCESS
    with Device(info) as e:
        assert lib.acDeviceReadMeshFromDisk(e.handle, str(tmp_path / "t").encode(), b"y",
                                            0) != capi.AC_SUCCESS
