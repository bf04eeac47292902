"""The auxiliary field B = curl A (AC_lbfield, the reference's LBFIELD) on the
GPU: after a step it equals the 6th-order curl of the input of substep 2,
computed here with numpy from that state."""
import ctypes as C

import numpy as np
import pytest

from astaroth_b200 import capi
from astaroth_b200.device import AstarothError, Device, _check, make_info, seeded_mesh
from oracle import oracle

pytestmark = pytest.mark.gpu

DT = 1e-3
D1 = (3 / 4, -3 / 20, 1 / 60)


def _d1(f, axis, ds):
    """6th-order first derivative of a halo-filled (mz, my, mx) array, interior only."""
    out = 0
    for k, c in zip((1, 2, 3), D1):
        out = out + c * (np.roll(f, -k, axis) - np.roll(f, k, axis))
    return (out / ds)[3:-3, 3:-3, 3:-3]


def _curl(state, info):
    ds = info.real3_params[capi.Real3Param.AC_ds]
    dx, dy, dz = ds.x, ds.y, ds.z
    ax, ay, az = state[4], state[5], state[6]
    # array axes (z, y, x) = (0, 1, 2)
    return np.stack([_d1(az, 1, dy) - _d1(ay, 0, dz), _d1(ax, 0, dz) - _d1(az, 2, dx),
                     _d1(ay, 2, dx) - _d1(ax, 1, dy)])


def _store_b(d, info):
    nx, ny, nz = (info.int3_params[capi.Int3Param.AC_nlocal].x,
                  info.int3_params[capi.Int3Param.AC_nlocal].y,
                  info.int3_params[capi.Int3Param.AC_nlocal].z)
    b = np.zeros((3, nz + 6, ny + 6, nx + 6))
    p = [b[c].ctypes.data_as(C.POINTER(C.c_double)) for c in range(3)]
    _check(d.lib.acDeviceStoreBfield(d.handle, 0, *p), "acDeviceStoreBfield")
    return b


@pytest.mark.parametrize("precision,tol", [(0, 1e-13), (1, 1e-6)])
@pytest.mark.parametrize("shape", [40, (36, 44, 32)])
def test_bfield_is_curl_of_substep2_input(shape, precision, tol):
    info = make_info(shape, precision=precision)
    info.int_params[capi.IntParam.AC_lbfield] = 1
    with Device(info) as d:
        d.load_mesh(seeded_mesh(info, 91))
        for s in (0, 1):
            d.periodic_boundconds()
            d.integrate_substep(s, DT)
            d.swap_buffers()
        d.periodic_boundconds()
        d.synchronize()
        state = d.store_mesh()  # the input of substep 2, halos filled
        d.integrate_substep(2, DT)
        d.swap_buffers()
        d.synchronize()
        b = _store_b(d, info)
    want = _curl(state, info)
    got = b[:, 3:-3, 3:-3, 3:-3]
    assert np.abs(got - want).max() <= tol * np.abs(want).max()
    assert not b[:, :3].any()  # halo entries stay 0


def test_bfield_after_graph_step_and_switching():
    info = make_info(40)
    with Device(info) as d:
        d.load_mesh(seeded_mesh(info, 92))
        with pytest.raises(AstarothError):
            _store_b(d, info)  # AC_lbfield not set
        d.set_int(capi.IntParam.AC_lbfield, 1)
        d.integrate_step(DT)
        d.synchronize()
        b1 = _store_b(d, info)
        # the same through the per-substep calls from the same start
        d.load_mesh(seeded_mesh(info, 92))
        for s in range(3):
            d.periodic_boundconds()
            d.integrate_substep(s, DT)
            d.swap_buffers()
        d.synchronize()
        b2 = _store_b(d, info)
    assert np.array_equal(b1, b2)
    assert np.abs(b1).max() > 0
