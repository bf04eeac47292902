"""The failure path of the tiled solve kernels, exercised without a GPU fault.

The kernels wait on mbarriers for their shared-memory plane loads, each wait
with an iteration bound.  acDeviceDebugSkipPlaneLoad makes every block skip the
load of its last plane: that wait runs out (after a short bound), the kernel
sets the device error word, waits (bounded) until every load it did issue has
landed, frees its tensor memory and completes.  acDeviceSynchronizeStream then
reports AC_FAILURE once, and the device keeps working: a clean run on it
afterwards gives the same bits as a fresh device.
"""
import numpy as np
import pytest

import astaroth_b200 as ab
from astaroth_b200 import capi
from tests.conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

P = capi.IntParam


def clean_step(info, f, kernel):
    with ab.Device(info) as dev:
        dev.set_int(P.AC_debug_plain_kernel, kernel)
        dev.load_mesh(f)
        dev.integrate_step(1e-3)
        return dev.store_mesh()


@pytest.mark.parametrize("precision", [0, 1])
# the leading-plane kernel with the group exchange through tensor memory or
# shared memory, the per-plane tap kernel
@pytest.mark.parametrize("kernel", [3, 4, 2])
def test_bounded_wait_gives_up_and_device_recovers(precision, kernel):
    info = ab.make_info((64, 16, 40), precision=precision, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 3)
    lib = capi.load()
    with ab.Device(info) as dev:
        dev.set_int(P.AC_debug_plain_kernel, kernel)
        dev.load_mesh(f)
        dev.synchronize()
        assert lib.acDeviceDebugSkipPlaneLoad(dev.handle, 1) == capi.AC_SUCCESS
        dev.periodic_boundconds()
        dev.integrate_substep(0, 1e-3)
        # the wait that ran out is reported once ...
        assert lib.acDeviceSynchronizeStream(dev.handle, 0) == capi.AC_FAILURE
        # ... and cleared with the report
        assert lib.acDeviceSynchronizeStream(dev.handle, 0) == capi.AC_SUCCESS
        # the device stays usable: a clean step from a reloaded mesh
        assert lib.acDeviceDebugSkipPlaneLoad(dev.handle, 0) == capi.AC_SUCCESS
        dev.load_mesh(f)
        dev.integrate_step(1e-3)
        assert lib.acDeviceSynchronizeStream(dev.handle, capi.STREAM_ALL) == capi.AC_SUCCESS
        got = dev.store_mesh()
    assert np.array_equal(got, clean_step(info, f, kernel))
