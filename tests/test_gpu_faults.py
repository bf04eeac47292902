"""Failure detection, exercised without a GPU fault: the bounded waits of the
tiled solve kernels, the non-finite flag of the reductions, and host-side fault
injection into device creation and substep launches (AC_FAULT_INJECT).

Bounded waits: the kernels wait on mbarriers for their shared-memory plane loads, each wait
with an iteration bound.  acDeviceDebugSkipPlaneLoad makes every block skip the
load of its last plane: that wait runs out (after a short bound), the kernel
sets the device error word, waits (bounded) until every load it did issue has
landed, frees its tensor memory and completes.  acDeviceSynchronizeStream then
reports AC_FAILURE once, and the device keeps working: a clean run on it
afterwards gives the same bits as a fresh device.
"""
import ctypes as C

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


# ---------------------------------------------------------------- NaN / Inf flag

@pytest.mark.parametrize("precision", [0, 1])
def test_reduction_flags_nonfinite_values(precision):
    """acDeviceGetReduceNonFinite: a NaN in a field is dropped by a maximum
    (fmax), so only the flag shows it; an infinity makes a sum non-finite and
    sets the flag; clean fields clear it."""
    info = ab.make_info(24, precision=precision, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 5)
    f[1, 10, 11, 12] = np.nan
    f[2, 13, 9, 7] = np.inf
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        assert np.isfinite(dev.reduce_scal("RTYPE_MAX", 1))
        assert dev.reduce_nonfinite()
        assert not np.isfinite(dev.reduce_scal("RTYPE_SUM", 2))
        assert dev.reduce_nonfinite()
        dev.reduce_scal("RTYPE_MAX", 3)
        assert not dev.reduce_nonfinite()
        dev.reduce_vec("RTYPE_RMS", 1, 3, 4)  # the NaN through a vector map
        assert dev.reduce_nonfinite()
        dev.reduce_vec_scal("RTYPE_ALFVEN_MAX", 4, 5, 6, 0)
        assert not dev.reduce_nonfinite()


# ---------------------------------------------------------------- fault injection

def _free_bytes():
    import torch

    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


@pytest.mark.parametrize("site", ["create", "alloc"])
def test_injected_create_failure_leaks_nothing(site, monkeypatch):
    """AC_FAULT_INJECT=create / alloc: acDeviceCreate returns AC_FAILURE (the
    alloc case after its first state block was allocated) and releases what it
    took; without the variable the next create works."""
    info = ab.make_info(128, **ab.CONFIG_PARAMS)  # 154 MB per state block
    with ab.Device(info):
        pass  # context and library set-up outside the measurement
    free0 = _free_bytes()
    lib = capi.load()
    monkeypatch.setenv("AC_FAULT_INJECT", site)
    handle = capi.Device_p()
    assert lib.acDeviceCreate(0, info, C.byref(handle)) == capi.AC_FAILURE
    assert not handle
    assert abs(_free_bytes() - free0) < 64 << 20
    monkeypatch.delenv("AC_FAULT_INJECT")
    with ab.Device(info) as dev:
        dev.load_mesh(ab.seeded_mesh(info, 1))
        dev.integrate_step(1e-3)
    assert abs(_free_bytes() - free0) < 64 << 20


@pytest.mark.parametrize("precision", [0, 1])
def test_injected_launch_failure_keeps_state(precision, monkeypatch):
    """AC_FAULT_INJECT=launch: substeps and whole steps (whose graph capture
    then ends early) return AC_FAILURE and leave the buffers as they were; once
    the variable is gone the device steps to the bits of a fresh one."""
    info = ab.make_info((64, 16, 40), precision=precision, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 6)
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        monkeypatch.setenv("AC_FAULT_INJECT", "launch")
        with pytest.raises(ab.AstarothError):
            dev.integrate_substep(0, 1e-3)
        with pytest.raises(ab.AstarothError):
            dev.integrate_step(1e-3)
        monkeypatch.delenv("AC_FAULT_INJECT")
        dev.integrate_step(1e-3)
        got = dev.store_mesh()
    with ab.Device(info) as ref:
        ref.load_mesh(f)
        ref.integrate_step(1e-3)
        want = ref.store_mesh()
    assert np.array_equal(got, want)
