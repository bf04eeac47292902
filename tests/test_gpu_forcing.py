"""Helical forcing (AC_lforcing, the reference's LFORCING option) on the GPU,
against the oracle restatement (pinned bit-exact to the reference model built
with LFORCING=1, tests/test_forcing.py): FP64 tiled and plain kernels within
1e-12, the time switch, parameters changed between steps, FP32-compensated
within 1e-5 of FP64."""
import ctypes as C

import numpy as np
import pytest

from astaroth_b200 import capi
from astaroth_b200.capi import IntParam, Real3, RealParam as RP
from astaroth_b200.device import CONFIG_PARAMS, Device, info_to_dict, make_info, seeded_mesh
from oracle import oracle

pytestmark = pytest.mark.gpu

DT = 1e-3


def _forcing_dict(info):
    r = info.real_params
    return dict(forcing=1, forcing_magnitude=r[RP.AC_forcing_magnitude],
                forcing_phase=r[RP.AC_forcing_phase], kaver=r[RP.AC_kaver],
                k_force=[r[RP.AC_k_forcex], r[RP.AC_k_forcey], r[RP.AC_k_forcez]],
                ff_hel_re=[r[RP.AC_ff_hel_rex], r[RP.AC_ff_hel_rey], r[RP.AC_ff_hel_rez]],
                ff_hel_im=[r[RP.AC_ff_hel_imx], r[RP.AC_ff_hel_imy], r[RP.AC_ff_hel_imz]])


def _info(n, precision=0, k=(1, 1, 0), phi=1.3, phase=0.9, magnitude=0.5, **extra):
    info = make_info(n, precision=precision, **dict(CONFIG_PARAMS, relhel=0.5,
                                                    forcing_magnitude=magnitude, kmin=0.8,
                                                    kmax=2.2, current_time=1.0, **extra))
    info.int_params[IntParam.AC_lforcing] = 1
    assert capi.load().acHostForcingParams(Real3(*k), phi, phase, C.byref(info)) == 0
    return info


def _gpu(info, f, steps, plain=False):
    info.int_params[IntParam.AC_debug_plain_kernel] = int(plain)
    with Device(info) as d:
        d.load_mesh(f)
        for _ in range(steps):
            d.integrate_step(DT)
        d.synchronize()
        out = d.store_mesh()
    info.int_params[IntParam.AC_debug_plain_kernel] = 0
    return out


@pytest.mark.parametrize("plain", [False, True])
@pytest.mark.parametrize("shape", [48, (40, 36, 44)])
def test_fp64_forcing_matches_oracle(shape, plain):
    info = _info(shape)
    f = seeded_mesh(info, 71)
    ref = f.copy()
    oracle.integrate(ref, dict(info_to_dict(info), **_forcing_dict(info)), DT, 3, "port")
    err = oracle.rel_linf(_gpu(info, f, 3, plain), ref)
    assert err.max() <= 1e-12, err


def test_switch_time_and_flag():
    """No force while AC_current_time <= AC_switch_forcing, or with AC_lforcing = 0."""
    f = None
    for info in (_info(40, switch_forcing=2.0), _info(40)):
        if info.real_params[RP.AC_switch_forcing] == 0.0:
            info.int_params[IntParam.AC_lforcing] = 0
        f = seeded_mesh(info, 72) if f is None else f
        ref = f.copy()
        oracle.integrate(ref, info_to_dict(info), DT, 1, "port")  # no forcing
        assert oracle.rel_linf(_gpu(info, f, 1), ref).max() <= 1e-12


def test_parameters_changed_between_steps():
    """New forcing parameters each step (acDeviceLoadScalarUniform), as a run
    that draws them per step does; the step graph is captured again."""
    info = _info(40)
    f = seeded_mesh(info, 73)
    lib = capi.load()
    ref = f.copy()
    with Device(info) as d:
        d.load_mesh(f)
        for step in range(3):
            cur = _info(40)
            assert lib.acHostGenerateForcingParams(11, step, C.byref(cur)) == 0
            for name in ("AC_forcing_phase", "AC_k_forcex", "AC_k_forcey", "AC_k_forcez",
                         "AC_ff_hel_rex", "AC_ff_hel_rey", "AC_ff_hel_rez", "AC_ff_hel_imx",
                         "AC_ff_hel_imy", "AC_ff_hel_imz", "AC_kaver"):
                d.set_real(RP[name], cur.real_params[RP[name]])
            d.integrate_step(DT)
            oracle.integrate(ref, dict(info_to_dict(cur), **_forcing_dict(cur)), DT, 1, "port")
        d.synchronize()
        got = d.store_mesh()
    assert oracle.rel_linf(got, ref).max() <= 1e-12


def test_fp32comp_forcing_near_fp64():
    i64, i32 = _info(48), _info(48, precision=1)
    f = seeded_mesh(i64, 74)
    err = oracle.rel_linf(_gpu(i32, f, 10), _gpu(i64, f, 10))
    assert err.max() <= 1e-5, err
