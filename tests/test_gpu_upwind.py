"""The upwinding terms (AC_upwind, the reference's LUPWD option) on the GPU,
against the oracle restatement with the same terms (itself pinned bit-exact to
the reference model built with LUPWD=1): FP64 within 1e-12 after one step for
the tiled and the plain kernel, FP32-compensated within 1e-5 of FP64."""
import numpy as np
import pytest

from astaroth_b200 import capi
from astaroth_b200.device import AstarothError, Device, info_to_dict, make_info, seeded_mesh
from astaroth_b200.ensemble import Ensemble
from oracle import oracle

pytestmark = pytest.mark.gpu

DT = 1e-3
AMP = dict(amp_scalar=1e-2, sigma_uu=3e-2, sigma_aa=3e-3)


def _gpu(info, f, steps, plain=False):
    info.int_params[capi.IntParam.AC_debug_plain_kernel] = int(plain)
    with Device(info) as d:
        d.load_mesh(f)
        for _ in range(steps):
            d.integrate_step(DT)
        d.synchronize()
        out = d.store_mesh()
    info.int_params[capi.IntParam.AC_debug_plain_kernel] = 0
    return out


@pytest.mark.parametrize("plain", [False, True])
@pytest.mark.parametrize("shape", [48, (40, 36, 44)])
def test_fp64_upwind_matches_oracle(shape, plain):
    info = make_info(shape, upwind=1)
    f = seeded_mesh(info, 51, **AMP)
    ref = f.copy()
    oracle.integrate(ref, info_to_dict(info), DT, 1, "port")
    got = _gpu(info, f, 1, plain)
    err = oracle.rel_linf(got, ref)
    assert err.max() <= 1e-12, err
    # the terms matter at this amplitude: without them lnrho and u differ
    off = f.copy()
    oracle.integrate(off, dict(info_to_dict(info), upwind=0), DT, 1, "port")
    assert oracle.rel_linf(off, ref)[:4].min() > 1e-9


def test_fp64_upwind_ten_steps():
    info = make_info(40, upwind=1)
    f = seeded_mesh(info, 52, **AMP)
    ref = f.copy()
    oracle.integrate(ref, info_to_dict(info), DT, 10, "port")
    err = oracle.rel_linf(_gpu(info, f, 10), ref)
    assert err.max() <= 1e-11, err


def test_fp32comp_upwind_near_fp64():
    i64 = make_info(48, upwind=1)
    i32 = make_info(48, precision=1, upwind=1)
    f = seeded_mesh(i64, 53, **AMP)
    err = oracle.rel_linf(_gpu(i32, f, 20), _gpu(i64, f, 20))
    assert err.max() <= 1e-5, err


def test_switching_at_run_time():
    """acDeviceLoadIntUniform(AC_upwind) selects the terms for later steps."""
    info = make_info(40)
    f = seeded_mesh(info, 54, **AMP)
    with Device(info) as d:
        d.load_mesh(f)
        d.set_int(capi.IntParam.AC_upwind, 1)
        d.integrate_step(DT)
        d.set_int(capi.IntParam.AC_upwind, 0)
        d.integrate_step(DT)
        d.synchronize()
        got = d.store_mesh()
    ref = f.copy()
    p = info_to_dict(info)
    oracle.integrate(ref, dict(p, upwind=1), DT, 1, "port")
    oracle.integrate(ref, dict(p, upwind=0), DT, 1, "port")
    assert oracle.rel_linf(got, ref).max() <= 1e-12


def test_adjoint_and_ensemble_refuse_upwinding():
    info = make_info(32, upwind=1)
    with Device(info) as d:
        d.load_mesh(seeded_mesh(info, 55))
        with pytest.raises(AstarothError):
            d.load_adjoint(None)
    with pytest.raises(AstarothError):
        Ensemble([make_info(32, precision=1, upwind=1)])
