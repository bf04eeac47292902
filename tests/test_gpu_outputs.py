"""The CFL outputs through the reference's output interface
(acDeviceFinishReduceReal[Stream], acDeviceGetOutput, acDeviceSetOutput):
the values equal the maxima of the last substep 2 and the CPU formula of the
additive timestep; values set by acDeviceSetOutput are used by
acDeviceGetTimestep until the next launch that reduces them; the slab grid
combines them over slabs for both timestep forms."""
import ctypes as C
import math

import numpy as np
import pytest

from astaroth_b200 import capi
from astaroth_b200.capi import IntParam, MapKernel, RealOutputParam as Out, RealParam, ReduceOp
from astaroth_b200.device import AstarothError, Device, _check, make_info, seeded_mesh
from astaroth_b200.grid import Grid

pytestmark = pytest.mark.gpu

DT = 1e-3


def _additive_dt(info, uu_max, va_max):
    """mhdsolver.ac:558-569 with a uniform visc_dt: min(visc_dt, min over cells
    of cdt dsmin / (|u| + sqrt(cs^2 + vA^2))), bounded here from the maxima."""
    r = info.real_params
    visc = max(r[RealParam.AC_nu_visc], r[RealParam.AC_eta],
               r[RealParam.AC_gamma] * r[RealParam.AC_chi])
    visc_dt = r[RealParam.AC_cdtv] * r[RealParam.AC_dsmin] ** 2 / visc
    cs2 = r[RealParam.AC_cs_sound] ** 2
    advec_dt = r[RealParam.AC_cdt] * r[RealParam.AC_dsmin] / (uu_max + math.sqrt(cs2 + va_max ** 2))
    return visc_dt, advec_dt


@pytest.mark.parametrize("precision", [0, 1])
def test_outputs_equal_the_maxima(precision):
    info = make_info(40, precision=precision)
    with Device(info) as d:
        d.load_mesh(seeded_mesh(info, 101, sigma_uu=1e-2))
        d.integrate_step(DT)
        u, va = d.timestep_maxima()
        assert u > 0 and va > 0
        assert d.finish_reduce(Out.UU_MAX_ADVEC) == u
        assert d.finish_reduce(Out.ALFVEN_SPEED_MAX, MapKernel.AC_KERNEL_CALC_TIMESTEP) == va
        assert d.get_output(Out.UU_MAX_ADVEC) == u
        assert d.get_output(Out.ALFVEN_SPEED_MAX) == va
        # in the maximum form the additive advective sum is not formed (as the
        # reference's calc_timestep, which evaluates one form): dt_min is the
        # viscous bound alone
        visc_dt, _ = _additive_dt(info, u, va)
        assert d.get_output(Out.AC_dt_min) == visc_dt


def test_additive_timestep_is_dt_min():
    info = make_info(36)
    info.int_params[IntParam.AC_additive_timestep] = 1
    with Device(info) as d:
        d.load_mesh(seeded_mesh(info, 102, sigma_uu=1e-1))
        d.integrate_step(DT)
        assert d.timestep() == d.get_output(Out.AC_dt_min)
        # dt_min is bounded by the form evaluated with the maxima (max of a sum
        # <= sum of maxima) and by the viscous bound
        u, va = d.timestep_maxima()
        visc_dt, advec_lo = _additive_dt(info, u, va)
        dt_min = d.get_output(Out.AC_dt_min)
        assert dt_min <= visc_dt
        assert dt_min >= min(visc_dt, advec_lo) * (1 - 1e-12)
        assert d.finish_reduce(Out.AC_dt_min) == dt_min
        d.set_int(IntParam.AC_additive_timestep, 0)
        u, va = d.timestep_maxima()
        assert d.timestep() == capi.load().acHostTimestepFromMaxima(info, u, va)


def test_set_output_until_the_next_reduction():
    info = make_info(36)
    lib = capi.load()
    with Device(info) as d:
        d.load_mesh(seeded_mesh(info, 103, sigma_uu=1e-2))
        d.integrate_step(DT)
        u, va = d.timestep_maxima()
        d.set_output(Out.UU_MAX_ADVEC, 10 * u)
        assert d.get_output(Out.UU_MAX_ADVEC) == 10 * u
        assert d.get_output(Out.ALFVEN_SPEED_MAX) == va
        assert d.timestep() == lib.acHostTimestepFromMaxima(info, 10 * u, va)
        assert d.timestep_maxima() == (10 * u, va)
        # finishing the reduction again replaces the set value by the device's
        assert d.finish_reduce(Out.UU_MAX_ADVEC) == u
        assert d.get_output(Out.UU_MAX_ADVEC) == u
        # a substep 2 (graph step, per-substep calls, calc_timestep) drops set values
        for recompute in ("step", "substeps", "calc"):
            d.set_output(Out.ALFVEN_SPEED_MAX, 7.0)
            if recompute == "step":
                d.integrate_step(DT)
            elif recompute == "substeps":
                for s in range(3):
                    d.periodic_boundconds()
                    d.integrate_substep(s, DT)
                    d.swap_buffers()
            else:
                d.periodic_boundconds()
                d.calc_timestep()
            assert d.get_output(Out.ALFVEN_SPEED_MAX) != 7.0, recompute
        # substeps 0 and 1 keep them
        d.set_output(Out.ALFVEN_SPEED_MAX, 7.0)
        d.periodic_boundconds()
        d.integrate_substep(0, DT)
        assert d.get_output(Out.ALFVEN_SPEED_MAX) == 7.0


def test_finish_reduce_stream_and_errors():
    import torch

    info = make_info(32)
    lib = capi.load()
    with Device(info) as d:
        d.load_mesh(seeded_mesh(info, 104, sigma_uu=1e-2))
        d.integrate_step(DT)
        d.synchronize()
        r = C.c_double()
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        assert lib.acDeviceFinishReduceRealStream(d.handle, st, C.byref(r),
                                                  MapKernel.AC_KERNEL_SOLVE,
                                                  ReduceOp.AC_REDUCE_OP_MAX,
                                                  Out.UU_MAX_ADVEC) == 0
        assert r.value == d.timestep_maxima()[0]
        bad = [  # wrong op for the output, a map kernel, an invalid output, an invalid stream
            (0, MapKernel.AC_KERNEL_SOLVE, ReduceOp.AC_REDUCE_OP_MIN, Out.UU_MAX_ADVEC),
            (0, MapKernel.AC_KERNEL_SOLVE, ReduceOp.AC_REDUCE_OP_MAX, Out.AC_dt_min),
            (0, MapKernel.AC_MAP_VTXBUF, ReduceOp.AC_REDUCE_OP_MAX, Out.UU_MAX_ADVEC),
            (0, MapKernel.AC_KERNEL_SOLVE, ReduceOp.AC_REDUCE_OP_MAX, capi.NUM_REAL_OUTPUTS),
            (capi.STREAM_ALL, MapKernel.AC_KERNEL_SOLVE, ReduceOp.AC_REDUCE_OP_MAX,
             Out.UU_MAX_ADVEC),
        ]
        for stream, kernel, op, out in bad:
            assert lib.acDeviceFinishReduceReal(d.handle, stream, C.byref(r), kernel, op, out) != 0
        assert math.isnan(lib.acDeviceGetOutput(d.handle, capi.NUM_REAL_OUTPUTS))
        assert math.isnan(lib.acDeviceGetOutput(None, Out.UU_MAX_ADVEC))
        assert lib.acDeviceSetOutput(d.handle, -1, 1.0) != 0
        with pytest.raises(AstarothError):
            d.set_output(capi.NUM_REAL_OUTPUTS, 1.0)


@pytest.mark.parametrize("additive", [0, 1])
def test_grid_combines_outputs(additive):
    info = make_info((40, 36, 30))
    info.int_params[IntParam.AC_additive_timestep] = additive
    f = seeded_mesh(info, 105, sigma_uu=1e-2)
    with Grid(info, slabs=3) as g, Device(info) as d:
        g.load_mesh(f)
        d.load_mesh(f)
        g.integrate_step(DT)
        d.integrate_step(DT)
        assert g.timestep() == d.timestep()
        for p in Out:
            assert g.devs[1].get_output(p) == d.get_output(p)
