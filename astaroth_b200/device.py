"""Python host side over the C ABI: mesh configuration, seeded host meshes and
a thin `Device` object whose methods are the acDevice* calls.

Host meshes are numpy arrays of shape (8, mz, my, mx), float64, C order --
field-major SoA with x fastest, the layout of the reference's AcMesh
(acc-runtime/api/acc_runtime.h:58-59).  Errors from the library raise
``AstarothError`` (the C functions return AcResult codes).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import capi
from .capi import AcMesh, AcMeshInfo, Field, Int3Param, IntParam, Real3Param, RealParam, Volume


class AstarothError(RuntimeError):
    pass


def _check(res: int, what: str) -> None:
    if res != capi.AC_SUCCESS:
        raise AstarothError(f"{what} returned AcResult {res}")


# Parameters of the benchmark configurations; the rest come from the
# defaults of config/astaroth.conf (acHostMeshInfoDefault).
CONFIG_PARAMS = dict(nu_visc=5e-3, eta=5e-3, cs_sound=1.0, gamma=5.0 / 3.0, cp_sound=1.0,
                     lnT0=1.2, lnrho0=1.3, mu0=1.4, zeta=0.01, K_heatcond=1e-3)


def make_info(n, precision: int = 0, **params) -> AcMeshInfo:
    """AcMeshInfo for an n^3 (or (nx, ny, nz)) periodic box [0, 2 pi)^3.

    Keyword arguments override real params by name without the AC_ prefix,
    e.g. ``make_info(128, nu_visc=5e-3)``.
    """
    lib = capi.load()
    nx, ny, nz = (n, n, n) if np.isscalar(n) else n
    info = AcMeshInfo()
    _check(lib.acHostMeshInfoDefault(nx, ny, nz, C.byref(info)), "acHostMeshInfoDefault")
    info.int_params[IntParam.AC_precision] = precision
    for k, v in params.items():
        if k == "upwind":
            info.int_params[IntParam.AC_upwind] = int(v)
        elif k == "ds":
            info.real3_params[Real3Param.AC_ds] = capi.Real3(*v)
        else:
            info.real_params[RealParam["AC_" + k]] = float(v)
    _check(lib.acHostUpdateParams(C.byref(info)), "acHostUpdateParams")
    return info


def info_to_dict(info: AcMeshInfo) -> dict:
    """The physics params of an AcMeshInfo as a plain dict (for the oracle)."""
    r = info.real_params
    ds = info.real3_params[Real3Param.AC_ds]
    return dict(ds=(ds.x, ds.y, ds.z), nu_visc=r[RealParam.AC_nu_visc], eta=r[RealParam.AC_eta],
                cs_sound=r[RealParam.AC_cs_sound], gamma=r[RealParam.AC_gamma],
                cp_sound=r[RealParam.AC_cp_sound], lnrho0=r[RealParam.AC_lnrho0],
                lnT0=r[RealParam.AC_lnT0], mu0=r[RealParam.AC_mu0], zeta=r[RealParam.AC_zeta],
                K_heatcond=r[RealParam.AC_K_heatcond],
                upwind=info.int_params[IntParam.AC_upwind])


def dims(info: AcMeshInfo):
    n = info.int3_params[Int3Param.AC_nlocal]
    return n.x, n.y, n.z


def empty_mesh(info: AcMeshInfo) -> np.ndarray:
    nx, ny, nz = dims(info)
    g = capi.NGHOST
    return np.zeros((capi.NUM_FIELDS, nz + 2 * g, ny + 2 * g, nx + 2 * g), dtype=np.float64)


def mesh_struct(fields: np.ndarray, info: AcMeshInfo) -> AcMesh:
    """An AcMesh view of a (8, mz, my, mx) float64 C-contiguous array (no copy)."""
    if fields.dtype != np.float64 or not fields.flags.c_contiguous:
        raise ValueError("host mesh must be a C-contiguous float64 array")
    nx, ny, nz = dims(info)
    g = capi.NGHOST
    if fields.shape != (capi.NUM_FIELDS, nz + 2 * g, ny + 2 * g, nx + 2 * g):
        raise ValueError(f"host mesh shape {fields.shape} does not match the config")
    m = AcMesh()
    for q in range(capi.NUM_FIELDS):
        m.vertex_buffer[q] = fields[q].ctypes.data_as(C.POINTER(C.c_double))
    m.info = info
    return m


def seeded_mesh(info: AcMeshInfo, seed: int, amp_scalar: float = 1e-5, sigma_uu: float = 1e-3,
                sigma_aa: float = 1e-4) -> np.ndarray:
    """Seeded initial condition of the benchmark workloads (every cell incl. halos):
    lnrho, entropy ~ U(-amp, amp); uu ~ N(0, sigma_uu^2); aa ~ N(0, sigma_aa^2)."""
    lib = capi.load()
    f = empty_mesh(info)
    m = mesh_struct(f, info)
    _check(lib.acHostMeshRandomizeSeeded(C.byref(m), seed, amp_scalar, sigma_uu, sigma_aa),
           "acHostMeshRandomizeSeeded")
    return f


def solenoidal_velocity(fields: np.ndarray, info: AcMeshInfo, seed: int, nmodes: int = 64,
                        kmax: int = 8, amplitude: float = 1e-2) -> None:
    lib = capi.load()
    m = mesh_struct(fields, info)
    _check(lib.acHostMeshSolenoidalModes(C.byref(m), seed, nmodes, kmax, amplitude),
           "acHostMeshSolenoidalModes")


def timestep_from_maxima(info: AcMeshInfo, uu_max: float, alfven_max: float) -> float:
    return capi.load().acHostTimestepFromMaxima(info, uu_max, alfven_max)


@dataclass
class _Vols:
    m0: Volume
    m1: Volume
    n0: Volume
    n1: Volume


class Device:
    """One GPU running one mesh: the acDevice* API as methods."""

    def __init__(self, info: AcMeshInfo, device_id: int = 0):
        self.lib = capi.load()
        self.info = info
        self._h = capi.Device_p()
        _check(self.lib.acDeviceCreate(device_id, info, C.byref(self._h)), "acDeviceCreate")
        self.tape_token = None  # see adjoint_tape_forward
        nx, ny, nz = dims(info)
        g = capi.NGHOST
        self.vols = _Vols(Volume(0, 0, 0), Volume(nx + 2 * g, ny + 2 * g, nz + 2 * g),
                          Volume(g, g, g), Volume(nx + g, ny + g, nz + g))

    @property
    def handle(self):
        return self._h

    def destroy(self) -> None:
        if self._h:
            _check(self.lib.acDeviceDestroy(C.byref(self._h)), "acDeviceDestroy")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # ---- data movement ----
    def load_mesh(self, fields: np.ndarray, stream: int = 0) -> None:
        _check(self.lib.acDeviceLoadMesh(self._h, stream, mesh_struct(fields, self.info)),
               "acDeviceLoadMesh")

    def store_mesh(self, out: np.ndarray | None = None, stream: int = 0) -> np.ndarray:
        if out is None:
            out = empty_mesh(self.info)
        m = mesh_struct(out, self.info)
        _check(self.lib.acDeviceStoreMesh(self._h, stream, C.byref(m)), "acDeviceStoreMesh")
        return out

    def load_mesh_staged(self, fields: np.ndarray, stream: int = 1) -> None:
        """acDeviceLoadMeshStaged: starts the copy of `fields` into the device-side
        stage and returns.  `fields` must stay alive (and should be page-locked,
        e.g. a pinned torch tensor's numpy view) until commit_staged."""
        self._staged = fields  # keeps the host array alive while the copy runs
        _check(self.lib.acDeviceLoadMeshStaged(self._h, stream, mesh_struct(fields, self.info)),
               "acDeviceLoadMeshStaged")

    def commit_staged(self, stream: int = 0) -> None:
        """acDeviceCommitStagedMesh: `stream` waits for the staged copy, then the
        stage becomes the in-buffer."""
        _check(self.lib.acDeviceCommitStagedMesh(self._h, stream), "acDeviceCommitStagedMesh")

    def transfer_mesh(self, other: "Device", stream: int = 0) -> None:
        """acDeviceTransferMesh: this device's in-buffer into other's (equal dims
        and precision), on this device's stream."""
        _check(self.lib.acDeviceTransferMesh(self._h, stream, other.handle),
               "acDeviceTransferMesh")

    def swap_buffers(self) -> None:
        _check(self.lib.acDeviceSwapBuffers(self._h), "acDeviceSwapBuffers")

    def synchronize(self, stream: int = capi.STREAM_ALL) -> None:
        _check(self.lib.acDeviceSynchronizeStream(self._h, stream), "acDeviceSynchronizeStream")

    def flush_output(self, stream: int = 0) -> None:
        _check(self.lib.acDeviceFlushOutputBuffers(self._h, stream), "acDeviceFlushOutputBuffers")

    def set_int(self, param: IntParam, value: int) -> None:
        _check(self.lib.acDeviceLoadIntUniform(self._h, 0, int(param), int(value)),
               "acDeviceLoadIntUniform")

    def set_real(self, param: RealParam, value: float) -> None:
        _check(self.lib.acDeviceLoadScalarUniform(self._h, 0, int(param), float(value)),
               "acDeviceLoadScalarUniform")

    # ---- compute ----
    def periodic_boundconds(self, stream: int = 0) -> None:
        _check(self.lib.acDevicePeriodicBoundconds(self._h, stream, self.vols.m0, self.vols.m1),
               "acDevicePeriodicBoundconds")

    def integrate_substep(self, step: int, dt: float, stream: int = 0) -> None:
        _check(self.lib.acDeviceIntegrateSubstep(self._h, stream, step, self.vols.n0,
                                                 self.vols.n1, dt), "acDeviceIntegrateSubstep")

    def integrate_step_loop(self, dt: float, stream: int = 0) -> None:
        """One RK3 step as the reference's loop: boundconds, substep, swap (x3)."""
        for s in range(3):
            self.periodic_boundconds(stream)
            self.integrate_substep(s, dt, stream)
            self.swap_buffers()

    def integrate_step(self, dt: float, stream: int = 0) -> None:
        """One RK3 step through acDeviceIntegrateStep (CUDA graph)."""
        _check(self.lib.acDeviceIntegrateStep(self._h, stream, dt), "acDeviceIntegrateStep")

    # ---- reductions ----
    def reduce_scal(self, rtype: str, field: int, post: bool = True) -> float:
        out = C.c_double()
        fn = self.lib.acDeviceReduceScal if post else self.lib.acDeviceReduceScalNoPostProcessing
        _check(fn(self._h, 0, capi.RTYPES[rtype], int(field), C.byref(out)), "acDeviceReduceScal")
        return out.value

    def reduce_vec(self, rtype: str, a: int, b: int, c: int, post: bool = True) -> float:
        out = C.c_double()
        fn = self.lib.acDeviceReduceVec if post else self.lib.acDeviceReduceVecNoPostProcessing
        _check(fn(self._h, 0, capi.RTYPES[rtype], int(a), int(b), int(c), C.byref(out)),
               "acDeviceReduceVec")
        return out.value

    def reduce_vec_scal(self, rtype: str, a: int, b: int, c: int, d: int,
                        post: bool = True) -> float:
        out = C.c_double()
        fn = (self.lib.acDeviceReduceVecScal if post
              else self.lib.acDeviceReduceVecScalNoPostProcessing)
        _check(fn(self._h, 0, capi.RTYPES[rtype], int(a), int(b), int(c), int(d), C.byref(out)),
               "acDeviceReduceVecScal")
        return out.value

    def reduce_nonfinite(self) -> bool:
        """Whether the last reduction met a NaN or infinite value (after its map)."""
        v = C.c_int()
        _check(self.lib.acDeviceGetReduceNonFinite(self._h, C.byref(v)),
               "acDeviceGetReduceNonFinite")
        return bool(v.value)

    # ---- CFL timestep (computed by substep 2, or by calc_timestep) ----
    def calc_timestep(self, stream: int = 0) -> None:
        _check(self.lib.acDeviceCalcTimestep(self._h, stream), "acDeviceCalcTimestep")

    def timestep_maxima(self):
        u, va = C.c_double(), C.c_double()
        _check(self.lib.acDeviceGetTimestepMaxima(self._h, C.byref(u), C.byref(va)),
               "acDeviceGetTimestepMaxima")
        return u.value, va.value

    def timestep(self) -> float:
        dt = C.c_double()
        _check(self.lib.acDeviceGetTimestep(self._h, C.byref(dt)), "acDeviceGetTimestep")
        return dt.value

    def finish_reduce(self, output, kernel=capi.MapKernel.AC_KERNEL_SOLVE, stream: int = 0) -> float:
        """acDeviceFinishReduceReal of one CFL output (capi.RealOutputParam)."""
        op = (capi.ReduceOp.AC_REDUCE_OP_MIN if output == capi.RealOutputParam.AC_dt_min
              else capi.ReduceOp.AC_REDUCE_OP_MAX)
        r = C.c_double()
        _check(self.lib.acDeviceFinishReduceReal(self._h, stream, C.byref(r), kernel, op, output),
               "acDeviceFinishReduceReal")
        return r.value

    def get_output(self, output) -> float:
        return self.lib.acDeviceGetOutput(self._h, output)

    def set_output(self, output, value: float) -> None:
        _check(self.lib.acDeviceSetOutput(self._h, output, value), "acDeviceSetOutput")

    # ---- caller-owned device arrays (torch tensors of shape (8, mz, my, mx), float64) ----
    @staticmethod
    def _ptrs(t):
        if t is None:
            return None
        if t.dtype.__str__() != "torch.float64" or not t.is_contiguous() or t.shape[0] != 8:
            raise ValueError("expected a contiguous float64 tensor of shape (8, mz, my, mx)")
        return (C.c_void_p * 8)(*[t[q].data_ptr() for q in range(8)])

    # The library works on its own non-blocking streams, which do not order
    # against torch's stream: a read of a torch tensor first waits for torch's
    # pending work, and a write into one completes before the call returns.
    @staticmethod
    def _torch_ready(t) -> None:
        if t is not None:
            import torch
            torch.cuda.current_stream(t.device).synchronize()

    def load_mesh_device(self, t, stream: int = 0, wait_torch: bool = True) -> None:
        """wait_torch=False when t was last written by this device's own stream."""
        if wait_torch:
            self._torch_ready(t)
        _check(self.lib.acDeviceLoadMeshDevice(self._h, stream, self._ptrs(t)),
               "acDeviceLoadMeshDevice")

    def store_mesh_device(self, t, stream: int = 0, sync: bool = True):
        """sync=False when only this device's stream reads t afterwards."""
        if sync:
            self._torch_ready(t)
        _check(self.lib.acDeviceStoreMeshDevice(self._h, stream, self._ptrs(t)),
               "acDeviceStoreMeshDevice")
        if sync:
            self.synchronize(stream)
        return t

    def load_adjoint(self, t=None, stream: int = 0) -> None:
        self._torch_ready(t)
        _check(self.lib.acDeviceLoadAdjoint(self._h, stream, self._ptrs(t)), "acDeviceLoadAdjoint")

    def store_adjoint(self, t, stream: int = 0):
        self._torch_ready(t)
        _check(self.lib.acDeviceStoreAdjoint(self._h, stream, self._ptrs(t)),
               "acDeviceStoreAdjoint")
        self.synchronize(stream)
        return t

    def integrate_substep_adjoint(self, step: int, dt: float, stream: int = 0) -> None:
        _check(self.lib.acDeviceIntegrateSubstepAdjoint(self._h, stream, step, self.vols.n0,
                                                        self.vols.n1, dt),
               "acDeviceIntegrateSubstepAdjoint")

    def adjoint_tape_forward(self, steps: int, dt: float, stream: int = 0) -> object:
        """acDeviceAdjointTapeForward; returns a token that stays the device's
        `tape_token` until the tape is written again."""
        _check(self.lib.acDeviceAdjointTapeForward(self._h, stream, steps, dt),
               "acDeviceAdjointTapeForward")
        self.tape_token = object()
        return self.tape_token

    def adjoint_tape_backward(self, steps: int, dt: float, stream: int = 0) -> None:
        _check(self.lib.acDeviceAdjointTapeBackward(self._h, stream, steps, dt),
               "acDeviceAdjointTapeBackward")

    def param_adjoints(self):
        nu, eta = C.c_double(), C.c_double()
        _check(self.lib.acDeviceGetParamAdjoints(self._h, C.byref(nu), C.byref(eta)),
               "acDeviceGetParamAdjoints")
        return nu.value, eta.value

    # ---- introspection ----
    def stream_handle(self, stream: int = 0) -> int:
        return self.lib.acDeviceGetStreamHandle(self._h, stream) or 0

    def launch_count(self) -> int:
        return int(self.lib.acDeviceGetLaunchCount(self._h))

    def vertex_buffer_ptrs(self, field: int):
        pin = C.POINTER(C.c_double)()
        pout = C.POINTER(C.c_double)()
        _check(self.lib.acDeviceGetVertexBufferPtrs(self._h, int(field), C.byref(pin),
                                                    C.byref(pout)), "acDeviceGetVertexBufferPtrs")
        return C.cast(pin, C.c_void_p).value, C.cast(pout, C.c_void_p).value


__all__ = ["AstarothError", "Device", "Field", "make_info", "info_to_dict", "seeded_mesh",
           "solenoidal_velocity", "empty_mesh", "mesh_struct", "timestep_from_maxima",
           "CONFIG_PARAMS", "dims"]
