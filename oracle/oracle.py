"""Test infrastructure only: ctypes access to the two CPU oracles.

* ``port``      -- liboracle.so, the project's C restatement (astaroth_oracle.c)
* ``reference`` -- _ref/libastaroth_ref.so, the reference's own host model files
                   (src/utils/{modelsolver,memory,modelreduce,verification}.cc)
                   compiled unchanged against oracle/shim (oracle/Makefile).
* ``reference_upwd`` -- the same built with LUPWD=1 (the upwinding terms).
* ``reference_forcing`` -- the same built with LFORCING=1 (helical forcing).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker; the product library never loads it.  Meshes are
numpy arrays of shape (8, mz, my, mx), float64, C order.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libastaroth_ref.so"
REF_UPWD_LIB = HERE / "_ref" / "libastaroth_ref_upwd.so"
REF_FORCING_LIB = HERE / "_ref" / "libastaroth_ref_forcing.so"
_PATHS = {"port": PORT_LIB, "reference": REF_LIB, "reference_upwd": REF_UPWD_LIB,
          "reference_forcing": REF_FORCING_LIB}
# The reference tree: $AC_REFERENCE, else a checkout named "reference" beside
# this repository.  Only the reference model build (_ref/) needs it.
REF_SRC = Path(os.environ.get("AC_REFERENCE", str(HERE.parent.parent / "reference")))

# Physics of the benchmark workloads (the reference's config/astaroth.conf
# values where the workloads give none): nu = eta = 5e-3, cs = 1, gamma = 5/3.
BENCH_PARAMS = dict(nu_visc=5e-3, eta=5e-3, cs_sound=1.0, gamma=5.0 / 3.0, cp_sound=1.0,
                    lnT0=1.2, lnrho0=1.3, mu0=1.4, zeta=0.01, K_heatcond=1e-3)

RTYPE_NAMES = ["RTYPE_MAX", "RTYPE_MIN", "RTYPE_SUM", "RTYPE_RMS", "RTYPE_RMS_EXP",
               "RTYPE_ALFVEN_MAX", "RTYPE_ALFVEN_MIN", "RTYPE_ALFVEN_RMS"]


class OracleParams(C.Structure):
    _fields_ = [("ds", C.c_double * 3), ("nu_visc", C.c_double), ("eta", C.c_double),
                ("cs_sound", C.c_double), ("gamma", C.c_double), ("cp_sound", C.c_double),
                ("lnrho0", C.c_double), ("lnT0", C.c_double), ("mu0", C.c_double),
                ("zeta", C.c_double), ("K_heatcond", C.c_double), ("upwind", C.c_int),
                ("forcing", C.c_int), ("f_magnitude", C.c_double), ("f_phase", C.c_double),
                ("f_kaver", C.c_double), ("f_k", C.c_double * 3), ("f_re", C.c_double * 3),
                ("f_im", C.c_double * 3)]


def make_params(p: dict) -> OracleParams:
    o = OracleParams()
    o.ds[:] = list(p["ds"])
    for k in ("nu_visc", "eta", "cs_sound", "gamma", "cp_sound", "lnrho0", "lnT0", "mu0", "zeta",
              "K_heatcond"):
        setattr(o, k, float(p[k]))
    o.upwind = int(p.get("upwind", 0))
    o.forcing = int(p.get("forcing", 0))
    if o.forcing:
        o.f_magnitude = float(p["forcing_magnitude"])
        o.f_phase = float(p["forcing_phase"])
        o.f_kaver = float(p["kaver"])
        o.f_k[:] = list(p["k_force"])
        o.f_re[:] = list(p["ff_hel_re"])
        o.f_im[:] = list(p["ff_hel_im"])
    return o


def build() -> None:
    """Builds liboracle.so, and _ref/ where the reference sources are present."""
    subprocess.run(["make", "-s", "-C", str(HERE), f"REF={REF_SRC}"], check=True)


_libs: dict[str, C.CDLL] = {}


def available(kind: str) -> bool:
    return _PATHS[kind].exists()


def lib(kind: str = "port") -> C.CDLL:
    if kind in _libs:
        return _libs[kind]
    path = _PATHS[kind]
    if not path.exists():
        raise RuntimeError(f"oracle library {path} is missing (run `make -C oracle`)")
    L = C.CDLL(str(path))
    pp = C.POINTER(C.POINTER(C.c_double))
    prefix = "oracle" if kind == "port" else "ref"
    f = getattr(L, f"{prefix}_integrate")
    f.restype, f.argtypes = C.c_int, [pp, C.c_int, C.c_int, C.c_int, C.POINTER(OracleParams),
                                      C.c_double, C.c_int]
    f = getattr(L, f"{prefix}_periodic_bounds")
    f.restype, f.argtypes = C.c_int, [pp, C.c_int, C.c_int, C.c_int]
    f = getattr(L, f"{prefix}_reduce")
    f.restype, f.argtypes = C.c_double, [pp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                         C.c_int, C.c_int, C.c_int, C.c_int]
    if kind == "port":
        L.oracle_seeded_mesh.restype = C.c_int
        L.oracle_seeded_mesh.argtypes = [pp, C.c_int, C.c_int, C.c_int, C.c_ulonglong,
                                         C.c_double, C.c_double, C.c_double]
        L.oracle_rates.restype = C.c_int
        L.oracle_rates.argtypes = [pp, C.c_int, C.c_int, C.c_int, C.POINTER(OracleParams), pp]
    else:
        L.ref_verify.restype = C.c_int
        L.ref_verify.argtypes = [pp, pp, C.c_int, C.c_int, C.c_int, C.c_double]
        L.ref_get_error.restype = None
        L.ref_get_error.argtypes = [C.c_double, C.c_double, C.POINTER(C.c_longdouble)]
    _libs[kind] = L
    return L


def box_params(n, **over) -> dict:
    """Oracle params of an n^3 (or (nx, ny, nz)) periodic box [0, 2 pi)^3 with
    the benchmark physics, overridden by keyword."""
    nx, ny, nz = (n, n, n) if np.isscalar(n) else n
    two_pi = 6.283185307179586476925286766559
    p = dict(BENCH_PARAMS, ds=(two_pi / nx, two_pi / ny, two_pi / nz), upwind=0)
    p.update(over)
    return p


def seeded_mesh(n, seed: int, amp_scalar: float = 1e-5, sigma_uu: float = 1e-3,
                sigma_aa: float = 1e-4) -> np.ndarray:
    """The seeded initial condition of the benchmark workloads, made by the port
    (bytes equal to the product's acHostMeshRandomizeSeeded; the golden input
    hashes pin both)."""
    nx, ny, nz = (n, n, n) if np.isscalar(n) else n
    f = np.zeros((8, nz + 6, ny + 6, nx + 6))
    if lib("port").oracle_seeded_mesh(_ptrs(f), nx, ny, nz, seed, amp_scalar, sigma_uu,
                                      sigma_aa) != 0:
        raise RuntimeError("oracle seeded mesh failed")
    return f


def _ptrs(fields: np.ndarray):
    assert fields.dtype == np.float64 and fields.flags.c_contiguous and fields.shape[0] == 8
    arr = (C.POINTER(C.c_double) * 8)()
    for q in range(8):
        arr[q] = fields[q].ctypes.data_as(C.POINTER(C.c_double))
    return arr


def _n(fields: np.ndarray):
    _, mz, my, mx = fields.shape
    return mx - 6, my - 6, mz - 6


def integrate(fields: np.ndarray, params: dict, dt: float, nsteps: int = 1,
              kind: str = "port") -> None:
    """In place: nsteps RK3 steps, each with a periodic halo fill before every substep."""
    L = lib(kind)
    fn = L.oracle_integrate if kind == "port" else L.ref_integrate
    p = make_params(params)
    rc = fn(_ptrs(fields), *_n(fields), C.byref(p), dt, nsteps)
    if rc != 0:
        raise RuntimeError("oracle integrate failed")


def periodic_bounds(fields: np.ndarray, kind: str = "port") -> None:
    L = lib(kind)
    fn = L.oracle_periodic_bounds if kind == "port" else L.ref_periodic_bounds
    if fn(_ptrs(fields), *_n(fields)) != 0:
        raise RuntimeError("oracle periodic bounds failed")


def reduce(fields: np.ndarray, rtype: str, handles, kind: str = "port") -> float:
    """Reduction of the interior; len(handles) = 1 (scal), 3 (vec) or 4 (vec+scal)."""
    L = lib(kind)
    fn = L.oracle_reduce if kind == "port" else L.ref_reduce
    h = list(handles) + [0] * (4 - len(handles))
    return fn(_ptrs(fields), *_n(fields), len(handles), RTYPE_NAMES.index(rtype), *h)


def rates(fields: np.ndarray, params: dict) -> np.ndarray:
    """RHS at every interior cell (halos of `fields` must be filled)."""
    out = np.zeros_like(fields)
    p = make_params(params)
    if lib("port").oracle_rates(_ptrs(fields), *_n(fields), C.byref(p), _ptrs(out)) != 0:
        raise RuntimeError("oracle rates failed")
    return out


def ref_verify(model: np.ndarray, candidate: np.ndarray, max_ulp: float = 5.0) -> bool:
    """The reference's acVerifyMeshWithMaximumError verdict (True = all fields pass)."""
    return lib("reference").ref_verify(_ptrs(model), _ptrs(candidate), *_n(model), max_ulp) == 0


def interior(f: np.ndarray) -> np.ndarray:
    return f[..., 3:-3, 3:-3, 3:-3]


def rel_linf(cand: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """Per-field relative L-infinity error over the interior: max|c - r| / max|r|."""
    c, r = interior(cand), interior(ref)
    num = np.abs(c - r).reshape(8, -1).max(axis=1)
    den = np.abs(r).reshape(8, -1).max(axis=1)
    return num / np.where(den > 0, den, 1.0)


def rel_l2(cand: np.ndarray, ref: np.ndarray) -> np.ndarray:
    c, r = interior(cand), interior(ref)
    num = np.sqrt(((c - r) ** 2).reshape(8, -1).sum(axis=1))
    den = np.sqrt((r ** 2).reshape(8, -1).sum(axis=1))
    return num / np.where(den > 0, den, 1.0)
