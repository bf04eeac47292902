"""ctypes mirror of the astaroth_b200 C ABI (include/astaroth_b200.h).

Every structure and enum here has the layout and values of the header; a
CPU test parses the header and checks them.  The library is loaded from the
package directory; there is no fallback: a missing or stale library raises.
"""
from __future__ import annotations

import ctypes as C
import enum
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libastaroth_b200.so"

NGHOST = 3
NUM_FIELDS = 8
NUM_STREAMS = 32


class Field(enum.IntEnum):
    LNRHO = 0
    UUX = 1
    UUY = 2
    UUZ = 3
    AX = 4
    AY = 5
    AZ = 6
    ENTROPY = 7


FIELD_NAMES = ["VTXBUF_LNRHO", "VTXBUF_UUX", "VTXBUF_UUY", "VTXBUF_UUZ",
               "VTXBUF_AX", "VTXBUF_AY", "VTXBUF_AZ", "VTXBUF_ENTROPY"]

STREAM_DEFAULT = 0
STREAM_ALL = 32


class IntParam(enum.IntEnum):
    AC_precision = 0
    AC_additive_timestep = 1
    AC_debug_plain_kernel = 2
    AC_upwind = 3
    AC_lforcing = 4
    AC_lbfield = 5


NUM_INT_PARAMS = 6


class Int3Param(enum.IntEnum):
    AC_ngrid = 0
    AC_nlocal = 1
    AC_nmin = 2
    AC_nlocal_max = 3
    AC_ngrid_max = 4
    AC_mlocal = 5
    AC_mgrid = 6
    AC_multigpu_offset = 7


NUM_INT3_PARAMS = 8


class RealParam(enum.IntEnum):
    AC_nu_visc = 0
    AC_eta = 1
    AC_cs_sound = 2
    AC_gamma = 3
    AC_cp_sound = 4
    AC_lnrho0 = 5
    AC_lnT0 = 6
    AC_mu0 = 7
    AC_zeta = 8
    AC_K_heatcond = 9
    AC_cdt = 10
    AC_cdtv = 11
    AC_chi = 12
    AC_current_time = 13
    AC_cs2_sound = 14
    AC_dsmin = 15
    AC_forcing_magnitude = 16
    AC_forcing_phase = 17
    AC_k_forcex = 18
    AC_k_forcey = 19
    AC_k_forcez = 20
    AC_ff_hel_rex = 21
    AC_ff_hel_rey = 22
    AC_ff_hel_rez = 23
    AC_ff_hel_imx = 24
    AC_ff_hel_imy = 25
    AC_ff_hel_imz = 26
    AC_kaver = 27
    AC_switch_forcing = 28
    AC_relhel = 29
    AC_kmin = 30
    AC_kmax = 31


NUM_REAL_PARAMS = 32


class Real3Param(enum.IntEnum):
    AC_ds = 0
    AC_inv_ds = 1
    AC_inv_ds_2 = 2
    AC_len = 3


NUM_REAL3_PARAMS = 4


class ReduceOp(enum.IntEnum):
    AC_REDUCE_OP_NO_REDUCE = 0
    AC_REDUCE_OP_MIN = 1
    AC_REDUCE_OP_MAX = 2
    AC_REDUCE_OP_SUM = 3


class MapKernel(enum.IntEnum):
    AC_NULL_KERNEL = 0
    AC_MAP_VTXBUF = 1
    AC_MAP_VTXBUF_SQUARE = 2
    AC_MAP_VTXBUF_EXP_SQUARE = 3
    AC_MAP_VTXBUF3_NORM = 4
    AC_MAP_VTXBUF3_SQUARE = 5
    AC_MAP_VTXBUF3_EXP_SQUARE = 6
    AC_MAP_VTXBUF4_ALFVEN_NORM = 7
    AC_MAP_VTXBUF4_ALFVEN_SQUARE = 8
    AC_KERNEL_SOLVE = 9
    AC_KERNEL_CALC_TIMESTEP = 10


class RealOutputParam(enum.IntEnum):
    UU_MAX_ADVEC = 0
    ALFVEN_SPEED_MAX = 1
    AC_dt_min = 2


NUM_REAL_OUTPUTS = 3


AC_SUCCESS, AC_FAILURE, AC_NOT_ALLOCATED = 0, 1, 2


class Volume(C.Structure):
    _fields_ = [("x", C.c_size_t), ("y", C.c_size_t), ("z", C.c_size_t)]


class Int3(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("z", C.c_int)]


class Real3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class AcMeshInfo(C.Structure):
    _fields_ = [
        ("int_params", C.c_int * NUM_INT_PARAMS),
        ("int3_params", Int3 * NUM_INT3_PARAMS),
        ("real_params", C.c_double * NUM_REAL_PARAMS),
        ("real3_params", Real3 * NUM_REAL3_PARAMS),
    ]


class AcMesh(C.Structure):
    _fields_ = [("vertex_buffer", C.POINTER(C.c_double) * NUM_FIELDS), ("info", AcMeshInfo)]


class AcReduction(C.Structure):
    _fields_ = [
        ("reduce_op", C.c_int),
        ("post_processing_op", C.c_int),
        ("map_vtxbuf_single", C.c_int),
        ("map_vtxbuf_vec", C.c_int),
        ("map_vtxbuf_vec_scal", C.c_int),
        ("name", C.c_char_p),
    ]


def _rt(op, post, single, vec, vecscal, name):
    return AcReduction(op, post, single, vec, vecscal, name.encode())


M = MapKernel
RTYPES = {
    "RTYPE_MAX": _rt(2, 0, M.AC_MAP_VTXBUF, M.AC_MAP_VTXBUF3_NORM, 0, "RTYPE_MAX"),
    "RTYPE_MIN": _rt(1, 0, M.AC_MAP_VTXBUF, M.AC_MAP_VTXBUF3_NORM, 0, "RTYPE_MIN"),
    "RTYPE_SUM": _rt(3, 0, M.AC_MAP_VTXBUF, M.AC_MAP_VTXBUF3_NORM, 0, "RTYPE_SUM"),
    "RTYPE_RMS": _rt(3, 1, M.AC_MAP_VTXBUF_SQUARE, M.AC_MAP_VTXBUF3_SQUARE, 0, "RTYPE_RMS"),
    "RTYPE_RMS_EXP": _rt(3, 1, M.AC_MAP_VTXBUF_EXP_SQUARE, M.AC_MAP_VTXBUF3_EXP_SQUARE, 0,
                         "RTYPE_RMS_EXP"),
    "RTYPE_ALFVEN_MAX": _rt(2, 0, 0, 0, M.AC_MAP_VTXBUF4_ALFVEN_NORM, "RTYPE_ALFVEN_MAX"),
    "RTYPE_ALFVEN_MIN": _rt(1, 0, 0, 0, M.AC_MAP_VTXBUF4_ALFVEN_NORM, "RTYPE_ALFVEN_MIN"),
    "RTYPE_ALFVEN_RMS": _rt(3, 1, 0, 0, M.AC_MAP_VTXBUF4_ALFVEN_SQUARE, "RTYPE_ALFVEN_RMS"),
}
# Index of each reduction type in the oracle's table (oracle/astaroth_oracle.c).
RTYPE_INDEX = {name: i for i, name in enumerate(RTYPES)}

Device_p = C.c_void_p
Ensemble_p = C.c_void_p


class AcEnsembleTiles(C.Structure):
    _fields_ = [("tx", C.c_int), ("ty", C.c_int), ("zb", C.c_int), ("blocks_per_sm", C.c_int),
                ("mode", C.c_int)]

# name -> (restype, argtypes)
SIGNATURES = {
    "acHostUpdateParams": (C.c_int, [C.POINTER(AcMeshInfo)]),
    "acHostMeshInfoDefault": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(AcMeshInfo)]),
    "acLoadConfig": (C.c_int, [C.c_char_p, C.POINTER(AcMeshInfo)]),
    "acHostMeshCreate": (C.c_int, [AcMeshInfo, C.POINTER(AcMesh)]),
    "acHostMeshDestroy": (C.c_int, [C.POINTER(AcMesh)]),
    "acHostMeshRandomizeSeeded": (C.c_int, [C.POINTER(AcMesh), C.c_ulonglong, C.c_double,
                                            C.c_double, C.c_double]),
    "acHostMeshSolenoidalModes": (C.c_int, [C.POINTER(AcMesh), C.c_ulonglong, C.c_int, C.c_int,
                                            C.c_double]),
    "acHostTimestepFromMaxima": (C.c_double, [AcMeshInfo, C.c_double, C.c_double]),
    "acDeviceCreate": (C.c_int, [C.c_int, AcMeshInfo, C.POINTER(Device_p)]),
    "acDeviceDestroy": (C.c_int, [C.POINTER(Device_p)]),
    "acDeviceResetMesh": (C.c_int, [Device_p, C.c_int]),
    "acDevicePrintInfo": (C.c_int, [Device_p]),
    "acDeviceSynchronizeStream": (C.c_int, [Device_p, C.c_int]),
    "acDeviceSwapBuffer": (C.c_int, [Device_p, C.c_int]),
    "acDeviceSwapBuffers": (C.c_int, [Device_p]),
    "acDeviceLoadScalarUniform": (C.c_int, [Device_p, C.c_int, C.c_int, C.c_double]),
    "acDeviceLoadVectorUniform": (C.c_int, [Device_p, C.c_int, C.c_int, Real3]),
    "acDeviceLoadIntUniform": (C.c_int, [Device_p, C.c_int, C.c_int, C.c_int]),
    "acDeviceStoreScalarUniform": (C.c_int, [Device_p, C.c_int, C.c_int,
                                             C.POINTER(C.c_double)]),
    "acDeviceLoadMeshInfo": (C.c_int, [Device_p, AcMeshInfo]),
    "acDeviceGetConfig": (AcMeshInfo, [Device_p]),
    "acDeviceLoadVertexBuffer": (C.c_int, [Device_p, C.c_int, AcMesh, C.c_int]),
    "acDeviceLoadMesh": (C.c_int, [Device_p, C.c_int, AcMesh]),
    "acDeviceSetVertexBuffer": (C.c_int, [Device_p, C.c_int, C.c_int, C.c_double]),
    "acDeviceFlushOutputBuffers": (C.c_int, [Device_p, C.c_int]),
    "acDeviceStoreVertexBuffer": (C.c_int, [Device_p, C.c_int, C.c_int, C.POINTER(AcMesh)]),
    "acDeviceStoreMesh": (C.c_int, [Device_p, C.c_int, C.POINTER(AcMesh)]),
    "acDeviceLoadVertexBufferWithOffset": (C.c_int, [Device_p, C.c_int, AcMesh, C.c_int, Int3,
                                                     Int3, C.c_int]),
    "acDeviceLoadMeshWithOffset": (C.c_int, [Device_p, C.c_int, AcMesh, Int3, Int3, C.c_int]),
    "acDeviceStoreVertexBufferWithOffset": (C.c_int, [Device_p, C.c_int, C.c_int, Int3, Int3,
                                                      C.c_int, C.POINTER(AcMesh)]),
    "acDeviceStoreMeshWithOffset": (C.c_int, [Device_p, C.c_int, Int3, Int3, C.c_int,
                                              C.POINTER(AcMesh)]),
    "acDeviceTransferVertexBufferWithOffset": (C.c_int, [Device_p, C.c_int, C.c_int, Int3, Int3,
                                                         C.c_int, Device_p]),
    "acDeviceTransferMeshWithOffset": (C.c_int, [Device_p, C.c_int, Int3, Int3, C.c_int,
                                                 Device_p]),
    "acDeviceTransferVertexBuffer": (C.c_int, [Device_p, C.c_int, C.c_int, Device_p]),
    "acDeviceTransferMesh": (C.c_int, [Device_p, C.c_int, Device_p]),
    "acDeviceStoreVectorUniform": (C.c_int, [Device_p, C.c_int, C.c_int, C.POINTER(Real3)]),
    "acDeviceStoreIntUniform": (C.c_int, [Device_p, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "acDeviceStoreInt3Uniform": (C.c_int, [Device_p, C.c_int, C.c_int, C.POINTER(Int3)]),
    "acDeviceLoadInt3Uniform": (C.c_int, [Device_p, C.c_int, C.c_int, Int3]),
    "acDeviceLoadMeshStaged": (C.c_int, [Device_p, C.c_int, AcMesh]),
    "acDeviceCommitStagedMesh": (C.c_int, [Device_p, C.c_int]),
    "acDeviceUpdate": (C.c_int, [Device_p, AcMeshInfo]),
    "acDeviceGetLocalConfig": (AcMeshInfo, [Device_p]),
    "acDeviceVolumeCopy": (C.c_int, [Device_p, C.c_int, C.c_void_p, Volume, Volume, C.c_void_p,
                                     Volume, Volume]),
    "acDeviceIntegrateSubstep": (C.c_int, [Device_p, C.c_int, C.c_int, Volume, Volume,
                                           C.c_double]),
    "acDevicePeriodicBoundcondStep": (C.c_int, [Device_p, C.c_int, C.c_int, Volume, Volume]),
    "acDevicePeriodicBoundconds": (C.c_int, [Device_p, C.c_int, Volume, Volume]),
    "acDeviceReduceScalNoPostProcessing": (C.c_int, [Device_p, C.c_int, AcReduction, C.c_int,
                                                     C.POINTER(C.c_double)]),
    "acDeviceReduceScal": (C.c_int, [Device_p, C.c_int, AcReduction, C.c_int,
                                     C.POINTER(C.c_double)]),
    "acDeviceReduceVecNoPostProcessing": (C.c_int, [Device_p, C.c_int, AcReduction, C.c_int,
                                                    C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "acDeviceReduceVec": (C.c_int, [Device_p, C.c_int, AcReduction, C.c_int, C.c_int, C.c_int,
                                    C.POINTER(C.c_double)]),
    "acDeviceReduceVecScalNoPostProcessing": (C.c_int, [Device_p, C.c_int, AcReduction,
                                                        C.c_int, C.c_int, C.c_int, C.c_int,
                                                        C.POINTER(C.c_double)]),
    "acDeviceReduceVecScal": (C.c_int, [Device_p, C.c_int, AcReduction, C.c_int, C.c_int,
                                        C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "acDeviceGetReduceNonFinite": (C.c_int, [Device_p, C.POINTER(C.c_int)]),
    "acDeviceGetVertexBufferPtrs": (C.c_int, [Device_p, C.c_int,
                                              C.POINTER(C.POINTER(C.c_double)),
                                              C.POINTER(C.POINTER(C.c_double))]),
    "acDeviceMemGetInfo": (C.c_int, [Device_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "acDeviceIntegrateStep": (C.c_int, [Device_p, C.c_int, C.c_double]),
    "acDeviceCalcTimestep": (C.c_int, [Device_p, C.c_int]),
    "acDeviceGetTimestepMaxima": (C.c_int, [Device_p, C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]),
    "acDeviceGetTimestep": (C.c_int, [Device_p, C.POINTER(C.c_double)]),
    "acDeviceFinishReduceReal": (C.c_int, [Device_p, C.c_int, C.POINTER(C.c_double), C.c_int,
                                           C.c_int, C.c_int]),
    "acDeviceFinishReduceRealStream": (C.c_int, [Device_p, C.c_void_p, C.POINTER(C.c_double),
                                                 C.c_int, C.c_int, C.c_int]),
    "acDeviceGetOutput": (C.c_double, [Device_p, C.c_int]),
    "acDeviceSetOutput": (C.c_int, [Device_p, C.c_int, C.c_double]),
    "acDeviceLoadMeshDevice": (C.c_int, [Device_p, C.c_int, C.POINTER(C.c_void_p)]),
    "acDeviceStoreMeshDevice": (C.c_int, [Device_p, C.c_int, C.POINTER(C.c_void_p)]),
    "acDeviceLoadAdjoint": (C.c_int, [Device_p, C.c_int, C.POINTER(C.c_void_p)]),
    "acDeviceIntegrateSubstepAdjoint": (C.c_int, [Device_p, C.c_int, C.c_int, Volume, Volume,
                                                  C.c_double]),
    "acDeviceStoreAdjoint": (C.c_int, [Device_p, C.c_int, C.POINTER(C.c_void_p)]),
    "acDeviceGetParamAdjoints": (C.c_int, [Device_p, C.POINTER(C.c_double),
                                           C.POINTER(C.c_double)]),
    "acHostForcingParams": (C.c_int, [Real3, C.c_double, C.c_double, C.POINTER(AcMeshInfo)]),
    "acHostGenerateForcingParams": (C.c_int, [C.c_ulonglong, C.c_ulonglong,
                                              C.POINTER(AcMeshInfo)]),
    "acHostMeshWriteToFile": (C.c_int, [AcMesh, C.c_size_t]),
    "acHostMeshReadFromFile": (C.c_int, [C.c_size_t, C.POINTER(AcMesh)]),
    "acDeviceStoreBfield": (C.c_int, [Device_p, C.c_int, C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "acDevicePlaneBytes": (C.c_size_t, [Device_p]),
    "acDevicePackPlanes": (C.c_int, [Device_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "acDeviceUnpackPlanes": (C.c_int, [Device_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "acDeviceBoxBytes": (C.c_size_t, [Device_p, Int3]),
    "acDevicePackBox": (C.c_int, [Device_p, C.c_int, Int3, Int3, C.c_void_p]),
    "acDeviceUnpackBox": (C.c_int, [Device_p, C.c_int, Int3, Int3, C.c_void_p]),
    "acDeviceWriteMeshToDisk": (C.c_int, [Device_p, C.c_char_p, C.c_char_p, C.c_int]),
    "acDeviceReadMeshFromDisk": (C.c_int, [Device_p, C.c_char_p, C.c_char_p, C.c_int]),
    "acDeviceAdjointTapeForward": (C.c_int, [Device_p, C.c_int, C.c_int, C.c_double]),
    "acDeviceAdjointTapeBackward": (C.c_int, [Device_p, C.c_int, C.c_int, C.c_double]),
    "acDeviceGetStreamHandle": (C.c_void_p, [Device_p, C.c_int]),
    "acDeviceGetLaunchCount": (C.c_ulonglong, [Device_p]),
    "acDeviceDebugSkipPlaneLoad": (C.c_int, [Device_p, C.c_int]),
    "acEnergyFunctional": (C.c_int, [AcMeshInfo, C.POINTER(C.c_void_p), C.c_void_p,
                                     C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p]),
    "acEnergyFunctionalScratchBytes": (C.c_size_t, [AcMeshInfo]),
    "acB200Version": (C.c_char_p, []),
    "acReduceNoAlloc": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.c_int,
                                  AcReduction, C.c_void_p, C.c_int, C.c_void_p]),
    "acEnsembleCreate": (C.c_int, [C.c_int, C.c_int, C.POINTER(AcMeshInfo),
                                   C.POINTER(Ensemble_p)]),
    "acEnsembleDestroy": (C.c_int, [C.POINTER(Ensemble_p)]),
    "acEnsembleLoadMember": (C.c_int, [Ensemble_p, C.c_int, AcMesh]),
    "acEnsembleStoreMember": (C.c_int, [Ensemble_p, C.c_int, C.POINTER(AcMesh)]),
    "acEnsembleSetTimesteps": (C.c_int, [Ensemble_p, C.POINTER(C.c_double)]),
    "acEnsembleIntegrateStep": (C.c_int, [Ensemble_p]),
    "acEnsembleIntegrateStepSequential": (C.c_int, [Ensemble_p]),
    "acEnsembleSetTiles": (C.c_int, [Ensemble_p, AcEnsembleTiles]),
    "acEnsembleGetTiles": (C.c_int, [Ensemble_p, C.POINTER(AcEnsembleTiles)]),
    "acEnsembleAutotune": (C.c_int, [Ensemble_p, C.POINTER(AcEnsembleTiles),
                                     C.POINTER(C.c_double)]),
    "acEnsembleReduceScal": (C.c_int, [Ensemble_p, C.c_int, AcReduction, C.c_int,
                                       C.POINTER(C.c_double)]),
    "acEnsembleReduceVec": (C.c_int, [Ensemble_p, C.c_int, AcReduction, C.c_int, C.c_int,
                                      C.c_int, C.POINTER(C.c_double)]),
    "acEnsembleSynchronize": (C.c_int, [Ensemble_p]),
    "acEnsembleGetStreamHandle": (C.c_void_p, [Ensemble_p]),
    "acEnsembleGetLaunchCount": (C.c_ulonglong, [Ensemble_p]),
    "acEnsembleCellCount": (C.c_longlong, [Ensemble_p]),
}

# acReduceNoAlloc accepts at most this many thread blocks (its static scratch).
AC_REDUCE_NOALLOC_MAX_BLOCKS = 2048

_lib = None


def load() -> C.CDLL:
    """Loads libastaroth_b200.so (built by astaroth_b200.build) and binds every symbol."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m astaroth_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
