"""astaroth_b200: B200-native single-GPU MHD integrator behind Astaroth's device C API.

The product is the shared library ``libastaroth_b200.so`` (CUDA for sm_100a,
C ABI in ``include/astaroth_b200.h``); this package loads it with ctypes and
offers the same calls to Python.
"""
from .capi import Field, RTYPES, load  # noqa: F401
from .device import (CONFIG_PARAMS, AstarothError, Device, empty_mesh, info_to_dict,  # noqa: F401
                     make_info, seeded_mesh, solenoidal_velocity, timestep_from_maxima)

__version__ = "0.1.0"
