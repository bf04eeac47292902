"""acReduceNoAlloc: the reduction entry point that allocates no device memory.

It serves callers that cannot allocate: applications whose GPU memory is owned
by their own pool or arena (a cudaMalloc outside it can fail, and cudaFree
synchronizes the device) and coupled codes held to a fixed memory budget.  It
reduces fields the caller owns and writes the result to a device pointer the
caller owns, using a static scratch array inside the library.

This file is collected last on purpose: a failure here leaves every other test
already run.  The test works both alone in a fresh process (the first call
then sets up the scratch address on the device) and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import astaroth_b200 as ab
from astaroth_b200 import capi
from tests.conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

EPS = np.finfo(np.float64).eps
CASES = [("RTYPE_MAX", [0]), ("RTYPE_SUM", [0]), ("RTYPE_RMS", [1, 2, 3]),
         ("RTYPE_MIN", [1, 2, 3]), ("RTYPE_SUM", [4, 5, 6]), ("RTYPE_RMS_EXP", [0]),
         ("RTYPE_ALFVEN_MAX", [1, 2, 3, 0]), ("RTYPE_ALFVEN_RMS", [1, 2, 3, 0])]


def existing(dev, r, h):
    """The same reduction through the existing acDeviceReduce*NoPostProcessing."""
    if len(h) == 1:
        return dev.reduce_scal(r, h[0], post=False)
    if len(h) == 3:
        return dev.reduce_vec(r, *h, post=False)
    return dev.reduce_vec_scal(r, *h, post=False)


def test_no_alloc_matches_existing_entry_point_twice():
    import torch

    n = (40, 24, 16)
    info = ab.make_info(n, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 12, amp_scalar=0.2, sigma_uu=0.1, sigma_aa=0.05)
    lib = capi.load()
    # caller-owned device memory: the fields and the result (allocated here by
    # the caller, not by the entry point)
    fields_dev = torch.from_numpy(f).cuda()
    result = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        for r, h in CASES:
            want = existing(dev, r, h)
            ptrs = (C.c_void_p * len(h))(*[fields_dev[q].data_ptr() for q in h])
            for call in range(2):  # two calls in a row share the static scratch
                result.fill_(np.nan)
                rc = lib.acReduceNoAlloc(ptrs, len(h), n[0], n[1], n[2], capi.RTYPES[r],
                                         C.c_void_p(result.data_ptr()), 0,
                                         C.c_void_p(stream.cuda_stream))
                assert rc == capi.AC_SUCCESS, (r, h, call)
                torch.cuda.synchronize()
                got = float(result.item())
                assert abs(got - want) <= 8 * EPS * abs(want), (r, h, call, got, want)
        # caller-chosen grids: one block, an odd count, and the largest the
        # static scratch holds (more blocks than the 24 * 16 rows: the extra
        # blocks contribute only the identity of the reduction)
        for r, h in (("RTYPE_SUM", [0]), ("RTYPE_MAX", [1, 2, 3])):
            want = existing(dev, r, h)
            ptrs = (C.c_void_p * len(h))(*[fields_dev[q].data_ptr() for q in h])
            for blocks in (1, 7, capi.AC_REDUCE_NOALLOC_MAX_BLOCKS):
                for call in range(2):
                    result.fill_(np.nan)
                    rc = lib.acReduceNoAlloc(ptrs, len(h), n[0], n[1], n[2], capi.RTYPES[r],
                                             C.c_void_p(result.data_ptr()), blocks,
                                             C.c_void_p(stream.cuda_stream))
                    assert rc == capi.AC_SUCCESS, (r, h, blocks, call)
                    torch.cuda.synchronize()
                    got = float(result.item())
                    assert abs(got - want) <= 8 * EPS * abs(want), (r, h, blocks, got, want)


def test_no_alloc_rejects_too_many_blocks():
    import torch

    info = ab.make_info(16)
    f = ab.seeded_mesh(info, 1)
    lib = capi.load()
    fields_dev = torch.from_numpy(f).cuda()
    result = torch.zeros(1, dtype=torch.float64, device="cuda")
    ptrs = (C.c_void_p * 1)(fields_dev[0].data_ptr())
    rc = lib.acReduceNoAlloc(ptrs, 1, 16, 16, 16, capi.RTYPES["RTYPE_SUM"],
                             C.c_void_p(result.data_ptr()), capi.AC_REDUCE_NOALLOC_MAX_BLOCKS + 1,
                             None)
    assert rc == capi.AC_FAILURE
    # a negative grid size is a caller error, not a request for the default
    rc = lib.acReduceNoAlloc(ptrs, 1, 16, 16, 16, capi.RTYPES["RTYPE_SUM"],
                             C.c_void_p(result.data_ptr()), -1, None)
    assert rc == capi.AC_FAILURE
    # extents whose padded size would overflow an int are refused
    rc = lib.acReduceNoAlloc(ptrs, 1, 2147483647, 16, 16, capi.RTYPES["RTYPE_SUM"],
                             C.c_void_p(result.data_ptr()), 0, None)
    assert rc == capi.AC_FAILURE
    # a wrong field count for the reduction type is rejected too
    rc = lib.acReduceNoAlloc(ptrs, 1, 16, 16, 16, capi.RTYPES["RTYPE_ALFVEN_MAX"],
                             C.c_void_p(result.data_ptr()), 0, None)
    assert rc == capi.AC_FAILURE
