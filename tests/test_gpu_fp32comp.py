"""GPU tests of the FP32-compensated precision mode (AC_precision = 1).

Fields are stored as FP32 pairs (hi, lo) with |lo| <= ulp(hi)/2, the stencils
and RHS run in FP32 and the RK3 update is carried out on the pair with an
error-free two-sum.  Bars:
* periodic halo fill: bit-exact on the pairs;
* per-field relative L-inf against the FP64 path <= 1e-5 after 100 steps;
* reductions: FP64 accumulation of hi + lo, within FP64 rounding of the
  oracle evaluated on the same (joined) values.
"""
import numpy as np
import pytest

import astaroth_b200 as ab
from oracle import oracle
from tests.conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

EPS = np.finfo(np.float64).eps


def run(n, seed, steps, precision, dt=1e-3, graph=True, plain=False, kernel=None, **params):
    info = ab.make_info(n, precision=precision, **dict(ab.CONFIG_PARAMS, **params))
    f = ab.seeded_mesh(info, seed)
    with ab.Device(info) as dev:
        if plain:
            dev.set_int(ab.capi.IntParam.AC_debug_plain_kernel, 1)
        if kernel is not None:
            dev.set_int(ab.capi.IntParam.AC_debug_plain_kernel, kernel)
        dev.load_mesh(f)
        for _ in range(steps):
            dev.integrate_step(dt) if graph else dev.integrate_step_loop(dt)
        return dev.store_mesh()


def roundtrip(f):
    """What an FP32-compensated device holds for a double mesh: hi + lo."""
    hi = f.astype(np.float32)
    lo = (f - hi.astype(np.float64)).astype(np.float32)
    return hi.astype(np.float64) + lo.astype(np.float64)


def test_load_store_roundtrip_is_hi_plus_lo():
    info = ab.make_info(24, precision=1, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 3)
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        out = dev.store_mesh()
    assert np.array_equal(out, roundtrip(f))
    assert np.abs(out - f).max() <= 2.0 ** -48 * np.abs(f).max()


@pytest.mark.parametrize("n", [16, (40, 24, 12), (37, 9, 11), (9, 5, 6)])
def test_periodic_bitexact_on_pairs(n):
    info = ab.make_info(n, precision=1, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 4)
    ref = roundtrip(f)
    oracle.periodic_bounds(ref, "port")
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        dev.periodic_boundconds()
        assert np.array_equal(dev.store_mesh(), ref)


def test_fp32comp_vs_fp64_100_steps():
    """Accuracy bar at 128^3: per-field rel L-inf <= 1e-5 after 100 steps."""
    a = run(128, 2, 100, precision=0)
    b = run(128, 2, 100, precision=1)
    err = oracle.rel_linf(b, a)
    assert err.max() <= 1e-5, err


def test_fp32comp_vs_oracle_one_step():
    info = ab.make_info(32, precision=1, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 1)
    ref = roundtrip(f)
    oracle.integrate(ref, ab.info_to_dict(info), 1e-3, 1, "port")
    got = run(32, 1, 1, precision=1)
    err = oracle.rel_linf(got, ref)
    assert err.max() <= 1e-6, err


def test_compensated_error_well_inside_bar():
    """The compensated state keeps the 100-step error an order of magnitude
    inside the 1e-5 bar (plain FP32 storage would accumulate ~300 roundings
    of 2^-24 ~ 6e-8 relative each)."""
    a = run(48, 5, 100, precision=0)
    b = run(48, 5, 100, precision=1)
    err = oracle.rel_linf(b, a)
    assert err.max() <= 1e-6, err


@pytest.mark.parametrize("n", [(64, 40, 24), 32, (33, 20, 12)])
def test_plain_and_tiled_fp32comp_agree(n):
    """Including rows of mx = 38 and 39, whose 40-element pitch holds the tiled
    kernel's 40-wide plane box."""
    a = run(n, 6, 2, precision=1, plain=True)
    # the per-plane tap kernel evaluates every stencil in the plain kernel's order
    c = run(n, 6, 2, precision=1, kernel=2)
    err = oracle.rel_linf(a, c)
    assert err.max() <= 1e-8, err
    # the default kernel sums the mixed derivatives in another order: agreement
    # to FP32 rounding (2^-24 = 6e-8 relative per operation)
    b = run(n, 6, 2, precision=1, kernel=3)
    err = oracle.rel_linf(a, b)
    assert err.max() <= 1e-7, err
    # the exchange between the warp groups through shared memory instead of
    # tensor memory: the same bits
    d = run(n, 6, 2, precision=1, kernel=4)
    assert np.array_equal(d, b)


def test_graph_and_loop_agree_fp32comp():
    a = run(48, 7, 3, precision=1, graph=False)
    b = run(48, 7, 3, precision=1, graph=True)
    assert np.array_equal(oracle.interior(a), oracle.interior(b))


def test_reductions_fp32comp():
    info = ab.make_info(32, precision=1, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 8, amp_scalar=0.3, sigma_uu=0.2, sigma_aa=0.1)
    held = roundtrip(f)
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        for r in oracle.RTYPE_NAMES[:5]:
            got = dev.reduce_scal(r, 0)
            want = oracle.reduce(held, r, [0], "port")
            assert abs(got - want) <= 1e-13 * (abs(want) + 1.0), (r, got, want)
            got = dev.reduce_vec(r, 1, 2, 3)
            want = oracle.reduce(held, r, [1, 2, 3], "port")
            assert abs(got - want) <= 1e-13 * (abs(want) + 1.0), (r, got, want)
        for r in oracle.RTYPE_NAMES[5:]:
            got = dev.reduce_vec_scal(r, 1, 2, 3, 0)
            want = oracle.reduce(held, r, [1, 2, 3, 0], "port")
            assert abs(got - want) <= 1e-13 * (abs(want) + 1.0), (r, got, want)


def test_vertex_buffer_ptrs_rejected_for_fp32comp():
    info = ab.make_info(16, precision=1)
    with ab.Device(info) as dev:
        with pytest.raises(ab.AstarothError):
            dev.vertex_buffer_ptrs(0)
