"""GPU parity tests: the CUDA path through the C ABI against the oracle.

Bars (from the reference's own test strategy, samples/devicetest/main.cc):
* periodic halo fill: bit-exact (pure copying), whole mesh and sub-boxes;
* FP64 integration: per-field relative L-inf <= 1e-12 after 1 step and
  <= 1e-10 after 100 steps against the long-double oracle;
* reductions: within a few ulps of the long-double oracle, measured as
  |gpu - oracle| <= 8 eps (|oracle| + sum |mapped values|).
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import astaroth_b200 as ab
from astaroth_b200 import capi
from oracle import oracle
from tests.conftest import gpu_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

GOLDEN = Path(__file__).resolve().parent / "golden"
META = json.loads((GOLDEN / "golden.json").read_text())
EPS = np.finfo(np.float64).eps
TOL_1STEP = 1e-12
TOL_100STEP = 1e-10


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def rel_linf_interior(cand, ref):
    num = np.abs(cand - ref).reshape(8, -1).max(axis=1)
    den = np.abs(ref).reshape(8, -1).max(axis=1)
    return num / np.where(den > 0, den, 1.0)


def case(name):
    c = META["cases"][name]
    n = c["n"] if isinstance(c["n"], int) else tuple(c["n"])
    info = ab.make_info(n, **ab.CONFIG_PARAMS)
    return info, ab.seeded_mesh(info, c["seed"])


def gpu_run(info, f0, dt, nsteps, graph=False, plain=False, kernel=None):
    """kernel: AC_debug_plain_kernel (0 default, 1 plain, 2 per-plane taps, 3 leading
    plane, 4 leading plane with the other group exchange)"""
    with ab.Device(info) as dev:
        if plain:
            dev.set_int(capi.IntParam.AC_debug_plain_kernel, 1)
        if kernel is not None:
            dev.set_int(capi.IntParam.AC_debug_plain_kernel, kernel)
        dev.load_mesh(f0)
        for _ in range(nsteps):
            if graph:
                dev.integrate_step(dt)
            else:
                dev.integrate_step_loop(dt)
        return dev.store_mesh()


# ---------------------------------------------------------------- boundconds

@pytest.mark.parametrize("name", sorted(META["cases"]))
def test_periodic_bitexact_golden(name):
    info, f = case(name)
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        dev.periodic_boundconds()
        out = dev.store_mesh()
    assert sha(out) == META["cases"][name]["periodic_sha256"]


# 16-byte-aligned rows, odd rows (alternating 8-byte alignment), small x extents
@pytest.mark.parametrize("n", [16, (20, 12, 8), 33, (37, 9, 11), (8, 8, 8), (6, 7, 5)])
def test_periodic_bitexact_oracle(n):
    info = ab.make_info(n, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 21)
    ref = f.copy()
    oracle.periodic_bounds(ref, "port")
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        dev.periodic_boundconds()
        assert np.array_equal(dev.store_mesh(), ref)


def test_periodic_sub_box_and_single_field():
    info = ab.make_info(16, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 22)
    full = f.copy()
    oracle.periodic_bounds(full, "port")
    lib = capi.load()
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        # a sub-box covering the lower z ghost slab only
        start, end = capi.Volume(0, 0, 0), capi.Volume(22, 22, 3)
        assert lib.acDevicePeriodicBoundconds(dev.handle, 0, start, end) == 0
        out = dev.store_mesh()
        want = f.copy()
        want[:, 0:3] = full[:, 0:3]
        assert np.array_equal(out, want)
        # one field over the whole mesh
        assert lib.acDevicePeriodicBoundcondStep(dev.handle, 0, 5, capi.Volume(0, 0, 0),
                                                 capi.Volume(22, 22, 22)) == 0
        out = dev.store_mesh()
        want[5] = full[5]
        assert np.array_equal(out, want)
        # invalid box is rejected
        assert lib.acDevicePeriodicBoundconds(dev.handle, 0, start,
                                              capi.Volume(23, 22, 22)) == capi.AC_FAILURE


# ---------------------------------------------------------------- integration

@pytest.mark.parametrize("name", sorted(META["cases"]))
def test_integration_vs_reference_golden(name):
    info, f = case(name)
    g = np.load(GOLDEN / f"golden_{name}.npz")
    one = gpu_run(info, f, META["dt"], 1)
    ten = gpu_run(info, f, META["dt"], 10)
    e1 = rel_linf_interior(oracle.interior(one), g["step1"])
    e10 = rel_linf_interior(oracle.interior(ten), g["step10"])
    assert e1.max() <= TOL_1STEP, e1
    assert e10.max() <= TOL_1STEP * 10, e10


def test_128_cubed_one_step():
    """128^3, seed 1, dt = 1e-3: one step against the oracle."""
    info = ab.make_info(128, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 1)
    ref = f.copy()
    oracle.integrate(ref, ab.info_to_dict(info), 1e-3, 1, "port")
    got = gpu_run(info, f, 1e-3, 1)
    err = oracle.rel_linf(got, ref)
    assert err.max() <= TOL_1STEP, err


def test_100_steps_32_cubed():
    info = ab.make_info(32, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 1)
    ref = f.copy()
    oracle.integrate(ref, ab.info_to_dict(info), 1e-3, 100, "port")
    got = gpu_run(info, f, 1e-3, 100, graph=True)
    err = oracle.rel_linf(got, ref)
    assert err.max() <= TOL_100STEP, err


@pytest.mark.slow
def test_128_cubed_100_steps():
    """128^3, seed 1, 100 steps against the oracle (minutes of CPU)."""
    info = ab.make_info(128, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 1)
    ref = f.copy()
    oracle.integrate(ref, ab.info_to_dict(info), 1e-3, 100, "port")
    got = gpu_run(info, f, 1e-3, 100, graph=True)
    err = oracle.rel_linf(got, ref)
    assert err.max() <= TOL_100STEP, err


def test_non_cubic_and_odd_sizes():
    for n, seed in (((40, 24, 16), 31), ((17, 19, 23), 32)):
        info = ab.make_info(n, **ab.CONFIG_PARAMS)
        f = ab.seeded_mesh(info, seed)
        ref = f.copy()
        oracle.integrate(ref, ab.info_to_dict(info), 1e-3, 2, "port")
        err = oracle.rel_linf(gpu_run(info, f, 1e-3, 2), ref)
        assert err.max() <= TOL_1STEP, (n, err)


def test_large_amplitude_other_params():
    params = dict(ab.CONFIG_PARAMS, gamma=1.4, cp_sound=2.5, nu_visc=1e-2, eta=3e-3, zeta=0.02,
                  K_heatcond=5e-3, lnrho0=0.2, lnT0=-0.3, mu0=0.9)
    info = ab.make_info(24, **params)
    f = ab.seeded_mesh(info, 5, amp_scalar=0.1, sigma_uu=0.05, sigma_aa=0.02)
    ref = f.copy()
    oracle.integrate(ref, ab.info_to_dict(info), 2e-3, 3, "port")
    err = oracle.rel_linf(gpu_run(info, f, 2e-3, 3), ref)
    assert err.max() <= TOL_1STEP * 10, err


@pytest.mark.parametrize("kernel", [0, 3])
def test_graph_step_equals_loop_bitwise(kernel):
    """The graph-captured step equals halo fill + substep + swap three times, with
    the default kernel choice and with the leading-plane kernel (3)."""
    info = ab.make_info((64, 40, 48), **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 4)
    a = gpu_run(info, f, 1e-3, 3, graph=False, kernel=kernel)
    b = gpu_run(info, f, 1e-3, 3, graph=True, kernel=kernel)
    assert np.array_equal(oracle.interior(a), oracle.interior(b))


@pytest.mark.parametrize("n", [(64, 40, 24), (66, 14, 37), (96, 8, 150)])
def test_plain_and_tiled_kernels_agree(n):
    """The plain kernel, the per-plane tap kernel and the default leading-plane
    kernel (tensor-memory delay line, separable xz/yz mixed derivatives): partial
    tiles in x and y, z extents that split into uneven chunks."""
    info = ab.make_info(n, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 6, amp_scalar=0.05, sigma_uu=0.05, sigma_aa=0.02)
    a = gpu_run(info, f, 1e-3, 2, kernel=1)
    b = gpu_run(info, f, 1e-3, 2, kernel=3)
    c = gpu_run(info, f, 1e-3, 2, kernel=2)
    for cand in (b, c):
        err = oracle.rel_linf(cand, a)
        assert err.max() <= 1e-13, err
    # the exchange between the warp groups through shared memory instead of
    # tensor memory moves the same values: the same bits
    d = gpu_run(info, f, 1e-3, 2, kernel=4)
    assert np.array_equal(oracle.interior(d), oracle.interior(b))


def test_leading_plane_kernel_vs_oracle_3_steps():
    """The default kernel against the CPU oracle on a mesh with several z
    chunks per column and partial x/y tiles."""
    n = (66, 14, 37)
    info = ab.make_info(n, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 8, amp_scalar=0.05, sigma_uu=0.05, sigma_aa=0.02)
    got = gpu_run(info, f, 1e-3, 3, kernel=3)
    ref = f.copy()
    oracle.integrate(ref, ab.info_to_dict(info), 1e-3, 3, "port")
    err = oracle.rel_linf(got, ref)
    assert err.max() <= 1e-12, err


# ---------------------------------------------------------------- reductions

def valid_reductions():
    for r in oracle.RTYPE_NAMES[:5]:
        yield r, [0]
        yield r, [1, 2, 3]
    for r in oracle.RTYPE_NAMES[5:]:
        yield r, [1, 2, 3, 0]


def gpu_reduce(dev, r, h):
    if len(h) == 1:
        return dev.reduce_scal(r, h[0])
    if len(h) == 3:
        return dev.reduce_vec(r, *h)
    return dev.reduce_vec_scal(r, *h)


def magnitude_sum(f, r, h):
    """sum of |mapped value| over the interior (scale of the rounding bound)."""
    q = oracle.interior(f)
    if len(h) == 1:
        a = q[h[0]]
        m = {"RTYPE_RMS": a * a, "RTYPE_RMS_EXP": np.exp(a) ** 2}.get(r, a)
    elif len(h) == 3:
        s = q[h[0]] ** 2 + q[h[1]] ** 2 + q[h[2]] ** 2
        m = {"RTYPE_RMS": s, "RTYPE_RMS_EXP": sum(np.exp(q[c]) ** 2 for c in h)}.get(r, np.sqrt(s))
    else:
        s = q[h[0]] ** 2 + q[h[1]] ** 2 + q[h[2]] ** 2
        m = s / np.exp(q[h[3]]) if r == "RTYPE_ALFVEN_RMS" else np.sqrt(s / np.exp(q[h[3]]))
    return float(np.abs(m).sum())


@pytest.mark.parametrize("n", [8, 64, (30, 20, 10)])
def test_reductions_vs_oracle(n):
    info = ab.make_info(n, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 8, amp_scalar=0.3, sigma_uu=0.2, sigma_aa=0.1)
    nn = np.prod(n) if not np.isscalar(n) else n ** 3
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        for r, h in valid_reductions():
            got = gpu_reduce(dev, r, h)
            want = oracle.reduce(f, r, h, "port")
            scale = magnitude_sum(f, r, h)
            if r.endswith("RMS") or r.endswith("RMS_EXP"):
                scale = np.sqrt(scale / nn)
            assert abs(got - want) <= 8 * EPS * (abs(want) + scale), (r, h, got, want)
            again = gpu_reduce(dev, r, h)
            assert again == got  # deterministic


@pytest.mark.parametrize("name", sorted(META["cases"]))
def test_reductions_vs_reference_golden(name):
    info, f = case(name)
    ref = META["cases"][name]["reductions_after_1_step"]
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        dev.integrate_step_loop(META["dt"])
        host = dev.store_mesh()
        for r, h in valid_reductions():
            want = ref[f"{r}:{','.join(map(str, h))}"]
            got = gpu_reduce(dev, r, h)
            scale = magnitude_sum(host, r, h)
            if r.endswith("RMS") or r.endswith("RMS_EXP"):
                scale = np.sqrt(scale / oracle.interior(host)[0].size)
            # GPU integration differs from the reference by ~1e-16 relative
            assert abs(got - want) <= 1e-12 * (abs(want) + scale), (r, h, got, want)


def test_reduction_rejects_wrong_map():
    info = ab.make_info(8)
    with ab.Device(info) as dev:
        with pytest.raises(ab.AstarothError):
            dev.reduce_scal("RTYPE_ALFVEN_MAX", 0)
        with pytest.raises(ab.AstarothError):
            dev.reduce_vec_scal("RTYPE_MAX", 1, 2, 3, 0)


# ---------------------------------------------------------------- API behaviour

def test_api_errors_and_state():
    info = ab.make_info(16, **ab.CONFIG_PARAMS)
    lib = capi.load()
    with ab.Device(info) as dev:
        # substeps accept boxes of whole interior x-y planes and steps 0..2
        bad = capi.Volume(4, 3, 3)
        assert lib.acDeviceIntegrateSubstep(dev.handle, 0, 0, bad, dev.vols.n1, 1e-3) == 1
        assert lib.acDeviceIntegrateSubstep(dev.handle, 0, 3, dev.vols.n0, dev.vols.n1, 1e-3) == 1
        assert lib.acDeviceIntegrateSubstep(dev.handle, 99, 0, dev.vols.n0, dev.vols.n1, 1e-3) == 1
        # created buffers are zero
        assert not dev.store_mesh().any()
        # host mesh of another size is rejected
        other = ab.make_info(12)
        assert lib.acDeviceLoadMesh(dev.handle, 0,
                                    ab.device.mesh_struct(ab.empty_mesh(other), other)) == 1
        # uniform loads change the physics of later launches
        dev.set_real(capi.RealParam.AC_nu_visc, 1e-2)
        cfg = lib.acDeviceGetConfig(dev.handle)
        assert cfg.real_params[capi.RealParam.AC_nu_visc] == 1e-2
        # swap of one field moves only that field
        f = ab.seeded_mesh(info, 1)
        dev.load_mesh(f)
        assert lib.acDeviceSwapBuffer(dev.handle, 3) == 0
        out = dev.store_mesh()
        assert np.array_equal(out[2], f[2]) and not out[3].any()
        dev.periodic_boundconds()
        dev.synchronize()
        assert dev.launch_count() > 0
        # a dead (NULL) host field: AC_NOT_ALLOCATED, the other fields still move
        # (the reference's acDeviceLoadMesh / acDeviceStoreMesh, device.cc:671-672)
        g = ab.seeded_mesh(info, 2)
        m = ab.device.mesh_struct(g, info)
        m.vertex_buffer[5] = None
        assert lib.acDeviceLoadMesh(dev.handle, 0, m) == capi.AC_NOT_ALLOCATED
        dev.synchronize()
        out = dev.store_mesh()
        assert np.array_equal(out[4], g[4]) and np.array_equal(out[6], g[6])
        assert not np.array_equal(out[5], g[5])
        back = np.zeros_like(g)
        mb = ab.device.mesh_struct(back, info)
        mb.vertex_buffer[2] = None
        assert lib.acDeviceStoreMesh(dev.handle, 0, capi.C.byref(mb)) == capi.AC_NOT_ALLOCATED
        dev.synchronize()
        assert np.array_equal(back[3], out[3]) and not back[2].any()
    assert lib.acDeviceSynchronizeStream(None, 0) == 1


def test_two_devices_on_one_gpu_are_independent():
    info = ab.make_info(16, **ab.CONFIG_PARAMS)
    f1 = ab.seeded_mesh(info, 1)
    f2 = ab.seeded_mesh(info, 2)
    with ab.Device(info) as d1, ab.Device(info) as d2:
        d1.load_mesh(f1)
        d2.load_mesh(f2)
        d1.integrate_step(1e-3)
        d2.integrate_step(1e-3)
        a, b = d1.store_mesh(), d2.store_mesh()
    assert np.array_equal(oracle.interior(a), oracle.interior(gpu_run(info, f1, 1e-3, 1)))
    assert np.array_equal(oracle.interior(b), oracle.interior(gpu_run(info, f2, 1e-3, 1)))


# ---------------------------------------------------------------- CFL timestep

def _d1(f, axis, ds):
    c = (3 / 4, -3 / 20, 1 / 60)
    return sum(ck * (np.roll(f, -k, axis) - np.roll(f, k, axis))
               for k, ck in zip((1, 2, 3), c)) / ds


def numpy_cfl(f, info):
    """max |u|, max |curl A|/sqrt(rho), max |u| + sqrt(cs^2 + vA^2) on the periodic interior."""
    p = ab.info_to_dict(info)
    q = oracle.interior(f)
    ds = p["ds"]
    grad = lambda g: [_d1(g, 2, ds[0]), _d1(g, 1, ds[1]), _d1(g, 0, ds[2])]  # noqa: E731
    ga = [grad(q[4 + c]) for c in range(3)]
    B = [ga[2][1] - ga[1][2], ga[0][2] - ga[2][0], ga[1][0] - ga[0][1]]
    b2 = B[0] ** 2 + B[1] ** 2 + B[2] ** 2
    va2 = b2 / np.exp(q[0])
    umag = np.sqrt(q[1] ** 2 + q[2] ** 2 + q[3] ** 2)
    return umag.max(), np.sqrt(va2).max(), (umag + np.sqrt(p["cs_sound"] ** 2 + va2)).max()


@pytest.mark.parametrize("precision,tol", [(0, 1e-13), (1, 1e-5)])
def test_cfl_maxima_and_timestep(precision, tol):
    info = ab.make_info((48, 32, 24), precision=precision, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 14, amp_scalar=0.05, sigma_uu=0.05, sigma_aa=0.02)
    oracle.periodic_bounds(f, "port")
    want_u, want_va, _ = numpy_cfl(f, info)
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        dev.calc_timestep()
        u, va = dev.timestep_maxima()
        assert abs(u - want_u) <= tol * want_u and abs(va - want_va) <= tol * want_va
        dt = dev.timestep()
        assert dt == ab.timestep_from_maxima(info, u, va)
        # substep 2 computes the same maxima from its input state on the fly
        dev.integrate_substep(2, 1e-3)
        u2, va2 = dev.timestep_maxima()
        assert abs(u2 - want_u) <= tol * want_u and abs(va2 - want_va) <= tol * want_va


def test_additive_timestep():
    info = ab.make_info(32, **ab.CONFIG_PARAMS)
    info.int_params[ab.capi.IntParam.AC_additive_timestep] = 1
    f = ab.seeded_mesh(info, 15, amp_scalar=0.05, sigma_uu=0.05, sigma_aa=0.02)
    oracle.periodic_bounds(f, "port")
    _, _, want_adv = numpy_cfl(f, info)
    p = ab.info_to_dict(info)
    ds = p["ds"][0]
    chi = info.real_params[ab.capi.RealParam.AC_chi]
    visc = max(p["nu_visc"], p["eta"], p["gamma"] * chi)
    want = min(0.3 * ds * ds / visc, 0.4 * ds / want_adv)
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        dev.calc_timestep()
        assert dev.timestep() == pytest.approx(want, rel=1e-13)


def test_adaptive_run_is_stable():
    """The adaptive-CFL run in miniature: solenoidal modes, FP32-comp, dt from the maxima."""
    info = ab.make_info(64, precision=1, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 3)
    ab.solenoidal_velocity(f, info, seed=3, nmodes=64, kmax=8, amplitude=1e-2)
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        dev.periodic_boundconds()
        dev.calc_timestep()
        dts = []
        for _ in range(5):
            dt = dev.timestep()
            dts.append(dt)
            dev.integrate_step(dt)
        out = dev.store_mesh()
    assert all(np.isfinite(dts)) and min(dts) > 0
    assert np.all(np.isfinite(oracle.interior(out)))
