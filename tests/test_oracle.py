"""CPU tests of the oracle: the C restatement against the reference's own host
model (compiled from its sources) and against the committed golden vectors."""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from astaroth_b200 import CONFIG_PARAMS, info_to_dict, make_info, seeded_mesh
from oracle import oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
META = json.loads((GOLDEN / "golden.json").read_text())

needs_ref = pytest.mark.skipif(not oracle.available("reference"),
                               reason="reference model not built (no reference sources)")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def valid_reductions():
    for r in oracle.RTYPE_NAMES[:5]:
        yield r, [0]
        yield r, [1, 2, 3]
    for r in oracle.RTYPE_NAMES[5:]:
        yield r, [1, 2, 3, 0]


def case_mesh(name):
    c = META["cases"][name]
    n = c["n"] if isinstance(c["n"], int) else tuple(c["n"])
    info = make_info(n, **CONFIG_PARAMS)
    return info, seeded_mesh(info, c["seed"])


@pytest.mark.parametrize("name", sorted(META["cases"]))
def test_generator_reproduces_golden_inputs(name):
    _, f = case_mesh(name)
    assert sha(f) == META["cases"][name]["input_sha256"]


@pytest.mark.parametrize("name", sorted(META["cases"]))
def test_port_periodic_matches_golden(name):
    _, f = case_mesh(name)
    oracle.periodic_bounds(f, "port")
    assert sha(f) == META["cases"][name]["periodic_sha256"]


@pytest.mark.parametrize("name", sorted(META["cases"]))
def test_port_integration_matches_golden_bitexact(name):
    info, f = case_mesh(name)
    g = np.load(GOLDEN / f"golden_{name}.npz")
    p = info_to_dict(info)
    a = f.copy()
    oracle.integrate(a, p, META["dt"], 1, "port")
    assert np.array_equal(oracle.interior(a), g["step1"])
    oracle.integrate(a, p, META["dt"], 9, "port")
    assert np.array_equal(oracle.interior(a), g["step10"])


@pytest.mark.parametrize("name", sorted(META["cases"]))
def test_port_reductions_match_golden(name):
    info, f = case_mesh(name)
    oracle.integrate(f, info_to_dict(info), META["dt"], 1, "port")
    ref = META["cases"][name]["reductions_after_1_step"]
    for r, h in valid_reductions():
        assert oracle.reduce(f, r, h, "port") == ref[f"{r}:{','.join(map(str, h))}"], (r, h)


@needs_ref
@pytest.mark.parametrize("n,seed", [(16, 11), ((14, 9, 7), 12), (20, 13)])
def test_port_matches_reference_bitexact(n, seed):
    info = make_info(n, **CONFIG_PARAMS)
    p = info_to_dict(info)
    f = seeded_mesh(info, seed)
    a, b = f.copy(), f.copy()
    oracle.integrate(a, p, 1e-3, 2, "port")
    oracle.integrate(b, p, 1e-3, 2, "reference")
    assert np.array_equal(a, b)
    for r, h in valid_reductions():
        assert oracle.reduce(a, r, h, "port") == oracle.reduce(b, r, h, "reference")
    c, d = f.copy(), f.copy()
    oracle.periodic_bounds(c, "port")
    oracle.periodic_bounds(d, "reference")
    assert np.array_equal(c, d)


@pytest.mark.skipif(not oracle.available("reference_upwd"),
                    reason="reference model with LUPWD=1 not built")
@pytest.mark.parametrize("n,seed,amp", [(16, 41, 1e-3), ((14, 9, 7), 42, 5e-2)])
def test_port_upwinding_matches_reference_bitexact(n, seed, amp):
    """The LUPWD terms (modelsolver.cc:424-506,776-779,837-841) in the
    restatement equal the reference model built with LUPWD=1, bit for bit,
    and change the result (they are not a no-op)."""
    info = make_info(n, **CONFIG_PARAMS)
    p = dict(info_to_dict(info), upwind=1)
    f = seeded_mesh(info, seed, amp_scalar=amp, sigma_uu=amp, sigma_aa=amp / 10)
    a, b, c = f.copy(), f.copy(), f.copy()
    oracle.integrate(a, p, 1e-3, 2, "port")
    oracle.integrate(b, p, 1e-3, 2, "reference_upwd")
    oracle.integrate(c, dict(p, upwind=0), 1e-3, 2, "port")
    assert np.array_equal(a, b)
    assert not np.array_equal(a, c)


@needs_ref
def test_port_matches_reference_other_params():
    """Non-default physics (larger amplitudes, other gamma/cp) stay bit-exact."""
    params = dict(CONFIG_PARAMS, gamma=1.4, cp_sound=2.5, nu_visc=1e-2, eta=3e-3, zeta=0.02,
                  K_heatcond=5e-3, lnrho0=0.2, lnT0=-0.3, mu0=0.9)
    info = make_info(12, **params)
    p = info_to_dict(info)
    f = seeded_mesh(info, 5, amp_scalar=0.1, sigma_uu=0.05, sigma_aa=0.02)
    a, b = f.copy(), f.copy()
    oracle.integrate(a, p, 2e-3, 3, "port")
    oracle.integrate(b, p, 2e-3, 3, "reference")
    assert np.array_equal(a, b)


@needs_ref
def test_reference_verify_accepts_itself_and_rejects_perturbation():
    info = make_info(8, **CONFIG_PARAMS)
    f = seeded_mesh(info, 3)
    oracle.periodic_bounds(f, "port")
    assert oracle.ref_verify(f, f.copy())
    g = f.copy()
    g[2, 5, 5, 5] *= 1.0 + 1e-9  # far beyond 5 ulps
    assert not oracle.ref_verify(f, g)


def _d1(f, axis, ds):
    c = (3 / 4, -3 / 20, 1 / 60)
    return sum(ck * (np.roll(f, -k, axis) - np.roll(f, k, axis))
               for k, ck in zip((1, 2, 3), c)) / ds


def _d2(f, axis, ds):
    d = (-49 / 18, 3 / 2, -3 / 20, 1 / 90)
    return (d[0] * f + sum(dk * (np.roll(f, -k, axis) + np.roll(f, k, axis))
                           for k, dk in zip((1, 2, 3), d[1:]))) / ds**2


def test_rates_match_numpy_stencils():
    """Continuity and induction rates of the oracle against an independent
    numpy evaluation of the 6th-order stencils on the periodic interior."""
    info = make_info(12, **CONFIG_PARAMS)
    p = info_to_dict(info)
    f = seeded_mesh(info, 9)
    oracle.periodic_bounds(f, "port")
    r = oracle.interior(oracle.rates(f, p))
    q = oracle.interior(f)  # periodic interior: np.roll gives the wrapped taps
    ds = p["ds"][0]
    lnrho, u, a = q[0], q[1:4], q[4:7]
    # axes of a field array are (z, y, x)
    grad = lambda g: [_d1(g, 2, ds), _d1(g, 1, ds), _d1(g, 0, ds)]  # noqa: E731
    lap = lambda g: _d2(g, 2, ds) + _d2(g, 1, ds) + _d2(g, 0, ds)  # noqa: E731
    gl = grad(lnrho)
    gu = [grad(u[c]) for c in range(3)]
    cont = -(u[0] * gl[0] + u[1] * gl[1] + u[2] * gl[2]) - (gu[0][0] + gu[1][1] + gu[2][2])
    ga = [grad(a[c]) for c in range(3)]
    B = [ga[2][1] - ga[1][2], ga[0][2] - ga[2][0], ga[1][0] - ga[0][1]]
    ind = [u[1] * B[2] - u[2] * B[1] + p["eta"] * lap(a[0]),
           u[2] * B[0] - u[0] * B[2] + p["eta"] * lap(a[1]),
           u[0] * B[1] - u[1] * B[0] + p["eta"] * lap(a[2])]
    for got, want in [(r[0], cont)] + [(r[4 + c], ind[c]) for c in range(3)]:
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


def test_torch_reference_matches_oracle():
    """The torch restatement used for CPU reference gradients agrees with the oracle."""
    import sys
    import torch
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    import mhd_torch_ref as R
    info = make_info((12, 10, 8), **CONFIG_PARAMS)
    p = info_to_dict(info)
    f = seeded_mesh(info, 5, amp_scalar=0.1, sigma_uu=0.05, sigma_aa=0.02)
    oracle.periodic_bounds(f, "port")
    r_or = oracle.interior(oracle.rates(f, p))
    r_t = R.rates(torch.from_numpy(oracle.interior(f).copy()), p).numpy()
    err = np.abs(r_t - r_or).reshape(8, -1).max(1) / np.abs(r_or).reshape(8, -1).max(1)
    assert err.max() <= 1e-14
    a = f.copy()
    oracle.integrate(a, p, 2e-3, 3, "port")
    x = torch.from_numpy(oracle.interior(f).copy())
    for _ in range(3):
        x = R.step(x, p, 2e-3)
    err = oracle.rel_linf(np.pad(x.numpy(), ((0, 0),) + ((3, 3),) * 3), a)
    assert err.max() <= 1e-14


def test_oracle_seeded_mesh_matches_golden_and_product():
    """The oracle-side generator (used where the product library must not be
    loaded) gives the golden inputs' bytes and the product generator's bytes."""
    for name, c in META["cases"].items():
        n = c["n"] if isinstance(c["n"], int) else tuple(c["n"])
        assert sha(oracle.seeded_mesh(n, c["seed"])) == c["input_sha256"], name
    info = make_info((9, 7, 5), **CONFIG_PARAMS)
    a = seeded_mesh(info, 11, amp_scalar=0.1, sigma_uu=0.05, sigma_aa=0.02)
    b = oracle.seeded_mesh((9, 7, 5), 11, amp_scalar=0.1, sigma_uu=0.05, sigma_aa=0.02)
    assert np.array_equal(a, b)
    p = oracle.box_params((9, 7, 5))
    q = info_to_dict(info)
    for k, v in q.items():
        assert np.allclose(p[k], v, rtol=0, atol=0), k

