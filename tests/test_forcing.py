"""Helical forcing (the reference's LFORCING option) on the CPU:

* acHostForcingParams builds the helical vectors as the reference's
  helical_forcing_special_vector (src/utils/astaroth_forcing.cc:158-216,
  compiled into oracle/_ref) does;
* the oracle restatement's forcing term equals the reference model built with
  LFORCING=1 bit for bit (at magnitude 1, where the host model and the device
  code of the reference agree);
* acHostGenerateForcingParams is reproducible and stays in the wave-number shell.
"""
import ctypes as C

import numpy as np
import pytest

from astaroth_b200 import capi
from astaroth_b200.capi import Real3, RealParam as RP
from astaroth_b200.device import CONFIG_PARAMS, info_to_dict, make_info, seeded_mesh
from oracle import oracle

needs_forcing_ref = pytest.mark.skipif(not oracle.available("reference_forcing"),
                                       reason="reference model with LFORCING=1 not built")


def forcing_dict(info):
    r = info.real_params
    return dict(forcing=1, forcing_magnitude=r[RP.AC_forcing_magnitude],
                forcing_phase=r[RP.AC_forcing_phase], kaver=r[RP.AC_kaver],
                k_force=[r[RP.AC_k_forcex], r[RP.AC_k_forcey], r[RP.AC_k_forcez]],
                ff_hel_re=[r[RP.AC_ff_hel_rex], r[RP.AC_ff_hel_rey], r[RP.AC_ff_hel_rez]],
                ff_hel_im=[r[RP.AC_ff_hel_imx], r[RP.AC_ff_hel_imy], r[RP.AC_ff_hel_imz]])


def forced_info(n, k, phi, phase, relhel=0.5, magnitude=1.0, **params):
    info = make_info(n, **dict(CONFIG_PARAMS, relhel=relhel, forcing_magnitude=magnitude,
                               kmin=0.8, kmax=2.2, **params))
    assert capi.load().acHostForcingParams(Real3(*k), phi, phase, C.byref(info)) == 0
    return info


def _e_vector(k, phi):
    """The helical basis vector of helical_forcing_e_generator (astaroth_forcing.cc:137-155)
    for a given angle phi."""
    k = np.asarray(k, dtype=float)
    e = np.array([0.0, 1.0, 0.0]) if k[1] == 0 and k[2] == 0 else np.array([1.0, 0.0, 0.0])
    kxe = np.cross(k, e)
    kxe /= np.sqrt(kxe @ kxe)
    kkxe = np.cross(k, kxe)
    kkxe /= np.sqrt(kkxe @ kkxe)
    return np.cos(phi) * kxe + np.sin(phi) * kkxe


@needs_forcing_ref
@pytest.mark.parametrize("k,phi,relhel", [((1, 0, 1), 0.7, 0.5), ((2, -1, 0), 2.1, 1.0),
                                          ((1, 0, 0), 4.0, 0.0)])
def test_helical_vectors_match_reference(k, phi, relhel):
    info = forced_info(16, k, phi, 0.3, relhel=relhel)
    f = forcing_dict(info)
    e = _e_vector(k, phi)
    R = oracle.lib("reference_forcing")
    R.ref_forcing_special_vector.restype = None
    re, im = (C.c_double * 3)(), (C.c_double * 3)()
    R.ref_forcing_special_vector((C.c_double * 3)(*k), (C.c_double * 3)(*e), C.c_double(relhel),
                                 re, im)
    np.testing.assert_allclose(f["ff_hel_re"], list(re), rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(f["ff_hel_im"], list(im), rtol=1e-13, atol=1e-15)
    assert f["k_force"] == list(map(float, k))
    assert f["kaver"] == pytest.approx((2.2 - 0.8) / 2)
    assert abs(np.dot(f["ff_hel_im"], k)) < 1e-12  # k x e is perpendicular to k


@needs_forcing_ref
@pytest.mark.parametrize("n", [16, (14, 10, 12)])
def test_port_forcing_matches_reference_bitexact(n):
    info = forced_info(n, (1, 1, 0), 1.3, 0.9)
    p = dict(info_to_dict(info), **forcing_dict(info))
    f = seeded_mesh(info, 61)
    a, b = f.copy(), f.copy()
    oracle.integrate(a, p, 1e-3, 2, "port")
    oracle.integrate(b, p, 1e-3, 2, "reference_forcing")
    assert np.array_equal(a, b)
    # within one step the force acts on u only (it is added after the update)
    one, off = f.copy(), f.copy()
    oracle.integrate(one, p, 1e-3, 1, "port")
    oracle.integrate(off, dict(p, forcing=0), 1e-3, 1, "port")
    assert not np.array_equal(one[1:4], off[1:4])
    assert np.array_equal(one[[0, 4, 5, 6, 7]], off[[0, 4, 5, 6, 7]])


def test_generated_params_are_reproducible_and_in_the_shell():
    lib = capi.load()
    seen = set()
    for step in range(6):
        a = make_info(16, kmin=0.8, kmax=2.2, relhel=0.3)
        b = make_info(16, kmin=0.8, kmax=2.2, relhel=0.3)
        assert lib.acHostGenerateForcingParams(7, step, C.byref(a)) == 0
        assert lib.acHostGenerateForcingParams(7, step, C.byref(b)) == 0
        fa, fb = forcing_dict(a), forcing_dict(b)
        assert fa == fb
        k = np.array(fa["k_force"])
        assert np.all(k == np.round(k)) and 0.8 ** 2 <= k @ k <= 2.2 ** 2
        assert 0 <= fa["forcing_phase"] < 2 * np.pi
        seen.add((tuple(k), fa["forcing_phase"]))
    assert len(seen) > 1
    # an empty shell is an error
    c = make_info(16, kmin=0.1, kmax=0.5)
    assert lib.acHostGenerateForcingParams(7, 0, C.byref(c)) != 0
