"""CPU tests of the C ABI: the library loads and exports every declared symbol,
the Python mirror matches the header, and the host helpers behave."""
import ctypes as C
import math
import re
from pathlib import Path

import numpy as np
import pytest

import astaroth_b200 as ab
from astaroth_b200 import capi
from tests.conftest import gpu_available

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][A-Za-z0-9_ \t\*]*?\b(ac[A-Z][A-Za-z0-9_]*)\s*\(",
                             text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def header_enum_values():
    text = (ROOT / "include" / "astaroth_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    vals = {}
    for body in re.findall(r"typedef enum[^{]*\{(.*?)\}", text, flags=re.S):
        cur = -1
        for item in body.split(","):
            item = item.strip()
            if not item:
                continue
            if "=" in item:
                name, v = (s.strip() for s in item.split("="))
                cur = vals[v] if v in vals else int(v)
            else:
                name, cur = item, cur + 1
            vals[name] = cur
    return vals


def test_library_loads_and_exports_every_declared_symbol():
    lib = capi.load()
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(capi.SIGNATURES) <= set(names)


def test_python_enums_match_header():
    v = header_enum_values()
    for f in capi.Field:
        assert v["VTXBUF_" + f.name] == f.value
    for enum_cls, count in ((capi.IntParam, "NUM_INT_PARAMS"), (capi.Int3Param, "NUM_INT3_PARAMS"),
                            (capi.RealParam, "NUM_REAL_PARAMS"),
                            (capi.Real3Param, "NUM_REAL3_PARAMS")):
        for e in enum_cls:
            assert v[e.name] == e.value, e.name
        assert v[count] == len(enum_cls)
    for e in capi.MapKernel:
        assert v[e.name] == e.value
    for e in capi.ReduceOp:
        assert v[e.name] == e.value
    for e in capi.RealOutputParam:
        assert v[e.name] == e.value
    assert v["NUM_REAL_OUTPUTS"] == capi.NUM_REAL_OUTPUTS == len(capi.RealOutputParam)
    assert v["STREAM_ALL"] == capi.STREAM_ALL


def test_struct_sizes_match_the_c_compiler(tmp_path):
    """sizeof and member offsets of the ctypes mirrors equal those of the header
    compiled by the C compiler."""
    import subprocess

    src = tmp_path / "sizes.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "astaroth_b200.h"\n'
                   "int main(void) { printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(AcMeshInfo), "
                   "offsetof(AcMeshInfo, int3_params), offsetof(AcMeshInfo, real_params), "
                   "offsetof(AcMeshInfo, real3_params), sizeof(AcReduction), sizeof(AcMesh)); "
                   "return 0; }\n")
    exe = tmp_path / "sizes"
    inc = Path(__file__).resolve().parents[1] / "include"
    subprocess.run(["gcc", "-std=c11", f"-I{inc}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    M = capi.AcMeshInfo
    assert got == [C.sizeof(M), M.int3_params.offset, M.real_params.offset,
                   M.real3_params.offset, C.sizeof(capi.AcReduction), C.sizeof(capi.AcMesh)]


def test_make_info_derived_params():
    info = ab.make_info(64, nu_visc=5e-3)
    i3 = {p.name: (info.int3_params[p].x, info.int3_params[p].y, info.int3_params[p].z)
          for p in capi.Int3Param}
    assert i3["AC_nmin"] == (3, 3, 3)
    assert i3["AC_mlocal"] == (70, 70, 70)
    assert i3["AC_nlocal_max"] == (67, 67, 67)
    ds = info.real3_params[capi.Real3Param.AC_ds]
    inv = info.real3_params[capi.Real3Param.AC_inv_ds]
    assert ds.x == pytest.approx(2 * math.pi / 64)
    assert inv.x == 1.0 / ds.x
    assert info.real_params[capi.RealParam.AC_nu_visc] == 5e-3
    assert info.real_params[capi.RealParam.AC_dsmin] == ds.x


def test_load_config(tmp_path):
    conf = tmp_path / "astaroth.conf"
    conf.write_text("""
/* block
   comment */
AC_ngrid  = {32,16,8}
AC_ds = {0.1,0.2,0.3}   // trailing comment
AC_nu_visc  = 2e-5
AC_gamma = 0.5
AC_additive_timestep = T
AC_unknown_key = 7
""")
    info = capi.AcMeshInfo()
    assert capi.load().acLoadConfig(str(conf).encode(), C.byref(info)) == capi.AC_SUCCESS
    n = info.int3_params[capi.Int3Param.AC_ngrid]
    assert (n.x, n.y, n.z) == (32, 16, 8)
    assert info.real3_params[capi.Real3Param.AC_ds].z == 0.3
    assert info.real_params[capi.RealParam.AC_nu_visc] == 2e-5
    assert info.real_params[capi.RealParam.AC_gamma] == 0.5
    assert info.int_params[capi.IntParam.AC_additive_timestep] == 1
    m = info.int3_params[capi.Int3Param.AC_mlocal]
    assert (m.x, m.y, m.z) == (38, 22, 14)


def test_load_config_missing_file_fails():
    info = capi.AcMeshInfo()
    assert capi.load().acLoadConfig(b"/nonexistent/x.conf", C.byref(info)) == capi.AC_FAILURE


def test_seeded_mesh_deterministic_and_distributed():
    info = ab.make_info(24)
    a = ab.seeded_mesh(info, 42)
    b = ab.seeded_mesh(info, 42)
    c = ab.seeded_mesh(info, 43)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.abs(a[0]).max() <= 1e-5 and np.abs(a[7]).max() <= 1e-5
    assert a[0].std() == pytest.approx(1e-5 / math.sqrt(3), rel=0.05)
    for q in (1, 2, 3):
        assert a[q].std() == pytest.approx(1e-3, rel=0.05)
        assert abs(a[q].mean()) < 1e-4
    for q in (4, 5, 6):
        assert a[q].std() == pytest.approx(1e-4, rel=0.05)
    # fields are mutually independent streams
    assert abs(np.corrcoef(a[1].ravel(), a[2].ravel())[0, 1]) < 0.05


def test_solenoidal_modes_divergence_free():
    info = ab.make_info(32)
    f = ab.empty_mesh(info)
    ab.solenoidal_velocity(f, info, seed=3, nmodes=16, kmax=4, amplitude=1e-2)
    u = f[1:4, 3:-3, 3:-3, 3:-3]
    k = np.fft.fftfreq(32, d=1.0 / 32)
    kz, ky, kx = np.meshgrid(k, k, k, indexing="ij")
    div = kx * np.fft.fftn(u[0]) + ky * np.fft.fftn(u[1]) + kz * np.fft.fftn(u[2])
    assert np.abs(div).max() < 1e-9 * np.abs(np.fft.fftn(u[0])).max()
    assert 1e-3 < np.sqrt((u ** 2).sum(axis=0)).max() < 5e-2
    # halos are the periodic images
    assert np.allclose(f[1, 0:3, 3:-3, 3:-3], f[1, -6:-3, 3:-3, 3:-3], atol=1e-15)


def test_timestep_formula():
    info = ab.make_info(64, nu_visc=5e-3, eta=2e-3, cs_sound=1.0)
    dt = ab.timestep_from_maxima(info, 0.1, 0.05)
    ds = 2 * math.pi / 64
    adv = 0.4 * ds / (0.1 + math.sqrt(1.0 + 0.05 ** 2))
    vis = 0.3 * ds * ds / 5e-3
    assert dt == pytest.approx(min(adv, vis), rel=1e-14)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_device_create_fails_cleanly_without_gpu():
    info = ab.make_info(16)
    h = capi.Device_p()
    assert capi.load().acDeviceCreate(0, info, C.byref(h)) == capi.AC_FAILURE
    assert not h
    with pytest.raises(ab.AstarothError):
        ab.Device(info)


def test_ensemble_members_seeded():
    from astaroth_b200.ensemble import ENSEMBLE_SIZES, ensemble_members

    a = ensemble_members(64)
    b = ensemble_members(64)
    assert [capi_dims(i) for i, _ in a] == [capi_dims(i) for i, _ in b]
    assert [s for _, s in a] == list(range(100, 164))
    sizes = {capi_dims(i)[0] for i, _ in a}
    assert sizes <= set(ENSEMBLE_SIZES) and len(sizes) == len(ENSEMBLE_SIZES)
    for info, _ in a:
        nu = info.real_params[capi.RealParam.AC_nu_visc]
        eta = info.real_params[capi.RealParam.AC_eta]
        assert 1e-3 <= nu <= 1e-2 and 1e-3 <= eta <= 1e-2
        assert info.int_params[capi.IntParam.AC_precision] == 1


def capi_dims(info):
    from astaroth_b200.device import dims

    return dims(info)


def test_seeded_generator_one_field_at_a_time():
    """Each field's values do not depend on the other buffers: generating one
    field with the others NULL gives the field of the full generation."""
    from astaroth_b200.device import empty_mesh, make_info, mesh_struct, seeded_mesh

    info = make_info((10, 12, 9))
    full = seeded_mesh(info, 5)
    lib = capi.load()
    for q in (0, 3, 7):
        part = empty_mesh(info)
        m = capi.AcMesh()
        m.info = info
        m.vertex_buffer[q] = part[q].ctypes.data_as(C.POINTER(C.c_double))
        assert lib.acHostMeshRandomizeSeeded(C.byref(m), 5, 1e-5, 1e-3, 1e-4) == 0
        assert np.array_equal(part[q], full[q])
    # the solenoidal generator needs all three velocity buffers
    m = mesh_struct(empty_mesh(info), info)
    m.vertex_buffer[2] = C.POINTER(C.c_double)()
    assert lib.acHostMeshSolenoidalModes(C.byref(m), 3, 8, 4, 1e-2) != 0
