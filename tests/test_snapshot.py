"""Snapshot files (CPU): the host format of acHostMeshWriteToFile /
acHostMeshReadFromFile against the reference's own implementation
(src/utils/memory.cc:182-247, compiled into oracle/_ref), byte for byte and in
both directions, and the numpy reader/writer of astaroth_b200.snapshot."""
import ctypes as C
import os

import numpy as np
import pytest

from astaroth_b200 import capi
from astaroth_b200 import snapshot as snap
from astaroth_b200.device import dims, make_info, mesh_struct, seeded_mesh
from oracle import oracle

SHAPE = (10, 12, 9)


def _mesh():
    info = make_info(SHAPE)
    return info, seeded_mesh(info, 21)


def _files(d):
    return sorted(p for p in os.listdir(d))


@pytest.mark.skipif(not oracle.available("reference"), reason="reference model not built")
def test_host_format_is_byte_identical_to_reference(tmp_path, monkeypatch):
    info, f = _mesh()
    lib = capi.load()
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    monkeypatch.chdir(ours)
    assert lib.acHostMeshWriteToFile(mesh_struct(f, info), 7) == capi.AC_SUCCESS
    monkeypatch.chdir(ref)
    R = oracle.lib("reference")
    assert R.ref_write_to_file(oracle._ptrs(f), *SHAPE, C.c_ulong(7)) == 0
    assert _files(ours) == _files(ref)
    assert len(_files(ours)) == 9
    for name in _files(ours):
        assert (ours / name).read_bytes() == (ref / name).read_bytes(), name
    assert (ours / "data-format.csv").read_text() == "use_double, mx, my, mz\n1, 16, 18, 15\n"


@pytest.mark.skipif(not oracle.available("reference"), reason="reference model not built")
def test_host_format_reads_across_implementations(tmp_path, monkeypatch):
    info, f = _mesh()
    lib = capi.load()
    R = oracle.lib("reference")
    monkeypatch.chdir(tmp_path)
    # reference writes, this library reads
    assert R.ref_write_to_file(oracle._ptrs(f), *SHAPE, C.c_ulong(3)) == 0
    got = np.zeros_like(f)
    m = mesh_struct(got, info)
    assert lib.acHostMeshReadFromFile(3, C.byref(m)) == capi.AC_SUCCESS
    assert np.array_equal(got, f)
    # this library writes, the reference reads
    g = seeded_mesh(info, 22)
    assert lib.acHostMeshWriteToFile(mesh_struct(g, info), 4) == capi.AC_SUCCESS
    back = np.zeros_like(g)
    assert R.ref_read_from_file(oracle._ptrs(back), *SHAPE, C.c_ulong(4)) == 0
    assert np.array_equal(back, g)


def test_numpy_reader_and_writer_match_the_library(tmp_path, monkeypatch):
    info, f = _mesh()
    lib = capi.load()
    monkeypatch.chdir(tmp_path)
    assert lib.acHostMeshWriteToFile(mesh_struct(f, info), 12) == capi.AC_SUCCESS
    assert snap.read_data_format(".") == (1, 16, 18, 15)
    assert np.array_equal(snap.read_dat(12, "."), f)
    g = seeded_mesh(info, 23)
    snap.write_dat(g, 13, ".")
    back = np.zeros_like(g)
    assert lib.acHostMeshReadFromFile(13, C.byref(mesh_struct(back, info))) == capi.AC_SUCCESS
    assert np.array_equal(back, g)


def test_host_read_rejects_mismatches(tmp_path, monkeypatch):
    info, f = _mesh()
    lib = capi.load()
    monkeypatch.chdir(tmp_path)
    assert lib.acHostMeshWriteToFile(mesh_struct(f, info), 1) == capi.AC_SUCCESS
    other = make_info((10, 12, 10))  # header says mz = 15, this mesh has 16
    buf = np.zeros((8, 16, 18, 16))
    assert lib.acHostMeshReadFromFile(1, C.byref(mesh_struct(buf, other))) != capi.AC_SUCCESS
    back = np.zeros_like(f)
    assert lib.acHostMeshReadFromFile(2, C.byref(mesh_struct(back, info))) != capi.AC_SUCCESS
    # a short field file
    path = snap.dat_path(".", 5, 1)
    path.write_bytes(path.read_bytes()[:-8])
    assert lib.acHostMeshReadFromFile(1, C.byref(mesh_struct(back, info))) != capi.AC_SUCCESS
    # a buffer that is not allocated
    m = mesh_struct(back, info)
    m.vertex_buffer[3] = C.POINTER(C.c_double)()
    assert lib.acHostMeshWriteToFile(m, 9) == capi.AC_NOT_ALLOCATED


def test_grid_format_numpy_roundtrip_and_segments(tmp_path):
    info, f = _mesh()
    nx, ny, nz = dims(info)
    snap.write_mesh(f, tmp_path / "a", "step-7")
    got = snap.read_mesh(tmp_path / "a", "step-7", (nx, ny, nz))
    assert np.array_equal(got, f[:, 3:-3, 3:-3, 3:-3])
    # two z segments, as two ranks would write them
    seg = {}
    for oz, sz in ((0, 5), (5, nz - 5)):
        part = np.zeros((8, sz + 6, ny + 6, nx + 6))
        part[:, 3:-3, 3:-3, 3:-3] = f[:, 3 + oz:3 + oz + sz, 3:-3, 3:-3]
        snap.write_mesh(part, tmp_path / "b", "L", segment=(0, 0, oz))
        seg[(0, 0, oz)] = (nx, ny, sz)
    got = snap.read_mesh(tmp_path / "b", "L", (nx, ny, nz), segments=seg)
    assert np.array_equal(got, f[:, 3:-3, 3:-3, 3:-3])
    with pytest.raises(ValueError):
        snap.read_mesh(tmp_path / "b", "L", (nx, ny, nz), segments={(0, 0, 0): (nx, ny, 5)})
