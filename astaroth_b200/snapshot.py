"""Snapshot files in the reference's formats, for Python tools and restarts.

Two formats, both raw little-endian AcReal (float64) arrays, x fastest:

* Host format (src/utils/memory.cc:182-247, acHostMeshWriteToFile /
  acHostMeshReadFromFile): ``data-format.csv`` holding
  ``use_double, mx, my, mz`` and one line of values, and one file
  ``<VTXBUF name>-<id, 5 digits>.dat`` per field with every cell, halos
  included.
* Grid format (src/core/grid.cc:3792-3935, acGridWriteMeshToDiskLaunch, which
  the reference's reader analysis/python/astar/data/read.py:48-184 reads as
  its segmented case): one file per field with the interior nx*ny*nz values,
  ``<dir>/<VTXBUF name>-<label>.mesh``, or per segment
  ``<dir>/<VTXBUF name>-segment-<ox>-<oy>-<oz>-<label>.mesh``.  The device
  layer writes and reads these with acDeviceWriteMeshToDisk /
  acDeviceReadMeshFromDisk.

Arrays are numpy (8, z, y, x) float64, the layout of ``device.seeded_mesh``.
"""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np

from .capi import FIELD_NAMES, NGHOST, NUM_FIELDS

DATA_FORMAT = "data-format.csv"
_DTYPE = np.dtype("<f8")


def dat_path(directory, q: int, snapshot_id: int) -> Path:
    return Path(directory) / f"{FIELD_NAMES[q]}-{snapshot_id:05d}.dat"


def mesh_path(directory, q: int, label: str, segment=None) -> Path:
    if segment is None:
        return Path(directory) / f"{FIELD_NAMES[q]}-{label}.mesh"
    ox, oy, oz = segment
    return Path(directory) / f"{FIELD_NAMES[q]}-segment-{ox}-{oy}-{oz}-{label}.mesh"


def write_dat(fields: np.ndarray, snapshot_id: int, directory=".") -> None:
    """Writes a whole mesh (halos included) in the host format."""
    nf, mz, my, mx = fields.shape
    if nf != NUM_FIELDS:
        raise ValueError(f"expected {NUM_FIELDS} fields, got {nf}")
    d = Path(directory)
    (d / DATA_FORMAT).write_text(f"use_double, mx, my, mz\n1, {mx}, {my}, {mz}\n")
    for q in range(NUM_FIELDS):
        np.ascontiguousarray(fields[q], dtype=_DTYPE).tofile(dat_path(d, q, snapshot_id))


def read_data_format(directory=".") -> tuple[int, int, int, int]:
    """(use_double, mx, my, mz) of a host-format snapshot directory."""
    lines = (Path(directory) / DATA_FORMAT).read_text().splitlines()
    if len(lines) < 2:
        raise ValueError(f"{DATA_FORMAT}: expected a header and a line of values")
    vals = [int(v) for v in lines[1].split(",")]
    if len(vals) != 4:
        raise ValueError(f"{DATA_FORMAT}: expected 4 values, got {lines[1]!r}")
    return tuple(vals)


def read_dat(snapshot_id: int, directory=".") -> np.ndarray:
    """Reads a host-format snapshot into a (8, mz, my, mx) array."""
    use_double, mx, my, mz = read_data_format(directory)
    if use_double != 1:
        raise ValueError("only double-precision snapshots are supported")
    out = np.empty((NUM_FIELDS, mz, my, mx), dtype=np.float64)
    for q in range(NUM_FIELDS):
        a = np.fromfile(dat_path(directory, q, snapshot_id), dtype=_DTYPE)
        if a.size != mx * my * mz:
            raise ValueError(f"{dat_path(directory, q, snapshot_id)}: {a.size} values, "
                             f"expected {mx * my * mz}")
        out[q] = a.reshape(mz, my, mx)
    return out


def write_mesh(fields: np.ndarray, directory, label: str, segment=None) -> None:
    """Writes the interior of a (8, mz, my, mx) mesh (halos included) in the
    grid format; ``segment`` = (ox, oy, oz) selects the segmented names."""
    os.makedirs(directory, exist_ok=True)
    g = NGHOST
    for q in range(NUM_FIELDS):
        inner = np.ascontiguousarray(fields[q, g:-g, g:-g, g:-g], dtype=_DTYPE)
        inner.tofile(mesh_path(directory, q, label, segment))


def read_mesh(directory, label: str, n, segments=None) -> np.ndarray:
    """Reads a grid-format snapshot of interior size n = (nx, ny, nz).

    segments: None for one file per field; else a dict {(ox, oy, oz): (sx, sy, sz)}
    of segment offsets and sizes, assembled into the (8, nz, ny, nx) interior.
    """
    nx, ny, nz = n
    out = np.empty((NUM_FIELDS, nz, ny, nx), dtype=np.float64)
    for q in range(NUM_FIELDS):
        if segments is None:
            a = np.fromfile(mesh_path(directory, q, label), dtype=_DTYPE)
            if a.size != nx * ny * nz:
                raise ValueError(f"{mesh_path(directory, q, label)}: {a.size} values, "
                                 f"expected {nx * ny * nz}")
            out[q] = a.reshape(nz, ny, nx)
            continue
        covered = 0
        for (ox, oy, oz), (sx, sy, sz) in segments.items():
            a = np.fromfile(mesh_path(directory, q, label, (ox, oy, oz)), dtype=_DTYPE)
            if a.size != sx * sy * sz:
                raise ValueError(f"segment {(ox, oy, oz)}: {a.size} values, "
                                 f"expected {sx * sy * sz}")
            out[q, oz:oz + sz, oy:oy + sy, ox:ox + sx] = a.reshape(sz, sy, sx)
            covered += a.size
        if covered != nx * ny * nz:
            raise ValueError(f"segments cover {covered} of {nx * ny * nz} cells")
    return out


__all__ = ["DATA_FORMAT", "write_dat", "read_dat", "read_data_format", "write_mesh",
           "read_mesh", "dat_path", "mesh_path"]
