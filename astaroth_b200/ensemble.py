"""Ensembles of independent meshes on one GPU (the acEnsemble* C ABI).

An ensemble advances members of different sizes and physics parameters
together: one persistent solve launch over a tile work-list of all members and
one halo-fill launch per substep, with the whole RK3 step captured as a CUDA
graph.  Each member's cells follow the arithmetic of a single-mesh Device
without tiling, so a member's result equals that Device's bit for bit.

The tile shape of the persistent launch comes from ``Ensemble.autotune``: the
library times a fixed candidate set on the current members, then compares a
whole substep of the best persistent launch with mode 1 (one shared-memory
tiled launch per member, the members' launches as concurrent graph branches)
and keeps the faster; the result can be cached in a JSON file keyed by the
member sizes, the precision and the GPU name.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from pathlib import Path

import numpy as np

from . import capi
from .capi import AcEnsembleTiles, AcMeshInfo
from .device import (AstarothError, _check, dims, empty_mesh, make_info, mesh_struct,
                     seeded_mesh)

# The ensemble workload: 64 members with N drawn from {32, 48, 64, 96} and
# nu, eta log-uniform on [1e-3, 1e-2]; member m is seeded with 100 + m.
ENSEMBLE_SIZES = (32, 48, 64, 96)


def ensemble_members(n_members: int = 64, seed: int = 3, precision: int = 1,
                     sizes=ENSEMBLE_SIZES):
    """Configs of a seeded ensemble: a list of (AcMeshInfo, mesh seed).

    Sizes, nu and eta of the members are drawn from numpy's PCG64 generator
    with ``seed``; every member is a periodic box [0, 2 pi)^3 with N^3 cells.
    """
    rng = np.random.default_rng(seed)
    ns = rng.choice(np.asarray(sizes), size=n_members)
    nus = 10.0 ** rng.uniform(-3.0, -2.0, size=n_members)
    etas = 10.0 ** rng.uniform(-3.0, -2.0, size=n_members)
    out = []
    for m in range(n_members):
        info = make_info(int(ns[m]), precision=precision, nu_visc=float(nus[m]),
                         eta=float(etas[m]))
        out.append((info, 100 + m))
    return out


def _default_cache() -> Path:
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return Path(base) / "astaroth_b200" / "ensemble_tiles.json"


class Ensemble:
    """n member meshes on one GPU; methods are the acEnsemble* calls."""

    def __init__(self, infos, device_id: int = 0):
        self.lib = capi.load()
        self.infos = list(infos)
        arr = (AcMeshInfo * len(self.infos))(*self.infos)
        self._h = capi.Ensemble_p()
        _check(self.lib.acEnsembleCreate(device_id, len(self.infos), arr, C.byref(self._h)),
               "acEnsembleCreate")
        self.n = len(self.infos)

    def destroy(self) -> None:
        if self._h:
            _check(self.lib.acEnsembleDestroy(C.byref(self._h)), "acEnsembleDestroy")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # ---- data ----
    def _member(self, m: int) -> int:
        if not 0 <= m < self.n:
            raise AstarothError(f"ensemble member {m} out of range [0, {self.n})")
        return m

    def load_member(self, m: int, fields: np.ndarray) -> None:
        self._member(m)
        _check(self.lib.acEnsembleLoadMember(self._h, m, mesh_struct(fields, self.infos[m])),
               "acEnsembleLoadMember")

    def store_member(self, m: int, out: np.ndarray | None = None) -> np.ndarray:
        self._member(m)
        out = empty_mesh(self.infos[m]) if out is None else out
        mesh = mesh_struct(out, self.infos[m])
        _check(self.lib.acEnsembleStoreMember(self._h, m, C.byref(mesh)), "acEnsembleStoreMember")
        return out

    def load_seeded(self, seeds) -> None:
        """Loads member m with the seeded initial condition of seeds[m]."""
        for m, s in enumerate(seeds):
            self.load_member(m, seeded_mesh(self.infos[m], s))

    def set_timesteps(self, dts) -> None:
        v = np.ascontiguousarray(np.broadcast_to(np.asarray(dts, dtype=np.float64), (self.n,)))
        _check(self.lib.acEnsembleSetTimesteps(self._h, v.ctypes.data_as(C.POINTER(C.c_double))),
               "acEnsembleSetTimesteps")

    # ---- stepping ----
    def integrate_step(self) -> None:
        _check(self.lib.acEnsembleIntegrateStep(self._h), "acEnsembleIntegrateStep")

    def integrate_step_sequential(self) -> None:
        _check(self.lib.acEnsembleIntegrateStepSequential(self._h),
               "acEnsembleIntegrateStepSequential")

    def synchronize(self) -> None:
        _check(self.lib.acEnsembleSynchronize(self._h), "acEnsembleSynchronize")

    # ---- tiles ----
    @property
    def tiles(self) -> tuple:
        t = AcEnsembleTiles()
        _check(self.lib.acEnsembleGetTiles(self._h, C.byref(t)), "acEnsembleGetTiles")
        return (t.tx, t.ty, t.zb, t.blocks_per_sm, t.mode)

    def set_tiles(self, tx: int, ty: int, zb: int, blocks_per_sm: int = 0, mode: int = 0) -> None:
        """mode 0: persistent work-list solve with these tiles; mode 1: concurrent
        per-member tiled launches (the tiles still describe mode 0's work list)."""
        _check(self.lib.acEnsembleSetTiles(self._h, AcEnsembleTiles(tx, ty, zb, blocks_per_sm,
                                                                    mode)),
               "acEnsembleSetTiles")

    def _cache_key(self) -> str:
        import torch  # only for the device name

        sizes = sorted(dims(i) for i in self.infos)
        prec = self.infos[0].int_params[capi.IntParam.AC_precision]
        return f"{torch.cuda.get_device_name()}|p{prec}|" + ",".join(
            f"{a}x{b}x{c}" for a, b, c in sizes)

    def autotune(self, cache: str | os.PathLike | None = None, use_cache: bool = True):
        """Tunes the tile shape (or takes it from the cache) and returns
        ((tx, ty, zb, blocks_per_sm), ms per solve launch or None if cached)."""
        path = Path(cache) if cache is not None else _default_cache()
        key = self._cache_key()
        table = {}
        if use_cache and path.exists():
            try:
                table = json.loads(path.read_text())
            except (OSError, ValueError):
                table = {}
            if key in table:
                self.set_tiles(*table[key])
                return tuple(table[key]), None
        best = AcEnsembleTiles()
        ms = C.c_double()
        _check(self.lib.acEnsembleAutotune(self._h, C.byref(best), C.byref(ms)),
               "acEnsembleAutotune")
        tiles = (best.tx, best.ty, best.zb, best.blocks_per_sm, best.mode)
        if use_cache:
            table[key] = list(tiles)
            try:
                path.parent.mkdir(parents=True, exist_ok=True)
                path.write_text(json.dumps(table, indent=1))
            except OSError:
                pass
        return tiles, ms.value

    # ---- analysis ----
    def reduce_scal(self, m: int, rtype: str, field: int) -> float:
        out = C.c_double()
        _check(self.lib.acEnsembleReduceScal(self._h, m, capi.RTYPES[rtype], int(field),
                                             C.byref(out)), "acEnsembleReduceScal")
        return out.value

    def reduce_vec(self, m: int, rtype: str, a: int, b: int, c: int) -> float:
        out = C.c_double()
        _check(self.lib.acEnsembleReduceVec(self._h, m, capi.RTYPES[rtype], int(a), int(b),
                                            int(c), C.byref(out)), "acEnsembleReduceVec")
        return out.value

    @property
    def cells(self) -> int:
        return int(self.lib.acEnsembleCellCount(self._h))

    def stream_handle(self) -> int:
        return self.lib.acEnsembleGetStreamHandle(self._h) or 0

    def launch_count(self) -> int:
        return int(self.lib.acEnsembleGetLaunchCount(self._h))


__all__ = ["Ensemble", "ensemble_members", "ENSEMBLE_SIZES", "AstarothError"]
