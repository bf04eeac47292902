"""Ensemble (acEnsemble*) parity on the GPU.

Every member of an ensemble must equal, bit for bit, a single-mesh Device of
the same config without tiling (AC_debug_plain_kernel = 1) after the same
steps: the persistent launch computes each cell with the plain kernel's
per-cell function.  The graph step, the sequential per-member launches and any
tile shape give the same bits.  FP64 members are also checked against the
oracle after one step.
"""
import numpy as np
import pytest

from astaroth_b200 import capi
from astaroth_b200.device import (AstarothError, Device, info_to_dict, make_info, mesh_struct,
                                  seeded_mesh)
from astaroth_b200.ensemble import Ensemble, ensemble_members
from oracle import oracle

pytestmark = pytest.mark.gpu

DT = 1e-3


def _members(precision, shapes, seed0=100):
    rng = np.random.default_rng(7)
    infos = []
    for n in shapes:
        nu, eta = 10.0 ** rng.uniform(-3, -2, size=2)
        infos.append(make_info(n, precision=precision, nu_visc=nu, eta=eta))
    return infos, [seed0 + m for m in range(len(infos))]


def _device_run(info, seed, steps, dt=DT):
    info.int_params[capi.IntParam.AC_debug_plain_kernel] = 1
    with Device(info) as d:
        f = seeded_mesh(info, seed)
        d.load_mesh(f)
        for _ in range(steps):
            d.integrate_step(dt)
        d.synchronize()
        out = d.store_mesh()
    info.int_params[capi.IntParam.AC_debug_plain_kernel] = 0
    return out


SHAPES = [32, 48, (40, 36, 44), 64, 33, 96]


@pytest.mark.parametrize("precision", [1, 0])
def test_members_equal_single_device(precision):
    infos, seeds = _members(precision, SHAPES)
    steps = 3
    with Ensemble(infos) as e:
        e.load_seeded(seeds)
        e.set_timesteps(DT)
        for _ in range(steps):
            e.integrate_step()
        e.synchronize()
        got = [e.store_member(m) for m in range(e.n)]
    for m, (info, seed) in enumerate(zip(infos, seeds)):
        ref = _device_run(info, seed, steps)
        assert np.array_equal(got[m], ref), f"member {m} differs from its single-mesh run"


def test_graph_sequential_and_tiles_agree():
    infos, seeds = _members(1, SHAPES)
    outs = []
    for mode in ("graph", "sequential", "tiles"):
        with Ensemble(infos) as e:
            e.load_seeded(seeds)
            e.set_timesteps(DT)
            if mode == "tiles":
                e.set_tiles(16, 8, 5, 1)
                assert e.tiles == (16, 8, 5, 1, 0)
            for _ in range(2):
                if mode == "sequential":
                    e.integrate_step_sequential()
                else:
                    e.integrate_step()
            e.synchronize()
            outs.append([e.store_member(m) for m in range(e.n)])
    for m in range(len(infos)):
        assert np.array_equal(outs[0][m], outs[1][m])
        assert np.array_equal(outs[0][m], outs[2][m])


def test_autotune_keeps_state_and_results(tmp_path):
    infos, seeds = _members(1, [32, 48, 64])
    with Ensemble(infos) as e:
        e.load_seeded(seeds)
        e.set_timesteps(DT)
        before = [e.store_member(m) for m in range(e.n)]
        tiles, ms = e.autotune(cache=tmp_path / "tiles.json")
        assert ms is not None and ms > 0
        tx, ty, zb, bps, mode = tiles
        assert mode in (0, 1)
        assert tx * ty % 32 == 0 and tx * ty <= 256 and zb >= 1
        for m in range(e.n):  # tuning leaves the in-buffers as they were
            assert np.array_equal(e.store_member(m), before[m])
        e.integrate_step()
        e.synchronize()
        got = [e.store_member(m) for m in range(e.n)]
        # a second ensemble takes the tiles from the cache
        with Ensemble(infos) as e2:
            t2, ms2 = e2.autotune(cache=tmp_path / "tiles.json")
            assert t2 == tiles and ms2 is None
    # mode 0 computes every cell with the plain kernel's arithmetic, mode 1 runs
    # the tiled kernel a Device of the member uses: each agrees with that
    # Device bit for bit
    ref = _device_run if mode == 0 else _device_tiled
    for m in range(len(infos)):
        assert np.array_equal(got[m], ref(infos[m], seeds[m], 1))


def _device_tiled(info, seed, steps):
    with Device(info) as d:
        d.load_mesh(seeded_mesh(info, seed))
        for _ in range(steps):
            d.integrate_step(DT)
        d.synchronize()
        return d.store_mesh()


@pytest.mark.parametrize("precision", [1, 0])
def test_mode1_members_equal_default_device(precision):
    """Mode 1 runs each member through the kernel its own Device uses (tiled,
    or plain where the mesh does not fit the tiled kernel, e.g. 32^3 in FP32
    and nx = 24): the same bits as that Device."""
    infos, seeds = _members(precision, [32, 48, (40, 36, 44), 64, 96, (24, 32, 16)])
    with Ensemble(infos) as e:
        e.load_seeded(seeds)
        e.set_timesteps(DT)
        e.set_tiles(32, 4, 8, 0, mode=1)
        for _ in range(3):
            e.integrate_step()
        e.synchronize()
        got = [e.store_member(m) for m in range(e.n)]
        # dt changes take effect in mode 1 too (its launches take dt as a parameter)
        e.set_timesteps(2 * DT)
        e.integrate_step()
        e.synchronize()
        twice = e.store_member(0)
    for m in range(len(infos)):
        assert np.array_equal(got[m], _device_tiled(infos[m], seeds[m], 3)), m
    with Device(infos[0]) as d:
        d.load_mesh(got[0])
        d.integrate_step(2 * DT)
        d.synchronize()
        assert np.array_equal(twice[:, 3:-3, 3:-3, 3:-3], d.store_mesh()[:, 3:-3, 3:-3, 3:-3])


def test_fp64_member_matches_oracle():
    infos, seeds = _members(0, [32, (24, 40, 32)])
    with Ensemble(infos) as e:
        e.load_seeded(seeds)
        e.set_timesteps(DT)
        e.integrate_step()
        e.synchronize()
        for m in range(e.n):
            ref = seeded_mesh(infos[m], seeds[m])
            oracle.integrate(ref, info_to_dict(infos[m]), DT, 1, "port")
            err = oracle.rel_linf(e.store_member(m), ref)
            assert err.max() <= 1e-12, err


def test_member_reductions_match_device():
    infos, seeds = _members(1, [32, 48])
    with Ensemble(infos) as e:
        e.load_seeded(seeds)
        for m in range(e.n):
            with Device(infos[m]) as d:
                d.load_mesh(seeded_mesh(infos[m], seeds[m]))
                for rt in ("RTYPE_MAX", "RTYPE_MIN", "RTYPE_RMS", "RTYPE_RMS_EXP"):
                    assert e.reduce_scal(m, rt, 0) == d.reduce_scal(rt, 0)
                assert e.reduce_vec(m, "RTYPE_RMS", 1, 2, 3) == d.reduce_vec("RTYPE_RMS", 1, 2, 3)


def test_errors():
    infos, seeds = _members(1, [32, 32])
    with Ensemble(infos) as e:
        with pytest.raises(AstarothError):
            e.store_member(5)
        out = capi.AcMesh()
        assert e.lib.acEnsembleStoreMember(e._h, 5, out) != capi.AC_SUCCESS
        assert e.lib.acEnsembleLoadMember(e._h, -1, out) != capi.AC_SUCCESS
        with pytest.raises(AstarothError):
            e.set_tiles(7, 3, 4)  # 21 threads: not a multiple of 32
        info48 = make_info(48, precision=1)  # a host mesh of the wrong size
        wrong = mesh_struct(seeded_mesh(info48, 1), info48)
        assert e.lib.acEnsembleLoadMember(e._h, 0, wrong) != capi.AC_SUCCESS
        with pytest.raises(AstarothError):
            e.reduce_scal(0, "RTYPE_ALFVEN_MAX", 0)
    with pytest.raises(AstarothError):
        Ensemble([make_info(32, precision=0), make_info(32, precision=1)])


def test_64_member_ensemble_graph_equals_sequential():
    """The 64-member FP32-compensated ensemble: graph == sequential launches
    after 2 steps; prints both rates."""
    import time

    members = ensemble_members(64)
    infos = [i for i, _ in members]
    seeds = [s for _, s in members]
    outs, rates = [], {}
    for mode in ("graph", "sequential"):
        with Ensemble(infos) as e:
            e.load_seeded(seeds)
            e.set_timesteps(DT)
            if mode == "graph":
                e.autotune(use_cache=False)
            for _ in range(2):
                e.integrate_step() if mode == "graph" else e.integrate_step_sequential()
            e.synchronize()
            outs.append([e.store_member(m) for m in (0, 17, 63)])
            t0 = time.perf_counter()
            for _ in range(5):
                e.integrate_step() if mode == "graph" else e.integrate_step_sequential()
            e.synchronize()
            rates[mode] = 5 * e.cells / (time.perf_counter() - t0)
    print(f"64-member ensemble: {rates['graph']:.3e} cell-updates/s (graph, persistent), "
          f"{rates['sequential']:.3e} (sequential plain launches)")
    for a, b in zip(*outs):
        assert np.array_equal(a, b)
