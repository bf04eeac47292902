"""Parity at the benchmark's full size (512^3): one step against statistics of
the reference's own host model committed as a fixture, and size-independent
properties where the CPU oracle is too slow; and a 256^3 step against the
oracle.

* One FP64 RK3 step of the seeded benchmark mesh against golden_512.json
  (tests/golden/make_golden_512.py, from the reference's host model): 1024
  sampled cells within 1e-12 of each field's largest value, and the field
  minima, maxima, sums and sums of squares.

* Translation invariance: the update of every cell is the same arithmetic on
  the same values wherever the cell sits in the tiles, so integrating a
  periodically shifted mesh gives exactly the shifted result.  A mistake in
  tile edges, halo planes, z chunks or the exchange of the two warp groups
  breaks the equality.
* FP32-compensated against FP64 at 512^3 after 5 steps within the 1e-5 bar.
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import astaroth_b200 as ab
from astaroth_b200.device import info_to_dict
from oracle import oracle

pytestmark = pytest.mark.gpu

DT = 1e-3


def _torch():
    import torch

    return torch


def _random_mesh(torch, n, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    f = torch.empty((8, n + 6, n + 6, n + 6), dtype=torch.float64, device="cuda")
    f[0].uniform_(-1e-5, 1e-5, generator=g)
    f[7].uniform_(-1e-5, 1e-5, generator=g)
    f[1:4].normal_(0.0, 1e-3, generator=g)
    f[4:7].normal_(0.0, 1e-4, generator=g)
    return f


def _steps(dev, torch, f, steps):
    dev.load_mesh_device(f)
    for _ in range(steps):
        dev.integrate_step(DT)
    return dev.store_mesh_device(torch.empty_like(f))


GOLDEN_512 = Path(__file__).resolve().parent / "golden" / "golden_512.json"


def test_512_one_step_vs_reference_golden():
    """One FP64 RK3 step at 512^3 (default kernel choice) against the reference's
    host model: the statistics and sampled cells of tests/golden/golden_512.json."""
    from tests.golden.make_golden_512 import stats

    meta = json.loads(GOLDEN_512.read_text())
    n = meta["n"]
    info = ab.make_info(n, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, meta["seed"])
    assert hashlib.sha256(f.tobytes()).hexdigest() == meta["input_sha256"]
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        dev.integrate_step(meta["dt"])
        dev.synchronize()
        got = dev.store_mesh(f)
    s = stats(got, n)
    for q in range(8):
        scale = max(abs(meta["min"][q]), abs(meta["max"][q]))
        err = np.abs(np.array(s["samples"][q]) - np.array(meta["samples"][q])).max() / scale
        assert err <= 1e-12, (q, err)
        assert abs(s["min"][q] - meta["min"][q]) <= 1e-12 * scale, q
        assert abs(s["max"][q] - meta["max"][q]) <= 1e-12 * scale, q
        assert abs(s["sum_sq"][q] - meta["sum_sq"][q]) <= 2e-12 * meta["sum_sq"][q], q
        assert abs(s["sum"][q] - meta["sum"][q]) <= 1e-12 * meta["sum_abs"][q], q


@pytest.mark.parametrize("shift", [(5, 37, 100), (1, 1, 1), (64, 4, 0)])
def test_512_translation_invariance(shift):
    torch = _torch()
    n = 512
    info = ab.make_info(n, **ab.CONFIG_PARAMS)
    f = _random_mesh(torch, n, 11)
    dz, dy, dx = shift
    g = torch.zeros_like(f)
    g[:, 3:-3, 3:-3, 3:-3] = torch.roll(f[:, 3:-3, 3:-3, 3:-3], shifts=shift, dims=(1, 2, 3))
    with ab.Device(info) as dev:
        a = _steps(dev, torch, f, 1)
        del f
        b = _steps(dev, torch, g, 1)
    want = torch.roll(a[:, 3:-3, 3:-3, 3:-3], shifts=shift, dims=(1, 2, 3))
    assert torch.equal(b[:, 3:-3, 3:-3, 3:-3], want)


def test_512_fp32comp_within_bar_of_fp64():
    torch = _torch()
    n = 512
    f = _random_mesh(torch, n, 12)
    with ab.Device(ab.make_info(n, **ab.CONFIG_PARAMS)) as dev:
        a = _steps(dev, torch, f, 5)[:, 3:-3, 3:-3, 3:-3]
    with ab.Device(ab.make_info(n, precision=1, **ab.CONFIG_PARAMS)) as dev:
        b = _steps(dev, torch, f, 5)[:, 3:-3, 3:-3, 3:-3]
    num = (b - a).abs().reshape(8, -1).amax(dim=1)
    den = a.abs().reshape(8, -1).amax(dim=1)
    err = (num / den).cpu().numpy()
    assert err.max() <= 1e-5, err


@pytest.mark.slow
def test_256_cubed_one_step_against_oracle():
    """256^3, seed 2: one step against the oracle (about 20 s of oracle CPU time)."""
    info = ab.make_info(256, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 2)
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        dev.integrate_step(DT)
        dev.synchronize()
        got = dev.store_mesh()
    oracle.integrate(f, info_to_dict(info), DT, 1, "port")
    err = oracle.rel_linf(got, f)
    assert err.max() <= 1e-12, err
