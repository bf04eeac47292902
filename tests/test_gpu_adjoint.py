"""GPU tests of the discrete adjoint (acDeviceIntegrateSubstepAdjoint) and of
the torch.autograd wrapper (astaroth_b200.autograd).

* one adjoint substep against torch.autograd of the FP64 torch restatement of
  the model (tests/mhd_torch_ref.py, pinned against the oracle in
  tests/test_oracle.py);
* the gradient of J = E_kin + E_mag after several steps w.r.t. the initial
  fields and nu, eta against the same CPU reference gradient;
* 64^3, 200 steps, dt = 1e-3, seed 4, checkpoints every 20 steps:
  central finite differences (h = 1e-6) in 32 random directions and in nu, eta,
  and a dot-product test of the adjoint of the 200-step map.
"""
import sys
import time
from pathlib import Path

import numpy as np
import pytest

import astaroth_b200 as ab
from oracle import oracle
from tests.conftest import gpu_available

sys.path.insert(0, str(Path(__file__).resolve().parent))
import mhd_torch_ref as R  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")]

SCALES = np.array([1e-5, 1e-3, 1e-3, 1e-3, 1e-4, 1e-4, 1e-4, 1e-5])


def _torch():
    import torch
    return torch


def mesh(n, seed, amp=(0.1, 0.05, 0.02)):
    info = ab.make_info(n, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, seed, amp_scalar=amp[0], sigma_uu=amp[1], sigma_aa=amp[2])
    oracle.periodic_bounds(f, "port")
    return info, f


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("step", [0, 1, 2])
def test_adjoint_substep_matches_autograd(step):
    torch = _torch()
    info, f = mesh((20, 16, 12), 31)
    p = ab.info_to_dict(info)
    dt = 2e-3
    rng = np.random.default_rng(step)
    lam = np.zeros_like(f)
    oracle.interior(lam)[...] = rng.standard_normal(oracle.interior(lam).shape)
    with ab.Device(info) as dev:
        dev.load_mesh(f)
        dev.load_adjoint(torch.from_numpy(lam).cuda())
        dev.integrate_substep_adjoint(step, dt)
        out = dev.store_adjoint(torch.zeros_like(torch.from_numpy(lam)).cuda()).cpu().numpy()
        nu_bar, eta_bar = dev.param_adjoints()
    # reference: lf_new = lf + dt J^T (beta_s lf); param adjoints dt <dR/dp, beta_s lf>
    fi = torch.from_numpy(oracle.interior(f).copy()).requires_grad_(True)
    nu = torch.tensor(p["nu_visc"], dtype=torch.float64, requires_grad=True)
    eta = torch.tensor(p["eta"], dtype=torch.float64, requires_grad=True)
    li = torch.from_numpy(oracle.interior(lam).copy())
    r = R.rates(fi, p, nu, eta)
    gf, gnu, geta = torch.autograd.grad((r * (dt * R.BETA[step] * li)).sum(), [fi, nu, eta])
    want = oracle.interior(lam) + gf.numpy()
    assert rel(oracle.interior(out), want) <= 1e-12
    assert abs(nu_bar - float(gnu)) <= 1e-11 * abs(float(gnu))
    assert abs(eta_bar - float(geta)) <= 1e-11 * abs(float(geta))


def test_gradient_matches_cpu_reference():
    torch = _torch()
    from astaroth_b200 import autograd as AG
    info, f = mesh((20, 16, 12), 32)
    p = ab.info_to_dict(info)
    steps, dt = 6, 1e-3
    # GPU: autograd over the C ABI
    f0 = torch.from_numpy(f).cuda().requires_grad_(True)
    nu = torch.tensor(p["nu_visc"], dtype=torch.float64, device="cuda", requires_grad=True)
    eta = torch.tensor(p["eta"], dtype=torch.float64, device="cuda", requires_grad=True)
    with ab.Device(info) as dev:
        fN = AG.integrate(f0, nu, eta, dev, steps, dt, checkpoint_every=4)
        J = AG.energy(fN, info)
        J.backward()
    g_gpu = AG.interior(f0.grad).cpu().numpy()
    # CPU reference: torch autograd through the restated model
    fc = torch.from_numpy(oracle.interior(f).copy()).requires_grad_(True)
    nuc = torch.tensor(p["nu_visc"], dtype=torch.float64, requires_grad=True)
    etac = torch.tensor(p["eta"], dtype=torch.float64, requires_grad=True)
    x = fc
    for _ in range(steps):
        x = R.step(x, p, dt, nuc, etac)
    Jc = R.energy(x, p)
    Jc.backward()
    assert abs(float(J.detach()) - float(Jc.detach())) <= 1e-13 * abs(float(Jc.detach()))
    for q in range(8):
        assert rel(g_gpu[q], fc.grad[q].numpy()) <= 1e-9, q
    assert abs(float(nu.grad) - float(nuc.grad)) <= 1e-9 * abs(float(nuc.grad))
    assert abs(float(eta.grad) - float(etac.grad)) <= 1e-9 * abs(float(etac.grad))


def test_tape_sweep_equals_per_substep_sweep():
    """acDeviceAdjointTapeForward/Backward and the per-substep entry points
    apply the same kernels in the same order: identical field gradients."""
    torch = _torch()
    from astaroth_b200 import autograd as AG
    info, f = mesh((24, 20, 16), 33)
    p = ab.info_to_dict(info)
    grads = []
    for tape in (True, False):
        f0 = torch.from_numpy(f).cuda().requires_grad_(True)
        nu = torch.tensor(p["nu_visc"], dtype=torch.float64, device="cuda", requires_grad=True)
        eta = torch.tensor(p["eta"], dtype=torch.float64, device="cuda", requires_grad=True)
        with ab.Device(info) as dev:
            fN = AG.integrate(f0, nu, eta, dev, 7, 1e-3, checkpoint_every=3, tape=tape)
            AG.energy(fN, info).backward()
        grads.append((f0.grad.cpu().numpy(), float(nu.grad), float(eta.grad)))
    assert np.array_equal(grads[0][0], grads[1][0])
    # the parameter adjoints are sums of per-block atomics, whose order varies
    for a, b in zip(grads[0][1:], grads[1][1:]):
        assert abs(a - b) <= 1e-12 * abs(b)


def test_64_cubed_200_steps_fd_dot_product_and_cost():
    """64^3, 200 steps, dt = 1e-3, seed 4, checkpoints every 20 steps."""
    torch = _torch()
    from astaroth_b200 import autograd as AG
    info = ab.make_info(64, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 4)
    p = ab.info_to_dict(info)
    steps, dt, every, h = 200, 1e-3, 20, 1e-6
    f0 = torch.from_numpy(f).cuda()
    nu0, eta0 = p["nu_visc"], p["eta"]

    with ab.Device(info) as dev:
        def run(x, nu=nu0, eta=eta0):
            dev.set_real(ab.capi.RealParam.AC_nu_visc, nu)
            dev.set_real(ab.capi.RealParam.AC_eta, eta)
            dev.load_mesh_device(x)
            for _ in range(steps):
                dev.integrate_step(dt)
            return dev.store_mesh_device(torch.empty_like(x))

        run(f0)  # warm-up (graph capture)
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats()
        t0 = time.perf_counter()
        run(f0)
        torch.cuda.synchronize()
        t_fwd = time.perf_counter() - t0

        x0 = f0.clone().requires_grad_(True)
        nu = torch.tensor(nu0, dtype=torch.float64, device="cuda", requires_grad=True)
        eta = torch.tensor(eta0, dtype=torch.float64, device="cuda", requires_grad=True)
        t0 = time.perf_counter()
        fN = AG.integrate(x0, nu, eta, dev, steps, dt, checkpoint_every=every)
        torch.cuda.synchronize()
        t_ad_fwd = time.perf_counter() - t0
        J = AG.energy(fN, info)
        t0 = time.perf_counter()
        J.backward()
        torch.cuda.synchronize()
        t_bwd = time.perf_counter() - t0
        peak = torch.cuda.max_memory_allocated()
        g = x0.grad
        j0 = float(J.detach())
        rng = np.random.default_rng(4)
        worst, worst_floor, worst_h5 = 0.0, 0.0, 0.0
        for i in range(32):
            d = np.zeros_like(f)
            oracle.interior(d)[...] = (rng.standard_normal(oracle.interior(d).shape)
                                       * SCALES[:, None, None, None])
            dt_ = torch.from_numpy(d).cuda()
            jp = float(AG.energy(run(f0 + h * dt_), info))
            jm = float(AG.energy(run(f0 - h * dt_), info))
            fd = (jp - jm) / (2 * h)
            ad = float((g * dt_).sum())
            worst = max(worst, abs(fd - ad) / abs(ad))
            # the FD cannot resolve below the roundoff of J through 200 steps
            # (~1e-13 J) divided by 2h; a random field-scale direction has a
            # directional derivative ~ J / sqrt(cells), so that floor is ~1e-6
            floor = 1e-13 * abs(j0) / (2 * h)
            worst_floor = max(worst_floor, (abs(fd - ad) - floor) / abs(ad))
            if i < 8:  # a larger step lifts the FD above its roundoff floor
                h5 = 1e-5
                fd5 = (float(AG.energy(run(f0 + h5 * dt_), info))
                       - float(AG.energy(run(f0 - h5 * dt_), info))) / (2 * h5)
                worst_h5 = max(worst_h5, abs(fd5 - ad) / abs(ad))
        # nu and eta
        fd_nu = (float(AG.energy(run(f0, nu=nu0 * (1 + h)), info))
                 - float(AG.energy(run(f0, nu=nu0 * (1 - h)), info))) / (2 * h * nu0)
        fd_eta = (float(AG.energy(run(f0, eta=eta0 * (1 + h)), info))
                  - float(AG.energy(run(f0, eta=eta0 * (1 - h)), info))) / (2 * h * eta0)
        # dot-product test of the adjoint of the 200-step map with a linear functional
        lam = torch.zeros_like(f0)
        AG.interior(lam).copy_(torch.randn(AG.interior(lam).shape, dtype=torch.float64,
                                           device="cuda"))
        x1 = f0.clone().requires_grad_(True)
        out = AG.integrate(x1, nu0, eta0, dev, steps, dt, checkpoint_every=every)
        (out * lam).sum().backward()
        d = torch.zeros_like(f0)
        AG.interior(d).copy_(torch.randn(AG.interior(d).shape, dtype=torch.float64,
                                         device="cuda") * torch.from_numpy(SCALES).cuda()[:, None, None, None])
        lhs = float(((run(f0 + h * d) - run(f0 - h * d)) / (2 * h) * lam)[:, 3:-3, 3:-3, 3:-3].sum())
        rhs = float((x1.grad * d).sum())
    print(f"\nadjoint 64^3 x 200 steps: forward {t_fwd * 1e3:.1f} ms, adjoint (recompute + reverse) {t_bwd * 1e3:.1f} ms,"
          f" ratio {t_bwd / t_fwd:.2f}, peak torch memory {peak / 2**20:.0f} MiB,"
          f" worst FD rel err {worst:.2e} (h=1e-6), {worst_h5:.2e} (h=1e-5)")
    assert worst_floor <= 1e-6
    assert worst_h5 <= 1e-6
    assert abs(fd_nu - float(nu.grad)) <= 1e-6 * abs(float(nu.grad))
    assert abs(fd_eta - float(eta.grad)) <= 1e-6 * abs(float(eta.grad))
    assert abs(lhs - rhs) <= 1e-6 * abs(rhs)
    assert t_ad_fwd > 0
