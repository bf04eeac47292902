"""GPU tests of the discrete adjoint (acDeviceIntegrateSubstepAdjoint) and of
the torch.autograd wrapper (astaroth_b200.autograd).

* one adjoint substep against torch.autograd of the FP64 torch restatement of
  the model (tests/mhd_torch_ref.py, pinned against the oracle in
  tests/test_oracle.py);
* the gradient of J = E_kin + E_mag after several steps w.r.t. the initial
  fields and nu, eta against the same CPU reference gradient;
* 64^3, 200 steps, dt = 1e-3, seed 4, checkpoints every 20 steps:
  central finite differences (h = 1e-6) in 32 random directions and in nu, eta,
  strictly within 1e-6;
* the exact dot-product identity of the 200-step map against the tangent-linear
  model of the CPU torch restatement;
* the gradient on the 64^3 benchmark mesh over 5 steps against the CPU torch
  reference;
* the forward in FP32 compensated, against the FP64 gradient.
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


def test_energy_kernel_matches_torch():
    """acEnergyFunctional (J and dJ/dfields) against the torch expression of the
    same functional (per-cell densities summed, and torch autograd)."""
    torch = _torch()
    from astaroth_b200 import autograd as AG
    info, f = mesh((40, 24, 20), 36)
    x = torch.from_numpy(f).cuda().requires_grad_(True)
    J = AG.energy(x, info)  # the kernels
    J.backward()
    y = torch.from_numpy(f).cuda().requires_grad_(True)
    Jt = AG.energy_density(y, info).sum()  # torch
    Jt.backward()
    assert abs(float(J) - float(Jt)) <= 1e-13 * abs(float(Jt))
    g, gt = x.grad.cpu().numpy(), y.grad.cpu().numpy()
    for q in range(8):
        scale = max(np.abs(gt[q]).max(), 1e-300)
        assert np.abs(g[q] - gt[q]).max() <= 1e-12 * scale, q
    assert np.all(g[:, :3] == 0) and np.all(g[:, -3:] == 0)  # halos untouched


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


def fd_energy(run, info, f0, d, h):
    """Central difference of J along d: the per-cell energy differences are
    formed before the sum, so the difference of two nearly equal sums (each
    with roundoff ~1e-16 J log N) does not swamp it."""
    from astaroth_b200 import autograd as AG
    ep = AG.energy_density(run(f0 + h * d), info)
    em = AG.energy_density(run(f0 - h * d), info)
    return float((ep - em).sum()) / (2 * h)


def test_64_cubed_200_steps_fd_and_cost():
    """64^3, 200 steps, dt = 1e-3, seed 4, checkpoints every 20 steps: central
    finite differences with h = 1e-6 in 32 random directions (per field scaled
    to the field's initial amplitude) and in nu, eta, strictly within 1e-6."""
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
        fN = AG.integrate(x0, nu, eta, dev, steps, dt, checkpoint_every=every)
        J = AG.energy(fN, info)
        t0 = time.perf_counter()
        J.backward()
        torch.cuda.synchronize()
        t_bwd = time.perf_counter() - t0
        peak = torch.cuda.max_memory_allocated()
        g = x0.grad
        rng = np.random.default_rng(4)
        errs = []
        for i in range(32):
            d = np.zeros_like(f)
            oracle.interior(d)[...] = (rng.standard_normal(oracle.interior(d).shape)
                                       * SCALES[:, None, None, None])
            dt_ = torch.from_numpy(d).cuda()
            fd = fd_energy(run, info, f0, dt_, h)
            ad = float((g * dt_).sum())
            errs.append(abs(fd - ad) / abs(ad))
        # nu and eta (relative steps)
        def fd_param(which, v0):
            kw_p = {which: v0 * (1 + h)}
            kw_m = {which: v0 * (1 - h)}
            ep = AG.energy_density(run(f0, **kw_p), info)
            em = AG.energy_density(run(f0, **kw_m), info)
            return float((ep - em).sum()) / (2 * h * v0)
        fd_nu = fd_param("nu", nu0)
        fd_eta = fd_param("eta", eta0)
    print(f"\nadjoint 64^3 x 200 steps: forward {t_fwd * 1e3:.1f} ms, adjoint (recompute + "
          f"reverse) {t_bwd * 1e3:.1f} ms, ratio {t_bwd / t_fwd:.2f}, peak torch memory "
          f"{peak / 2**20:.0f} MiB; FD (h=1e-6, 32 directions) rel err max {max(errs):.2e}, "
          f"median {np.median(errs):.2e}; nu {abs(fd_nu - float(nu.grad)) / abs(float(nu.grad)):.2e}, "
          f"eta {abs(fd_eta - float(eta.grad)) / abs(float(eta.grad)):.2e}")
    assert max(errs) <= 1e-6, errs
    assert abs(fd_nu - float(nu.grad)) <= 1e-6 * abs(float(nu.grad))
    assert abs(fd_eta - float(eta.grad)) <= 1e-6 * abs(float(eta.grad))


def test_dot_product_against_tangent_linear_200_steps():
    """The exact adjoint identity <M dx, l> = <dx, M^T l> for the 200-step map M:
    M dx is the tangent-linear model of the CPU torch restatement of the solver
    (forward-mode derivatives, tests/mhd_torch_ref.py), M^T l the GPU adjoint
    through the checkpointed autograd wrapper; both are exact linearisations of
    the same discrete map, so they agree to FP64 rounding."""
    torch = _torch()
    from torch.func import jvp
    from astaroth_b200 import autograd as AG
    info, f = mesh((24, 20, 16), 35)
    p = ab.info_to_dict(info)
    steps, dt = 200, 1e-3
    rng = np.random.default_rng(35)
    lam = np.zeros_like(f)
    oracle.interior(lam)[...] = rng.standard_normal(oracle.interior(lam).shape)
    dx = np.zeros_like(f)
    oracle.interior(dx)[...] = (rng.standard_normal(oracle.interior(dx).shape)
                                * SCALES[:, None, None, None])
    # M^T l on the GPU
    x0 = torch.from_numpy(f).cuda().requires_grad_(True)
    with ab.Device(info) as dev:
        out = AG.integrate(x0, p["nu_visc"], p["eta"], dev, steps, dt, checkpoint_every=20)
        (out * torch.from_numpy(lam).cuda()).sum().backward()
    rhs = float((x0.grad.cpu() * torch.from_numpy(dx)).sum())
    # M dx on the CPU: forward-mode through the restated model
    def m(x):
        for _ in range(steps):
            x = R.step(x, p, dt)
        return x
    xi = torch.from_numpy(oracle.interior(f).copy())
    di = torch.from_numpy(oracle.interior(dx).copy())
    _, tangent = jvp(m, (xi,), (di,))
    lhs = float((tangent * torch.from_numpy(oracle.interior(lam).copy())).sum())
    print(f"\ndot-product test (200 steps): <M dx, l> = {lhs:.15e}, <dx, M^T l> = {rhs:.15e}, "
          f"rel {abs(lhs - rhs) / abs(rhs):.2e}")
    assert abs(lhs - rhs) <= 1e-10 * abs(rhs)


def test_64_cubed_gradient_matches_cpu_reference_5_steps():
    """The benchmark mesh (64^3, seed 4), 5 steps: the GPU gradient of J against
    torch autograd through the CPU restatement of the model."""
    torch = _torch()
    from astaroth_b200 import autograd as AG
    info = ab.make_info(64, **ab.CONFIG_PARAMS)
    f = ab.seeded_mesh(info, 4)
    oracle.periodic_bounds(f, "port")
    p = ab.info_to_dict(info)
    steps, dt = 5, 1e-3
    f0 = torch.from_numpy(f).cuda().requires_grad_(True)
    nu = torch.tensor(p["nu_visc"], dtype=torch.float64, device="cuda", requires_grad=True)
    eta = torch.tensor(p["eta"], dtype=torch.float64, device="cuda", requires_grad=True)
    with ab.Device(info) as dev:
        fN = AG.integrate(f0, nu, eta, dev, steps, dt, checkpoint_every=2)
        J = AG.energy(fN, info)
        J.backward()
    g_gpu = AG.interior(f0.grad).cpu().numpy()
    fc = torch.from_numpy(oracle.interior(f).copy()).requires_grad_(True)
    nuc = torch.tensor(p["nu_visc"], dtype=torch.float64, requires_grad=True)
    etac = torch.tensor(p["eta"], dtype=torch.float64, requires_grad=True)
    x = fc
    for _ in range(steps):
        x = R.step(x, p, dt, nuc, etac)
    Jc = R.energy(x, p)
    Jc.backward()
    errs = [rel(g_gpu[q], fc.grad[q].numpy()) for q in range(8)]
    print(f"\n64^3 x 5 steps: gradient vs CPU reference, per field rel Linf {errs}")
    assert max(errs) <= 1e-9, errs
    assert abs(float(nu.grad) - float(nuc.grad)) <= 1e-9 * abs(float(nuc.grad))
    assert abs(float(eta.grad) - float(etac.grad)) <= 1e-9 * abs(float(etac.grad))


def test_fp32comp_forward_gradient_vs_fp64():
    """The benchmark adjoint workload with the forward (and its tape) in FP32
    compensated: the reverse sweep, its inner products and the parameter
    adjoints stay FP64, about the (hi, lo) states joined to doubles.  Per-field
    relative L-inf of the gradient against the all-FP64 gradient."""
    torch = _torch()
    from astaroth_b200 import autograd as AG
    steps, dt, every = 200, 1e-3, 20
    grads = {}
    for prec in (0, 1):
        info = ab.make_info(64, precision=prec, **ab.CONFIG_PARAMS)
        f = ab.seeded_mesh(info, 4)
        p = ab.info_to_dict(info)
        x0 = torch.from_numpy(f).cuda().requires_grad_(True)
        nu = torch.tensor(p["nu_visc"], dtype=torch.float64, device="cuda", requires_grad=True)
        eta = torch.tensor(p["eta"], dtype=torch.float64, device="cuda", requires_grad=True)
        with ab.Device(info) as dev:
            fN = AG.integrate(x0, nu, eta, dev, steps, dt, checkpoint_every=every)
            AG.energy(fN, info).backward()
        grads[prec] = (AG.interior(x0.grad).cpu().numpy(), float(nu.grad), float(eta.grad))
    errs = [rel(grads[1][0][q], grads[0][0][q]) for q in range(8)]
    e_nu = abs(grads[1][1] - grads[0][1]) / abs(grads[0][1])
    e_eta = abs(grads[1][2] - grads[0][2]) / abs(grads[0][2])
    print(f"\nFP32-compensated forward: gradient rel Linf per field vs FP64 {errs}; "
          f"nu {e_nu:.2e}, eta {e_eta:.2e}")
    assert max(errs) <= 1e-4, errs
    assert e_nu <= 1e-4 and e_eta <= 1e-4
