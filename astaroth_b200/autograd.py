"""torch.autograd over the C ABI: the MHD time integration as a differentiable
function of the initial fields and of nu, eta.

Forward: N RK3 steps of the device integrator (acDeviceIntegrateStep), with a
checkpoint of the state every k steps.  Backward: for each checkpoint segment,
from the last to the first, the segment is integrated again from its
checkpoint, keeping the three substep states f_0, f_1, f_2 of every step
(acDeviceAdjointTapeForward); then for each step (last first) the discrete
adjoint substeps s = 2, 1, 0 are applied (acDeviceAdjointTapeBackward, i.e.
acDeviceIntegrateSubstepAdjoint about the taped states).  Every step is
recomputed once, except the last segment: the forward pass integrates it
through the tape already, and the backward pass uses those states unless the
device's tape was written since.  Memory: N/k checkpoints plus 3k substep
states.

Tensors are (8, mz, my, mx) float64 on the GPU (halos included, as the host
AcMesh).  The integration fills the halos itself, so gradients live on the
interior; the returned gradient is zero on the halo cells.
"""
from __future__ import annotations

import ctypes as C
import math

import torch

from . import capi
from .device import AstarothError, Device

D1 = (3 / 4, -3 / 20, 1 / 60)


def interior(t):
    return t[..., 3:-3, 3:-3, 3:-3]


def _d1(f, axis, inv_ds):
    """6th-order first derivative of periodic interior data along a tensor axis."""
    out = torch.zeros_like(f)
    for k, c in zip((1, 2, 3), D1):
        out = out + c * (torch.roll(f, -k, axis) - torch.roll(f, k, axis))
    return out * inv_ds


def energy_density(fields: torch.Tensor, info) -> torch.Tensor:
    """Per-cell terms of J over the interior: (1/2) exp(lnrho) |u|^2 dV +
    |curl A|^2 / (2 mu0) dV, with the same 6th-order first derivatives as the
    solver (periodic box).  Differences of J between nearby states are best
    formed cell by cell from these, before the sum."""
    q = interior(fields)
    ds = info.real3_params[capi.Real3Param.AC_ds]
    inv = (1.0 / ds.x, 1.0 / ds.y, 1.0 / ds.z)
    dV = ds.x * ds.y * ds.z
    mu0 = info.real_params[capi.RealParam.AC_mu0]
    lnrho, u, a = q[0], q[1:4], q[4:7]
    ekin = 0.5 * (torch.exp(lnrho) * (u * u).sum(0)) * dV
    # axes of a field: (z, y, x) -> x = 2, y = 1, z = 0
    g = [[_d1(a[c], 2, inv[0]), _d1(a[c], 1, inv[1]), _d1(a[c], 0, inv[2])] for c in range(3)]
    bx = g[2][1] - g[1][2]
    by = g[0][2] - g[2][0]
    bz = g[1][0] - g[0][1]
    emag = (bx * bx + by * by + bz * bz) / (2.0 * mu0) * dV
    return ekin + emag


class _Energy(torch.autograd.Function):
    """J and dJ/dfields by the library's energy kernels (acEnergyFunctional)."""

    @staticmethod
    def forward(ctx, fields, info):
        lib = capi.load()
        f = fields.detach().contiguous()
        scratch = torch.empty(lib.acEnergyFunctionalScratchBytes(info) // 8 + 1,
                              dtype=torch.float64, device=f.device)
        J = torch.empty((), dtype=torch.float64, device=f.device)
        ptrs = (C.c_void_p * 8)(*[f[q].data_ptr() for q in range(8)])
        stream = torch.cuda.current_stream(f.device).cuda_stream
        if lib.acEnergyFunctional(info, ptrs, C.c_void_p(J.data_ptr()), None,
                                  C.c_void_p(scratch.data_ptr()), C.c_void_p(stream)) != 0:
            raise AstarothError("acEnergyFunctional failed")
        ctx.save_for_backward(f)
        ctx.info = info
        return J

    @staticmethod
    def backward(ctx, gJ):
        (f,) = ctx.saved_tensors
        lib = capi.load()
        scratch = torch.empty(lib.acEnergyFunctionalScratchBytes(ctx.info) // 8 + 1,
                              dtype=torch.float64, device=f.device)
        J = torch.empty((), dtype=torch.float64, device=f.device)
        grad = torch.zeros_like(f)
        fp = (C.c_void_p * 8)(*[f[q].data_ptr() for q in range(8)])
        gp = (C.c_void_p * 8)(*[grad[q].data_ptr() for q in range(8)])
        stream = torch.cuda.current_stream(f.device).cuda_stream
        if lib.acEnergyFunctional(ctx.info, fp, C.c_void_p(J.data_ptr()), gp,
                                  C.c_void_p(scratch.data_ptr()), C.c_void_p(stream)) != 0:
            raise AstarothError("acEnergyFunctional failed")
        return grad * gJ, None


def energy(fields: torch.Tensor, info) -> torch.Tensor:
    """J = sum over the interior of (1/2) exp(lnrho) |u|^2 dV + |curl A|^2 / (2 mu0) dV,
    with the same 6th-order first derivatives as the solver (periodic box); on a
    CUDA tensor by the library's kernels (value and gradient), else in torch."""
    if fields.is_cuda:
        return _Energy.apply(fields, info)
    return energy_density(fields, info).sum()


class _Integrate(torch.autograd.Function):
    @staticmethod
    def forward(ctx, f0, nu, eta, dev, steps, dt, every, tape):
        dev.set_real(capi.RealParam.AC_nu_visc, float(nu))
        dev.set_real(capi.RealParam.AC_eta, float(eta))
        dev.load_mesh_device(f0.contiguous())
        ckpts = [f0.detach().clone()]
        last0 = (steps - 1) // every * every  # first step of the last segment
        token = None
        for n in range(steps):
            if tape and n == last0:
                # the last segment through the tape, whose substep states the
                # backward pass then uses without integrating it again
                try:
                    token = dev.adjoint_tape_forward(steps - last0, dt)
                    break
                except AstarothError:
                    pass  # no adjoint on this device (FP32, upwinding): plain steps
            dev.integrate_step(dt)
            if (n + 1) % every == 0 and n + 1 < steps:
                ckpts.append(dev.store_mesh_device(torch.empty_like(f0)))
        out = dev.store_mesh_device(torch.empty_like(f0))
        torch.cuda.synchronize()
        ctx.dev, ctx.steps, ctx.dt, ctx.every, ctx.ckpts = dev, steps, dt, every, ckpts
        ctx.nu, ctx.eta, ctx.tape, ctx.token = float(nu), float(eta), tape, token
        return out

    @staticmethod
    def backward(ctx, grad_out):
        dev, steps, dt, every = ctx.dev, ctx.steps, ctx.dt, ctx.every
        dev.set_real(capi.RealParam.AC_nu_visc, ctx.nu)
        dev.set_real(capi.RealParam.AC_eta, ctx.eta)
        lam = torch.zeros_like(grad_out)
        interior(lam).copy_(interior(grad_out))
        dev.load_adjoint(lam)
        torch.cuda.synchronize()
        for seg in reversed(range(len(ctx.ckpts))):
            n0 = seg * every
            n1 = min(n0 + every, steps)
            last = seg == len(ctx.ckpts) - 1
            if last and ctx.tape and ctx.token is not None and dev.tape_token is ctx.token:
                # the last segment's states are still on the tape from the forward pass
                dev.adjoint_tape_backward(n1 - n0, dt)
                continue
            dev.load_mesh_device(ctx.ckpts[seg], wait_torch=False)
            if ctx.tape:
                # the library keeps the segment's substep states on its own tape
                dev.adjoint_tape_forward(n1 - n0, dt)
                dev.adjoint_tape_backward(n1 - n0, dt)
                continue
            # the same sweep through the per-substep entry points, with the
            # substep states f_0, f_1, f_2 of every step kept in torch tensors
            buf = [torch.empty_like(grad_out) for _ in range(3 * (n1 - n0))]
            for n in range(n1 - n0):
                for s in range(3):
                    dev.store_mesh_device(buf[3 * n + s], sync=False)
                    if n == n1 - n0 - 1 and s == 2:
                        break  # the segment's final state is not needed
                    dev.periodic_boundconds()
                    dev.integrate_substep(s, dt)
                    dev.swap_buffers()
            for n in reversed(range(n1 - n0)):
                for s in (2, 1, 0):
                    dev.load_mesh_device(buf[3 * n + s], wait_torch=False)
                    dev.periodic_boundconds()
                    dev.integrate_substep_adjoint(s, dt)
        g0 = dev.store_adjoint(torch.zeros_like(grad_out))
        out = torch.zeros_like(g0)
        interior(out).copy_(interior(g0))
        nu_bar, eta_bar = dev.param_adjoints()
        dtype, device = grad_out.dtype, grad_out.device
        return (out, torch.tensor(nu_bar, dtype=dtype, device=device),
                torch.tensor(eta_bar, dtype=dtype, device=device), None, None, None, None, None)


def integrate(f0: torch.Tensor, nu, eta, dev: Device, steps: int, dt: float,
              checkpoint_every: int | None = None, tape: bool = True) -> torch.Tensor:
    """Differentiable N-step integration on `dev` (an FP64 Device of matching size).

    f0: (8, mz, my, mx) float64 CUDA tensor; nu, eta: 0-d tensors (may require grad).
    Returns the final state; backward gives d/d f0 (interior), d/d nu and d/d eta.
    tape=True sweeps each segment with acDeviceAdjointTapeForward/Backward (the
    library keeps the substep states); tape=False makes one call per substep
    (acDevicePeriodicBoundconds + acDeviceIntegrateSubstepAdjoint) with the
    states in torch tensors.  Both apply the same kernels in the same order.
    """
    every = checkpoint_every or max(1, int(math.sqrt(steps)))
    nu = torch.as_tensor(nu, dtype=torch.float64, device=f0.device)
    eta = torch.as_tensor(eta, dtype=torch.float64, device=f0.device)
    return _Integrate.apply(f0, nu, eta, dev, steps, dt, every, tape)
