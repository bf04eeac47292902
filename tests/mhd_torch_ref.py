"""Test infrastructure: the MHD RHS and 2N RK3 step written in PyTorch (FP64) on
the periodic interior, for CPU reference gradients through torch.autograd.

It restates the reference host model (src/utils/modelsolver.cc:772-964 for the
equations, :190-299 for the 6th-order stencils, :1078-1175 for RK3) with
torch.roll for the periodic taps; the tests pin it against the oracle before
using its gradients.  Arrays are (8, nz, ny, nx): lnrho, ux, uy, uz, ax, ay, az,
entropy; tensor axes (z, y, x).
"""
import torch

C1 = (3 / 4, -3 / 20, 1 / 60)
C2 = (-49 / 18, 3 / 2, -3 / 20, 1 / 90)
CM = (270 / 720, -27 / 720, 2 / 720)
AX = (2, 1, 0)  # tensor axis of x, y, z


def d1(f, a, inv):
    r = 0
    for k, c in zip((1, 2, 3), C1):
        r = r + c * (torch.roll(f, -k, AX[a]) - torch.roll(f, k, AX[a]))
    return r * inv[a]


def d2(f, a, inv):
    r = C2[0] * f
    for k, c in zip((1, 2, 3), C2[1:]):
        r = r + c * (torch.roll(f, -k, AX[a]) + torch.roll(f, k, AX[a]))
    return r * inv[a] * inv[a]


def dmix(f, a, b, inv):
    r = 0
    for k, c in zip((1, 2, 3), CM):
        pp = torch.roll(f, (-k, -k), (AX[a], AX[b]))
        mm = torch.roll(f, (k, k), (AX[a], AX[b]))
        pm = torch.roll(f, (-k, k), (AX[a], AX[b]))
        mp = torch.roll(f, (k, -k), (AX[a], AX[b]))
        r = r + c * (pp + mm - pm - mp)
    return r * inv[a] * inv[b]


def rates(f, p, nu=None, eta=None):
    """RHS of the 8 fields; nu / eta may be tensors (for parameter gradients)."""
    nu = p["nu_visc"] if nu is None else nu
    eta = p["eta"] if eta is None else eta
    inv = [1.0 / d for d in p["ds"]]
    lnrho, u, a, s = f[0], f[1:4], f[4:7], f[7]
    gl = [d1(lnrho, i, inv) for i in range(3)]
    gs = [d1(s, i, inv) for i in range(3)]
    lapl = sum(d2(lnrho, i, inv) for i in range(3))
    laps = sum(d2(s, i, inv) for i in range(3))
    gu = [[d1(u[c], i, inv) for i in range(3)] for c in range(3)]
    ga = [[d1(a[c], i, inv) for i in range(3)] for c in range(3)]
    hu = [[d2(u[c], i, inv) if i == c else None for i in range(3)] for c in range(3)]
    lapu = [sum(d2(u[c], i, inv) for i in range(3)) for c in range(3)]
    lapa = [sum(d2(a[c], i, inv) for i in range(3)) for c in range(3)]

    def graddiv(v, diag):
        return [diag(v, 0) + dmix(v[1], 0, 1, inv) + dmix(v[2], 0, 2, inv),
                dmix(v[0], 0, 1, inv) + diag(v, 1) + dmix(v[2], 1, 2, inv),
                dmix(v[0], 0, 2, inv) + dmix(v[1], 1, 2, inv) + diag(v, 2)]

    diag = lambda v, c: d2(v[c], c, inv)  # noqa: E731
    gdu = graddiv(u, diag)
    gda = graddiv(a, diag)
    del hu
    divu = gu[0][0] + gu[1][1] + gu[2][2]
    r_lnrho = -(u[0] * gl[0] + u[1] * gl[1] + u[2] * gl[2]) - divu
    B = [ga[2][1] - ga[1][2], ga[0][2] - ga[2][0], ga[1][0] - ga[0][1]]
    ind = [u[1] * B[2] - u[2] * B[1] + eta * lapa[0],
           u[2] * B[0] - u[0] * B[2] + eta * lapa[1],
           u[0] * B[1] - u[1] * B[0] + eta * lapa[2]]
    S = [[None] * 3 for _ in range(3)]
    for c in range(3):
        S[c][c] = (2 / 3) * gu[c][c] - (1 / 3) * sum(gu[d][d] for d in range(3) if d != c)
    for c, b in ((0, 1), (0, 2), (1, 2)):
        S[c][b] = S[b][c] = 0.5 * (gu[c][b] + gu[b][c])
    gamma, cp = p["gamma"], p["cp_sound"]
    cs2 = p["cs_sound"] ** 2 * torch.exp(gamma * s / cp + (gamma - 1) * (lnrho - p["lnrho0"]))
    jj = [(gda[c] - lapa[c]) / p["mu0"] for c in range(3)]
    inv_rho = 1.0 / torch.exp(lnrho)
    jxb = [jj[1] * B[2] - jj[2] * B[1], jj[2] * B[0] - jj[0] * B[2], jj[0] * B[1] - jj[1] * B[0]]
    mom = []
    for c in range(3):
        adv = gu[c][0] * u[0] + gu[c][1] * u[1] + gu[c][2] * u[2]
        sgl = S[c][0] * gl[0] + S[c][1] * gl[1] + S[c][2] * gl[2]
        mom.append(-adv - cs2 * (gs[c] / cp + gl[c]) + inv_rho * jxb[c]
                   + nu * (lapu[c] + gdu[c] / 3 + 2 * sgl) + p["zeta"] * gdu[c])
    lnT = p["lnT0"] + gamma * s / cp + (gamma - 1) * (lnrho - p["lnrho0"])
    inv_pT = 1.0 / (torch.exp(lnrho) * torch.exp(lnT))
    contract = sum(S[c][b] * S[c][b] for c in range(3) for b in range(3))
    rhs = (eta * p["mu0"] * (jj[0] ** 2 + jj[1] ** 2 + jj[2] ** 2)
           + 2 * torch.exp(lnrho) * nu * contract + p["zeta"] * torch.exp(lnrho) * divu * divu)
    first = gamma / cp * laps + (gamma - 1) * lapl
    second = [gamma / cp * gs[i] + (gamma - 1) * gl[i] for i in range(3)]
    third = [gamma * (gs[i] / cp + gl[i]) - gl[i] for i in range(3)]
    chi = p["K_heatcond"] / (torch.exp(lnrho) * cp)
    heat = cp * chi * (first + sum(second[i] * third[i] for i in range(3)))
    r_s = -(u[0] * gs[0] + u[1] * gs[1] + u[2] * gs[2]) + inv_pT * rhs + heat
    return torch.stack([r_lnrho, mom[0], mom[1], mom[2], ind[0], ind[1], ind[2], r_s])


ALPHA = (0.0, -5.0 / 9.0, -153.0 / 128.0)
BETA = (1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0)


def step(f, p, dt, nu=None, eta=None):
    """One 2N RK3 step (w form)."""
    w = torch.zeros_like(f)
    for s in range(3):
        w = ALPHA[s] * w + dt * rates(f, p, nu, eta)
        f = f + BETA[s] * w
    return f


def energy(f, p):
    inv = [1.0 / d for d in p["ds"]]
    dV = p["ds"][0] * p["ds"][1] * p["ds"][2]
    lnrho, u, a = f[0], f[1:4], f[4:7]
    ga = [[d1(a[c], i, inv) for i in range(3)] for c in range(3)]
    B = [ga[2][1] - ga[1][2], ga[0][2] - ga[2][0], ga[1][0] - ga[0][1]]
    ekin = 0.5 * (torch.exp(lnrho) * (u * u).sum(0)).sum() * dV
    emag = (B[0] ** 2 + B[1] ** 2 + B[2] ** 2).sum() / (2 * p["mu0"]) * dV
    return ekin + emag
