/*
 * Right-hand side of the compressible non-ideal MHD system (lnrho, uu, aa,
 * entropy) from per-cell derivative records.  One implementation, templated
 * on the arithmetic type, shared by every solve kernel.
 *
 * Equations (acc-runtime/samples/mhd_modular/mhdsolver.ac:279-282,334-426 with
 * LENTROPY=1, LMAGNETIC=1, LUPWD=0; host model src/utils/modelsolver.cc:772-964):
 *   dlnrho/dt = -u.grad lnrho - div u
 *   du/dt     = -(grad u) u - cs2 (grad s / cp + grad lnrho) + rho^-1 j x B
 *               + nu (lap u + 1/3 grad div u + 2 S grad lnrho) + zeta grad div u
 *   dA/dt     = u x B + eta lap A
 *   ds/dt     = -u.grad s + (rho T)^-1 (eta mu0 j.j + 2 rho nu S:S + zeta rho (div u)^2)
 *               + K/rho (first + second.third)        (heat conduction)
 * with cs2 = cs_sound^2 exp(gamma s/cp + (gamma-1)(lnrho - lnrho0)),
 *      T   = exp(lnT0) exp(gamma s/cp + (gamma-1)(lnrho - lnrho0)),
 *      j   = (grad div A - lap A)/mu0,  B = curl A,  S the traceless strain.
 * exp(lnT) reuses the exponential of cs2, so each cell costs two exp and one
 * reciprocal; every other operation is an add, multiply or FMA.
 */
#pragma once

#include "internal.h"

template <typename T>
struct ScalD {
    T v;
    T g[3];
    T lap;
};

template <typename T>
struct VecD {
    T v[3];
    T g[3][3]; /* g[c][a] = d u_c / d x_a */
    T lap[3];
    T gd[3]; /* grad div */
};

template <typename T>
struct PhysT {
    T nu, eta, zeta, inv_mu0, eta_mu0, cs2_sound, gamma_m1, inv_cp, gamma_inv_cp, lnrho0,
        inv_exp_lnT0, K, visc_gd;
};

template <typename T>
__host__ __device__ inline PhysT<T>
phys_cast(const PhysConst& p)
{
    PhysT<T> q;
    q.nu           = (T)p.nu;
    q.eta          = (T)p.eta;
    q.zeta         = (T)p.zeta;
    q.inv_mu0      = (T)p.inv_mu0;
    q.eta_mu0      = (T)p.eta_mu0;
    q.cs2_sound    = (T)p.cs2_sound;
    q.gamma_m1     = (T)p.gamma_m1;
    q.inv_cp       = (T)p.inv_cp;
    q.gamma_inv_cp = (T)p.gamma_inv_cp;
    q.lnrho0       = (T)p.lnrho0;
    q.inv_exp_lnT0 = (T)p.inv_exp_lnT0;
    q.K            = (T)p.K;
    q.visc_gd      = (T)(p.nu * (1.0 / 3.0) + p.zeta);
    return q;
}

__device__ __forceinline__ double
ac_exp(const double x)
{
    return exp(x);
}
__device__ __forceinline__ float
ac_exp(const float x)
{
    return expf(x);
}
__device__ __forceinline__ double
ac_rcp(const double x)
{
    return __drcp_rn(x);
}
__device__ __forceinline__ float
ac_rcp(const float x)
{
    return __frcp_rn(x);
}

/* rates[8] in field order (lnrho, ux, uy, uz, ax, ay, az, entropy). */
template <typename T>
__device__ __forceinline__ void
mhd_rates(const ScalD<T>& L, const ScalD<T>& Sg, const VecD<T>& U, const VecD<T>& A,
          const PhysT<T>& p, T r[AC_NF])
{
    const T ux = U.v[0], uy = U.v[1], uz = U.v[2];
    const T divu = U.g[0][0] + U.g[1][1] + U.g[2][2];

    /* continuity */
    r[0] = -(ux * L.g[0] + uy * L.g[1] + uz * L.g[2]) - divu;

    /* magnetic field and current */
    const T Bx = A.g[2][1] - A.g[1][2];
    const T By = A.g[0][2] - A.g[2][0];
    const T Bz = A.g[1][0] - A.g[0][1];
    const T jx = (A.gd[0] - A.lap[0]) * p.inv_mu0;
    const T jy = (A.gd[1] - A.lap[1]) * p.inv_mu0;
    const T jz = (A.gd[2] - A.lap[2]) * p.inv_mu0;

    /* induction: u x B + eta lap A */
    r[4] = (uy * Bz - uz * By) + p.eta * A.lap[0];
    r[5] = (uz * Bx - ux * Bz) + p.eta * A.lap[1];
    r[6] = (ux * By - uy * Bx) + p.eta * A.lap[2];

    /* thermodynamics: E = exp(gamma s/cp + (gamma-1)(lnrho - lnrho0)) */
    const T arg     = p.gamma_inv_cp * Sg.v + p.gamma_m1 * (L.v - p.lnrho0);
    const T E       = ac_exp(arg);
    const T cs2     = p.cs2_sound * E;
    const T inv_rho = ac_exp(-L.v);
    const T inv_T   = p.inv_exp_lnT0 * ac_rcp(E);

    /* traceless rate of strain */
    const T third = (T)(1.0 / 3.0);
    const T S00   = (T)(2.0 / 3.0) * U.g[0][0] - third * (U.g[1][1] + U.g[2][2]);
    const T S11   = (T)(2.0 / 3.0) * U.g[1][1] - third * (U.g[0][0] + U.g[2][2]);
    const T S22   = (T)(2.0 / 3.0) * U.g[2][2] - third * (U.g[0][0] + U.g[1][1]);
    const T S01   = (T)0.5 * (U.g[0][1] + U.g[1][0]);
    const T S02   = (T)0.5 * (U.g[0][2] + U.g[2][0]);
    const T S12   = (T)0.5 * (U.g[1][2] + U.g[2][1]);

    /* momentum */
    {
        const T jxBx = jy * Bz - jz * By;
        const T jxBy = jz * Bx - jx * Bz;
        const T jxBz = jx * By - jy * Bx;
        const T px   = p.inv_cp * Sg.g[0] + L.g[0];
        const T py   = p.inv_cp * Sg.g[1] + L.g[1];
        const T pz   = p.inv_cp * Sg.g[2] + L.g[2];
        const T SLx  = S00 * L.g[0] + S01 * L.g[1] + S02 * L.g[2];
        const T SLy  = S01 * L.g[0] + S11 * L.g[1] + S12 * L.g[2];
        const T SLz  = S02 * L.g[0] + S12 * L.g[1] + S22 * L.g[2];
        const T advx = U.g[0][0] * ux + U.g[0][1] * uy + U.g[0][2] * uz;
        const T advy = U.g[1][0] * ux + U.g[1][1] * uy + U.g[1][2] * uz;
        const T advz = U.g[2][0] * ux + U.g[2][1] * uy + U.g[2][2] * uz;
        r[1] = -advx - cs2 * px + inv_rho * jxBx +
               p.nu * (U.lap[0] + (T)2 * SLx) + p.visc_gd * U.gd[0];
        r[2] = -advy - cs2 * py + inv_rho * jxBy +
               p.nu * (U.lap[1] + (T)2 * SLy) + p.visc_gd * U.gd[1];
        r[3] = -advz - cs2 * pz + inv_rho * jxBz +
               p.nu * (U.lap[2] + (T)2 * SLz) + p.visc_gd * U.gd[2];
    }

    /* entropy */
    {
        const T SS = S00 * S00 + S11 * S11 + S22 * S22 +
                     (T)2 * (S01 * S01 + S02 * S02 + S12 * S12);
        const T jj = jx * jx + jy * jy + jz * jz;
        /* (rho T)^-1 (eta mu0 j.j + 2 rho nu S:S + zeta rho divu^2) */
        const T heating = inv_T * (inv_rho * p.eta_mu0 * jj + (T)2 * p.nu * SS +
                                   p.zeta * divu * divu);
        /* heat conduction: K/rho (first + second.third); the reference's
         * third term gamma (grad s/cp + grad lnrho) - grad lnrho equals its
         * second term, so the dot product is a square. */
        const T first = p.gamma_inv_cp * Sg.lap + p.gamma_m1 * L.lap;
        T dot2        = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const T second = p.gamma_inv_cp * Sg.g[a] + p.gamma_m1 * L.g[a];
            dot2 += second * second;
        }
        const T heat = p.K * inv_rho * (first + dot2);
        r[7] = -(ux * Sg.g[0] + uy * Sg.g[1] + uz * Sg.g[2]) + heating + heat;
    }
}
