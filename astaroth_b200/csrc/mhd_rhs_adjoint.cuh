/*
 * Reverse mode (vector-Jacobian product) of the per-cell MHD right-hand side of
 * mhd_rhs.cuh, written by hand.  Given the cell's derivative records (value,
 * gradient, Laplacian, grad div of each field) and an adjoint lam[8] of the
 * eight rates, it returns the adjoint of every derivative slot (mu, 46 values)
 * and the cell's contribution to d(lam . r)/d nu and d(lam . r)/d eta.
 *
 * The slots then go through the transposed stencils (adjoint.cu).  The forward
 * expressions are recomputed here in the same form as hydro_prepare,
 * mag_prepare, hydro_rates and mag_rates; each backward line names the forward
 * line it differentiates.
 */
#pragma once

#include "mhd_rhs.cuh"

/* Slot layout of mu: per scalar field (lnrho, entropy) v, g[3], lap; per
 * vector field (uu, aa) v[3], g[3][3] (row c = component), lap[3], gd[3]. */
enum {
    MU_L = 0,  /* lnrho: 0 v, 1..3 g, 4 lap */
    MU_S = 5,  /* entropy */
    MU_U = 10, /* uu: +0..2 v, +3..11 g, +12..14 lap, +15..17 gd */
    MU_A = 28, /* aa */
    MU_COUNT = 46
};
#define MU_SV 0
#define MU_SG 1
#define MU_SLAP 4
#define MU_VV 0
#define MU_VG 3
#define MU_VLAP 12
#define MU_VGD 15

template <typename T>
__device__ __forceinline__ void
mhd_rates_adjoint(const ScalD<T>& L, const ScalD<T>& Sg, const VecD<T>& U, const VecD<T>& A,
                  const PhysT<T>& p, const T lam[AC_NF], T mu[MU_COUNT], T& dnu, T& deta)
{
    /* ---- forward intermediates (hydro_prepare, mag_prepare) ---- */
    const T* u  = U.v;
    const T* gl = L.g;
    const T* gs = Sg.g;
    const T third = (T)(1.0 / 3.0);
    const T divu  = U.g[0][0] + U.g[1][1] + U.g[2][2];
    T S[3][3];
    S[0][0] = (T)(2.0 / 3.0) * U.g[0][0] - third * (U.g[1][1] + U.g[2][2]);
    S[1][1] = (T)(2.0 / 3.0) * U.g[1][1] - third * (U.g[0][0] + U.g[2][2]);
    S[2][2] = (T)(2.0 / 3.0) * U.g[2][2] - third * (U.g[0][0] + U.g[1][1]);
    S[0][1] = S[1][0] = (T)0.5 * (U.g[0][1] + U.g[1][0]);
    S[0][2] = S[2][0] = (T)0.5 * (U.g[0][2] + U.g[2][0]);
    S[1][2] = S[2][1] = (T)0.5 * (U.g[1][2] + U.g[2][1]);
    /* SS = S00^2 + S11^2 + S22^2 + 2(S01^2 + S02^2 + S12^2) = sum over all nine entries */
    T SS = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a)
            SS += S[c][a] * S[c][a];
    const T arg     = p.gamma_inv_cp * Sg.v + p.gamma_m1 * (L.v - p.lnrho0);
    const T E       = ac_exp(arg);
    const T inv_rho = ac_exp(-L.v);
    const T B[3]    = {A.g[2][1] - A.g[1][2], A.g[0][2] - A.g[2][0], A.g[1][0] - A.g[0][1]};
    const T j[3]    = {(A.gd[0] - A.lap[0]) * p.inv_mu0, (A.gd[1] - A.lap[1]) * p.inv_mu0,
                    (A.gd[2] - A.lap[2]) * p.inv_mu0};
    /* hydro_rates / mag_rates intermediates */
    const T cs2    = p.cs2_sound * E;
    const T jxB[3] = {j[1] * B[2] - j[2] * B[1], j[2] * B[0] - j[0] * B[2],
                      j[0] * B[1] - j[1] * B[0]};
    T SL[3], pg[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        SL[c] = S[c][0] * gl[0] + S[c][1] * gl[1] + S[c][2] * gl[2];
        pg[c] = p.inv_cp * gs[c] + gl[c];
    }
    const T inv_T = p.inv_exp_lnT0 * ac_rcp(E);
    const T jj    = j[0] * j[0] + j[1] * j[1] + j[2] * j[2];
    const T H     = inv_rho * p.eta_mu0 * jj + (T)2 * p.nu * SS + p.zeta * divu * divu;
    const T first = p.gamma_inv_cp * Sg.lap + p.gamma_m1 * L.lap;
    T second[3], dot2 = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        second[a] = p.gamma_inv_cp * gs[a] + p.gamma_m1 * gl[a];
        dot2 += second[a] * second[a];
    }

    /* ---- adjoints ---- */
    const T l0    = lam[0];
    const T lu[3] = {lam[1], lam[2], lam[3]};
    const T la[3] = {lam[4], lam[5], lam[6]};
    const T ls    = lam[7];
    T ub[3] = {0, 0, 0}, glb[3] = {0, 0, 0}, gsb[3] = {0, 0, 0}, Bb[3] = {0, 0, 0},
      jb[3] = {0, 0, 0};
    T Ugb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Sb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    T Agb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    T Ulapb[3] = {0, 0, 0}, Ugdb[3] = {0, 0, 0}, Alapb[3] = {0, 0, 0}, Agdb[3] = {0, 0, 0};
    T divub = 0, SSb = 0, Eb = 0, invrhob = 0, Slapb = 0, Llapb = 0, Lvb = 0, Svb = 0;

    /* r7 = -(u . gs) + heating + heat */
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        ub[a] -= ls * gs[a];
        gsb[a] -= ls * u[a];
    }
    /* heat = K inv_rho (first + dot2) */
    invrhob += ls * p.K * (first + dot2);
    const T fb = ls * p.K * inv_rho;
    Slapb += p.gamma_inv_cp * fb; /* first = gamma/cp lap s + (gamma-1) lap lnrho */
    Llapb += p.gamma_m1 * fb;
#pragma unroll
    for (int a = 0; a < 3; ++a) { /* dot2 = sum second^2, second = gamma/cp gs + (gamma-1) gl */
        const T sb = (T)2 * second[a] * fb;
        gsb[a] += p.gamma_inv_cp * sb;
        glb[a] += p.gamma_m1 * sb;
    }
    /* heating = inv_T H, H = inv_rho eta mu0 jj + 2 nu SS + zeta divu^2 */
    const T invTb = ls * H;
    const T Hb    = ls * inv_T;
    invrhob += Hb * p.eta_mu0 * jj;
    const T jjb = Hb * p.eta_mu0 * inv_rho;
    SSb += Hb * (T)2 * p.nu;
    divub += Hb * (T)2 * p.zeta * divu;
    Eb -= invTb * inv_T * ac_rcp(E); /* inv_T = exp(-lnT0) / E */
#pragma unroll
    for (int a = 0; a < 3; ++a) /* jj = j . j */
        jb[a] += (T)2 * j[a] * jjb;

    /* r[4+c] = (u x B)_c + eta lap A_c:  lam . (u x B) = u . (B x lam) = B . (lam x u) */
    ub[0] += B[1] * la[2] - B[2] * la[1];
    ub[1] += B[2] * la[0] - B[0] * la[2];
    ub[2] += B[0] * la[1] - B[1] * la[0];
    Bb[0] += la[1] * u[2] - la[2] * u[1];
    Bb[1] += la[2] * u[0] - la[0] * u[2];
    Bb[2] += la[0] * u[1] - la[1] * u[0];
#pragma unroll
    for (int c = 0; c < 3; ++c)
        Alapb[c] += p.eta * la[c];

    /* r[1+c] = -adv_c - cs2 pg_c + inv_rho (j x B)_c + nu (lap u_c + 2 SL_c) + visc_gd gd_c */
    T cs2b = 0, jxBb[3], SLb[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
        for (int a = 0; a < 3; ++a) { /* adv_c = sum_a g[c][a] u_a */
            Ugb[c][a] -= lu[c] * u[a];
            ub[a] -= lu[c] * U.g[c][a];
        }
        cs2b -= lu[c] * pg[c];
        const T pgb = -lu[c] * cs2; /* pg_c = gs_c/cp + gl_c */
        gsb[c] += p.inv_cp * pgb;
        glb[c] += pgb;
        invrhob += lu[c] * jxB[c];
        jxBb[c] = lu[c] * inv_rho;
        Ulapb[c] += p.nu * lu[c];
        SLb[c] = (T)2 * p.nu * lu[c];
        Ugdb[c] += p.visc_gd * lu[c];
    }
    /* jxB = j x B:  jxBb . (j x B) = j . (B x jxBb) = B . (jxBb x j) */
    jb[0] += B[1] * jxBb[2] - B[2] * jxBb[1];
    jb[1] += B[2] * jxBb[0] - B[0] * jxBb[2];
    jb[2] += B[0] * jxBb[1] - B[1] * jxBb[0];
    Bb[0] += jxBb[1] * j[2] - jxBb[2] * j[1];
    Bb[1] += jxBb[2] * j[0] - jxBb[0] * j[2];
    Bb[2] += jxBb[0] * j[1] - jxBb[1] * j[0];
#pragma unroll
    for (int c = 0; c < 3; ++c) /* SL_c = sum_a S[c][a] gl_a */
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            Sb[c][a] += SLb[c] * gl[a];
            glb[a] += SLb[c] * S[c][a];
        }
    Eb += p.cs2_sound * cs2b; /* cs2 = cs_sound^2 E */

    /* r0 = -(u . gl) - divu */
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        ub[a] -= l0 * gl[a];
        glb[a] -= l0 * u[a];
    }
    divub -= l0;

    /* mag_prepare: B = curl A, j = (grad div A - lap A) / mu0 */
    Agb[2][1] += Bb[0];
    Agb[1][2] -= Bb[0];
    Agb[0][2] += Bb[1];
    Agb[2][0] -= Bb[1];
    Agb[1][0] += Bb[2];
    Agb[0][1] -= Bb[2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        Agdb[a] += jb[a] * p.inv_mu0;
        Alapb[a] -= jb[a] * p.inv_mu0;
    }

    /* hydro_prepare */
    Lvb -= inv_rho * invrhob; /* inv_rho = exp(-lnrho) */
    const T argb = E * Eb;    /* E = exp(arg) */
    Svb += p.gamma_inv_cp * argb;
    Lvb += p.gamma_m1 * argb;
#pragma unroll
    for (int c = 0; c < 3; ++c) /* SS = sum of the nine S entries squared */
#pragma unroll
        for (int a = 0; a < 3; ++a)
            Sb[c][a] += (T)2 * S[c][a] * SSb;
    /* S from grad u: diagonal (2/3) g_cc - (1/3) sum_{d != c} g_dd; off-diagonal (g_ca + g_ac)/2 */
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (a == c) {
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    Ugb[d][d] += (d == c ? (T)(2.0 / 3.0) : -third) * Sb[c][c];
            }
            else {
                Ugb[c][a] += (T)0.5 * Sb[c][a];
                Ugb[a][c] += (T)0.5 * Sb[c][a];
            }
        }
#pragma unroll
    for (int c = 0; c < 3; ++c) /* divu = sum g_cc */
        Ugb[c][c] += divub;

    /* ---- slots ---- */
    mu[MU_L + MU_SV]   = Lvb;
    mu[MU_L + MU_SLAP] = Llapb;
    mu[MU_S + MU_SV]   = Svb;
    mu[MU_S + MU_SLAP] = Slapb;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        mu[MU_L + MU_SG + a] = glb[a];
        mu[MU_S + MU_SG + a] = gsb[a];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        mu[MU_U + MU_VV + c]   = ub[c];
        mu[MU_A + MU_VV + c]   = 0; /* the rates depend on A only through its derivatives */
        mu[MU_U + MU_VLAP + c] = Ulapb[c];
        mu[MU_A + MU_VLAP + c] = Alapb[c];
        mu[MU_U + MU_VGD + c]  = Ugdb[c];
        mu[MU_A + MU_VGD + c]  = Agdb[c];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mu[MU_U + MU_VG + 3 * c + a] = Ugb[c][a];
            mu[MU_A + MU_VG + 3 * c + a] = Agb[c][a];
        }
    }

    /* ---- parameters: d(lam . r)/d nu and d/d eta (visc_gd = nu/3 + zeta, eta_mu0 = eta mu0) */
    dnu = ls * inv_T * (T)2 * SS;
    deta = ls * inv_T * inv_rho * jj / p.inv_mu0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        dnu += lu[c] * (U.lap[c] + (T)2 * SL[c] + third * U.gd[c]);
        deta += la[c] * A.lap[c];
    }
}
