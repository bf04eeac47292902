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

/* The RHS is evaluated in two halves so that two warp groups can share one
 * cell: the hydro half owns lnrho and uu (continuity, momentum), the magnetic
 * half owns aa and entropy (induction, entropy).  Each half first prepares
 * the values the other needs, the two exchange them, then each finishes its
 * four rates.  mhd_rates() runs both halves in one thread, so split and
 * unsplit kernels evaluate the same expressions. */
/* Exchange records as flat arrays (registers, and one shared-memory row per
 * entry when two warp groups share a cell). */
enum {
    H2M_U   = 0, /* u[3] */
    H2M_GL  = 3, /* grad lnrho[3] */
    H2M_LAPL = 6,
    H2M_SS   = 7, /* S:S */
    H2M_DIVU = 8,
    H2M_E    = 9, /* exp(gamma s/cp + (gamma-1)(lnrho - lnrho0)) */
    H2M_INV_RHO = 10, /* exp(-lnrho) */
    AC_H2M_COUNT = 11
};
enum {
    M2H_GS = 0, /* grad s[3] */
    M2H_J  = 3, /* current density[3] */
    M2H_B  = 6, /* magnetic field[3] */
    AC_M2H_COUNT = 9
};

template <typename T>
struct HydroToMag {
    T a[AC_H2M_COUNT];
};

template <typename T>
struct MagToHydro {
    T a[AC_M2H_COUNT];
};

template <typename T>
struct Strain {
    T S00, S11, S22, S01, S02, S12;
};

template <typename T>
__device__ __forceinline__ void
hydro_prepare(const ScalD<T>& L, const T s_value, const VecD<T>& U, const PhysT<T>& p,
              HydroToMag<T>& x, Strain<T>& S)
{
    const T third     = (T)(1.0 / 3.0);
    x.a[H2M_DIVU]     = U.g[0][0] + U.g[1][1] + U.g[2][2];
    S.S00 = (T)(2.0 / 3.0) * U.g[0][0] - third * (U.g[1][1] + U.g[2][2]);
    S.S11 = (T)(2.0 / 3.0) * U.g[1][1] - third * (U.g[0][0] + U.g[2][2]);
    S.S22 = (T)(2.0 / 3.0) * U.g[2][2] - third * (U.g[0][0] + U.g[1][1]);
    S.S01 = (T)0.5 * (U.g[0][1] + U.g[1][0]);
    S.S02 = (T)0.5 * (U.g[0][2] + U.g[2][0]);
    S.S12 = (T)0.5 * (U.g[1][2] + U.g[2][1]);
    x.a[H2M_SS] = S.S00 * S.S00 + S.S11 * S.S11 + S.S22 * S.S22 +
                  (T)2 * (S.S01 * S.S01 + S.S02 * S.S02 + S.S12 * S.S12);
    const T arg      = p.gamma_inv_cp * s_value + p.gamma_m1 * (L.v - p.lnrho0);
    x.a[H2M_E]       = ac_exp(arg);
    x.a[H2M_INV_RHO] = ac_exp(-L.v);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        x.a[H2M_U + a]  = U.v[a];
        x.a[H2M_GL + a] = L.g[a];
    }
    x.a[H2M_LAPL] = L.lap;
}

/* hydro_prepare with the two exponentials (H2M_E and H2M_INV_RHO, the same
 * expressions) formed beforehand */
template <typename T>
__device__ __forceinline__ void
hydro_prepare_exp(const ScalD<T>& L, const VecD<T>& U, const T e, const T inv_rho,
                  HydroToMag<T>& x, Strain<T>& S)
{
    const T third     = (T)(1.0 / 3.0);
    x.a[H2M_DIVU]     = U.g[0][0] + U.g[1][1] + U.g[2][2];
    S.S00 = (T)(2.0 / 3.0) * U.g[0][0] - third * (U.g[1][1] + U.g[2][2]);
    S.S11 = (T)(2.0 / 3.0) * U.g[1][1] - third * (U.g[0][0] + U.g[2][2]);
    S.S22 = (T)(2.0 / 3.0) * U.g[2][2] - third * (U.g[0][0] + U.g[1][1]);
    S.S01 = (T)0.5 * (U.g[0][1] + U.g[1][0]);
    S.S02 = (T)0.5 * (U.g[0][2] + U.g[2][0]);
    S.S12 = (T)0.5 * (U.g[1][2] + U.g[2][1]);
    x.a[H2M_SS] = S.S00 * S.S00 + S.S11 * S.S11 + S.S22 * S.S22 +
                  (T)2 * (S.S01 * S.S01 + S.S02 * S.S02 + S.S12 * S.S12);
    x.a[H2M_E]       = e;
    x.a[H2M_INV_RHO] = inv_rho;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        x.a[H2M_U + a]  = U.v[a];
        x.a[H2M_GL + a] = L.g[a];
    }
    x.a[H2M_LAPL] = L.lap;
}

template <typename T>
__device__ __forceinline__ void
mag_prepare(const ScalD<T>& Sg, const VecD<T>& A, const PhysT<T>& p, MagToHydro<T>& m)
{
    m.a[M2H_B + 0] = A.g[2][1] - A.g[1][2];
    m.a[M2H_B + 1] = A.g[0][2] - A.g[2][0];
    m.a[M2H_B + 2] = A.g[1][0] - A.g[0][1];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        m.a[M2H_J + a]  = (A.gd[a] - A.lap[a]) * p.inv_mu0;
        m.a[M2H_GS + a] = Sg.g[a];
    }
}

/* r[0] = dlnrho/dt, r[1..3] = du/dt */
template <typename T>
__device__ __forceinline__ void
hydro_rates(const ScalD<T>& L, const VecD<T>& U, const Strain<T>& S, const HydroToMag<T>& x,
            const MagToHydro<T>& m, const PhysT<T>& p, T r[4])
{
    const T ux = U.v[0], uy = U.v[1], uz = U.v[2];
    r[0]        = -(ux * L.g[0] + uy * L.g[1] + uz * L.g[2]) - x.a[H2M_DIVU];
    const T cs2 = p.cs2_sound * x.a[H2M_E];
    const T* j  = &m.a[M2H_J];
    const T* B  = &m.a[M2H_B];
    const T jxB[3] = {j[1] * B[2] - j[2] * B[1], j[2] * B[0] - j[0] * B[2],
                      j[0] * B[1] - j[1] * B[0]};
    const T SL[3]  = {S.S00 * L.g[0] + S.S01 * L.g[1] + S.S02 * L.g[2],
                      S.S01 * L.g[0] + S.S11 * L.g[1] + S.S12 * L.g[2],
                      S.S02 * L.g[0] + S.S12 * L.g[1] + S.S22 * L.g[2]};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const T adv = U.g[c][0] * ux + U.g[c][1] * uy + U.g[c][2] * uz;
        const T pg  = p.inv_cp * m.a[M2H_GS + c] + L.g[c];
        r[1 + c]    = -adv - cs2 * pg + x.a[H2M_INV_RHO] * jxB[c] +
                   p.nu * (U.lap[c] + (T)2 * SL[c]) + p.visc_gd * U.gd[c];
    }
}

/* r[0..2] = dA/dt, r[3] = ds/dt */
template <typename T>
__device__ __forceinline__ void
mag_rates(const ScalD<T>& Sg, const VecD<T>& A, const MagToHydro<T>& m, const HydroToMag<T>& x,
          const PhysT<T>& p, T r[4])
{
    const T ux = x.a[H2M_U], uy = x.a[H2M_U + 1], uz = x.a[H2M_U + 2];
    const T* B = &m.a[M2H_B];
    const T* j = &m.a[M2H_J];
    /* induction: u x B + eta lap A */
    r[0] = (uy * B[2] - uz * B[1]) + p.eta * A.lap[0];
    r[1] = (uz * B[0] - ux * B[2]) + p.eta * A.lap[1];
    r[2] = (ux * B[1] - uy * B[0]) + p.eta * A.lap[2];
    /* entropy: (rho T)^-1 (eta mu0 j.j + 2 rho nu S:S + zeta rho divu^2) + heat */
    const T inv_rho = x.a[H2M_INV_RHO];
    const T divu    = x.a[H2M_DIVU];
    const T inv_T   = p.inv_exp_lnT0 * ac_rcp(x.a[H2M_E]);
    const T jj      = j[0] * j[0] + j[1] * j[1] + j[2] * j[2];
    const T heating = inv_T * (inv_rho * p.eta_mu0 * jj + (T)2 * p.nu * x.a[H2M_SS] +
                               p.zeta * divu * divu);
    /* heat conduction: K/rho (first + second.third); the reference's third term
     * gamma (grad s/cp + grad lnrho) - grad lnrho equals its second term */
    const T first = p.gamma_inv_cp * Sg.lap + p.gamma_m1 * x.a[H2M_LAPL];
    T dot2        = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const T second = p.gamma_inv_cp * Sg.g[a] + p.gamma_m1 * x.a[H2M_GL + a];
        dot2 += second * second;
    }
    const T heat = p.K * inv_rho * (first + dot2);
    r[3]         = -(ux * Sg.g[0] + uy * Sg.g[1] + uz * Sg.g[2]) + heating + heat;
}

/* The upwinding terms (the reference's LUPWD option, mhdsolver.ac:336-338,
 * 357-359; model src/utils/modelsolver.cc:776-779,837-841) added to the
 * hydro rates: r[0] += |u| . upwd(lnrho), r[1 + c] += upwd(u_c) . |u|.
 * up_l[a] and up_u[c][a] are the upwinding derivatives along axis a. */
template <typename T>
__device__ __forceinline__ void
upwind_terms(const T up_l[3], const T up_u[3][3], const T u[3], T add[4])
{
    const T au[3] = {fabs(u[0]), fabs(u[1]), fabs(u[2])};
    add[0]        = au[0] * up_l[0] + au[1] * up_l[1] + au[2] * up_l[2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
        add[1 + c] = up_u[c][0] * au[0] + up_u[c][1] * au[1] + up_u[c][2] * au[2];
}

/* Helical forcing added to u in substep 2 at interior cell (i, j, k): the
 * reference's forcing()/helical_forcing() (mhdsolver.ac:286-331; model
 * src/utils/modelsolver.cc:1003-1076), with the phase angle k . (2 pi x / L)
 * and scale sqrt(dt) cs magnitude sqrt(kaver cs) precomputed on the host. */
template <typename T>
__device__ __forceinline__ void
forcing_at(const PhysConst& pc, const int i, const int j, const int k, T f[3])
{
    const double a = pc.f_k[0] * i + pc.f_k[1] * j + pc.f_k[2] * k;
    double sa, ca;
    sincos(a, &sa, &ca);
    const double re = ca * pc.f_cos_phase - sa * pc.f_sin_phase;
    const double im = ca * pc.f_sin_phase + sa * pc.f_cos_phase;
#pragma unroll
    for (int c = 0; c < 3; ++c)
        f[c] = (T)(pc.f_scale * (pc.f_re[c] * re - pc.f_im[c] * im));
}

/* (h, l) += v for a compensated FP32 pair, renormalised (two-sum) */
__device__ __forceinline__ void
comp_add(float& h, float& l, const float v)
{
    const float s  = __fadd_rn(h, v);
    const float bb = __fsub_rn(s, h);
    const float e  = __fadd_rn(__fsub_rn(h, __fsub_rn(s, bb)), __fsub_rn(v, bb));
    const float l2 = __fadd_rn(l, e);
    h              = __fadd_rn(s, l2);
    l              = __fsub_rn(l2, __fsub_rn(h, s));
}

/* rates[8] in field order (lnrho, ux, uy, uz, ax, ay, az, entropy). */
template <typename T>
__device__ __forceinline__ void
mhd_rates(const ScalD<T>& L, const ScalD<T>& Sg, const VecD<T>& U, const VecD<T>& A,
          const PhysT<T>& p, T r[AC_NF])
{
    HydroToMag<T> x;
    Strain<T> S;
    MagToHydro<T> m;
    hydro_prepare(L, Sg.v, U, p, x, S);
    mag_prepare(Sg, A, p, m);
    T rh[4], rm[4];
    hydro_rates(L, U, S, x, m, p, rh);
    mag_rates(Sg, A, m, x, p, rm);
    r[0] = rh[0];
    r[1] = rh[1];
    r[2] = rh[2];
    r[3] = rh[3];
    r[4] = rm[0];
    r[5] = rm[1];
    r[6] = rm[2];
    r[7] = rm[3];
}

/* Single-pass 2N RK3 update of one value (acc-runtime/stdlib/integrators.h:16-29):
 *   f_new = f + beta (ab (f - f_prev) + dt rate)
 * FP64: plain arithmetic.  FP32 compensated: f = (h, l) with |l| <= ulp(h)/2;
 * the increment is formed in FP32 (it is small against f) and added with an
 * error-free two-sum, so the accumulated state keeps ~48 significant bits. */
struct RkT64 {
    double dt, beta, ab;
};
struct RkT32 {
    float dt, beta, ab;
};

__device__ __forceinline__ void
rk_update(const double f, const double f_prev, const double rate, const RkT64& c,
          const bool use_prev, double& out)
{
    double upd = c.dt * rate;
    if (use_prev)
        upd = fma(c.ab, f - f_prev, upd);
    out = fma(c.beta, upd, f);
}

__device__ __forceinline__ void
rk_update_comp(const float h, const float l, const float ph, const float pl, const float rate,
               const RkT32& c, const bool use_prev, float& oh, float& ol)
{
    float upd = c.dt * rate;
    if (use_prev) {
        const float d = (h - ph) + (l - pl);
        upd           = fmaf(c.ab, d, upd);
    }
    const float inc = c.beta * upd;
    /* two-sum (h, inc) -> (s, e), then fold in l and renormalise */
    const float s  = __fadd_rn(h, inc);
    const float bb = __fsub_rn(s, h);
    const float e  = __fadd_rn(__fsub_rn(h, __fsub_rn(s, bb)), __fsub_rn(inc, bb));
    const float l2 = __fadd_rn(l, e);
    oh             = __fadd_rn(s, l2);
    ol             = __fsub_rn(l2, __fsub_rn(oh, s));
}

/* Per-cell quantities of calc_timestep (acc-runtime/samples/mhd_modular/mhdsolver.ac:551-583):
 * |u| and the Alfven speed sqrt(|B|^2 / rho) for the maximum form, and, with
 * `with_sum` (the additive form, AC_additive_timestep), |u| + sqrt(cs_sound^2 + vA^2),
 * folded into running maxima m[3]; the reference evaluates only the form its
 * AC_additive_timestep selects.  m[0] and m[1] hold the maxima of the squares
 * (|u|^2, vA^2): sqrt is correctly rounded and monotone, so cfl_commit's sqrt
 * of the maximum is the maximum of the square roots, bit for bit.  In FP64 the
 * sum is formed only where a single-precision estimate of it reaches within
 * 1e-5 of the running maximum (the estimate's error is below 3e-7 relative), so
 * the result is the same as evaluating it at every cell. */
template <typename T>
__device__ __forceinline__ void
cfl_accumulate(const T u2, const T b2, const T inv_rho, const T cs2_sound, T m[3],
               const bool with_sum = true)
{
    const T va2 = b2 * inv_rho;
    m[0]        = fmax(m[0], u2);
    m[1]        = fmax(m[1], va2);
    if (!with_sum)
        return;
    if constexpr (sizeof(T) == 8) {
        const float est = __fsqrt_rn((float)u2) + __fsqrt_rn((float)(cs2_sound + va2));
        if (est >= (float)m[2] * 0.99999f)
            m[2] = fmax(m[2], sqrt(u2) + sqrt(cs2_sound + va2));
    }
    else {
        m[2] = fmax(m[2], sqrt(u2) + sqrt(cs2_sound + va2));
    }
}

/* Block-wide max of m[3] across all threads, then one atomicMax per value on
 * the device words (non-negative doubles order like their bit patterns).
 * Every thread of the block must call this; red holds 3 * warps entries. */
template <typename T>
__device__ __forceinline__ void
cfl_commit(T m[3], T* red, unsigned long long* cfl)
{
    const int lane = threadIdx.x & 31;
    const int nthreads = blockDim.x * blockDim.y;
    const int tid      = threadIdx.y * blockDim.x + threadIdx.x;
    const int warp     = tid >> 5;
    m[0]               = sqrt(m[0]); /* cfl_accumulate keeps the squares of these two */
    m[1]               = sqrt(m[1]);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            m[i] = fmax(m[i], __shfl_xor_sync(0xffffffffu, m[i], o));
    if (lane == 0)
        for (int i = 0; i < 3; ++i)
            red[3 * warp + i] = m[i];
    __syncthreads();
    if (tid == 0) {
        for (int i = 0; i < 3; ++i) {
            T v = red[i];
            for (int w = 1; w < nthreads / 32; ++w)
                v = fmax(v, red[3 * w + i]);
            atomicMax(cfl + i, (unsigned long long)__double_as_longlong((double)v));
        }
    }
}
