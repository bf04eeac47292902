/*
 * The MHD substep kernels (FP64): 6th-order stencils + RHS + the 2N RK3
 * update in single-pass form, one launch per substep.
 *
 * Reference: twopass_solve_intermediate/final and singlepass_solve,
 * acc-runtime/samples/mhd_modular/mhdsolver.ac:524-636, with the stencils of
 * acc-runtime/stdlib/derivs.h:374-427,591-690 (host model
 * src/utils/modelsolver.cc:190-299) and rk3() of
 * acc-runtime/stdlib/integrators.h:11-29.
 *
 * variant 0 ("plain"): one thread per cell, every tap an __ldg through L1.
 * It is the simple correctness baseline the tiled kernel is checked against.
 */
#include "internal.h"
#include "mhd_rhs.cuh"

namespace {

__device__ __forceinline__ double
ld(const double* p)
{
    return __ldg(p);
}

/* sum_k c_k (f[+ks] - f[-ks]) */
__device__ __forceinline__ double
der1(const double* f, const long long s, const double* c)
{
    double r = c[0] * (ld(f + s) - ld(f - s));
    r        = fma(c[1], ld(f + 2 * s) - ld(f - 2 * s), r);
    r        = fma(c[2], ld(f + 3 * s) - ld(f - 3 * s), r);
    return r;
}

/* sum_k d_k (f[+ks] + f[-ks]), k = 1..3 (centre term excluded) */
__device__ __forceinline__ double
der2_sides(const double* f, const long long s, const double* d)
{
    double r = d[1] * (ld(f + s) + ld(f - s));
    r        = fma(d[2], ld(f + 2 * s) + ld(f - 2 * s), r);
    r        = fma(d[3], ld(f + 3 * s) + ld(f - 3 * s), r);
    return r;
}

/* sum_k e_k (f(+k,+k) + f(-k,-k) - f(+k,-k) - f(-k,+k)) along strides a, b */
__device__ __forceinline__ double
dermix(const double* f, const long long a, const long long b, const double* e)
{
    double r = 0;
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
        const double t = (ld(f + k * a + k * b) + ld(f - k * a - k * b)) -
                         (ld(f + k * a - k * b) + ld(f - k * a + k * b));
        r = k == 1 ? e[0] * t : fma(e[k - 1], t, r);
    }
    return r;
}

__device__ __forceinline__ void
scal_derivs(const double* f, const long long* st, const StencilCoef& sc, ScalD<double>& o)
{
    o.v = ld(f);
#pragma unroll
    for (int a = 0; a < 3; ++a)
        o.g[a] = der1(f, st[a], sc.d1[a]);
    double lap = (sc.d2[0][0] + sc.d2[1][0] + sc.d2[2][0]) * o.v;
#pragma unroll
    for (int a = 0; a < 3; ++a)
        lap += der2_sides(f, st[a], sc.d2[a]);
    o.lap = lap;
}

__device__ __forceinline__ void
vec_derivs(const double* const* fc, const long long* st, const StencilCoef& sc,
           VecD<double>& o)
{
    double diag[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double* f = fc[c];
        o.v[c]          = ld(f);
#pragma unroll
        for (int a = 0; a < 3; ++a)
            o.g[c][a] = der1(f, st[a], sc.d1[a]);
        double side[3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
            side[a] = der2_sides(f, st[a], sc.d2[a]);
        diag[c]  = sc.d2[c][0] * o.v[c] + side[c];
        o.lap[c] = (sc.d2[0][0] + sc.d2[1][0] + sc.d2[2][0]) * o.v[c] + side[0] + side[1] +
                   side[2];
    }
    /* grad div: d_xx v_x + d_xy v_y + d_xz v_z, ... */
    const double mxy_y = dermix(fc[1], st[0], st[1], sc.mix[0]); /* d_xy v_y */
    const double mxz_z = dermix(fc[2], st[0], st[2], sc.mix[1]); /* d_xz v_z */
    const double mxy_x = dermix(fc[0], st[0], st[1], sc.mix[0]); /* d_xy v_x */
    const double myz_z = dermix(fc[2], st[1], st[2], sc.mix[2]); /* d_yz v_z */
    const double mxz_x = dermix(fc[0], st[0], st[2], sc.mix[1]); /* d_xz v_x */
    const double myz_y = dermix(fc[1], st[1], st[2], sc.mix[2]); /* d_yz v_y */
    o.gd[0]            = diag[0] + mxy_y + mxz_z;
    o.gd[1]            = mxy_x + diag[1] + myz_z;
    o.gd[2]            = mxz_x + myz_y + diag[2];
}

__global__ void __launch_bounds__(128)
solve_plain_kernel(const Geom g, const Fields64 f, const StencilCoef sc, const PhysConst pc,
                   const RkCoef rk)
{
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    const int j = threadIdx.y + blockIdx.y * blockDim.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k >= g.nz)
        return;
    const long long idx = (long long)(i + NGHOST) + (long long)(j + NGHOST) * g.mx +
                          (long long)(k + NGHOST) * g.mxy;
    const long long st[3] = {1, (long long)g.mx, g.mxy};
    /* previous-substep values, loaded before any store so the loads overlap */
    double prev[AC_NF];
#pragma unroll
    for (int q = 0; q < AC_NF; ++q)
        prev[q] = rk.step > 0 ? f.out[q][idx] : 0.0;

    ScalD<double> L, S;
    VecD<double> U, A;
    scal_derivs(f.in[VTXBUF_LNRHO] + idx, st, sc, L);
    scal_derivs(f.in[VTXBUF_ENTROPY] + idx, st, sc, S);
    {
        const double* uc[3] = {f.in[VTXBUF_UUX] + idx, f.in[VTXBUF_UUY] + idx,
                               f.in[VTXBUF_UUZ] + idx};
        vec_derivs(uc, st, sc, U);
        const double* ac[3] = {f.in[VTXBUF_AX] + idx, f.in[VTXBUF_AY] + idx,
                               f.in[VTXBUF_AZ] + idx};
        vec_derivs(ac, st, sc, A);
    }
    const PhysT<double> p = phys_cast<double>(pc);
    double r[AC_NF];
    mhd_rates(L, S, U, A, p, r);

    const double val[AC_NF] = {L.v, U.v[0], U.v[1], U.v[2], A.v[0], A.v[1], A.v[2], S.v};
#pragma unroll
    for (int q = 0; q < AC_NF; ++q) {
        const double fv = val[q];
        double upd      = rk.dt * r[q];
        if (rk.step > 0)
            upd = fma(rk.ab, fv - prev[q], upd);
        f.out[q][idx] = fma(rk.beta, upd, fv);
    }
}

} // namespace

cudaError_t
ac_launch_solve64(const Geom& g, const Fields64& f, const StencilCoef& sc, const PhysConst& pc,
                  const RkCoef& rk, const int variant, cudaStream_t stream,
                  unsigned long long* launches)
{
    (void)variant;
    const dim3 tpb(32, 4, 1);
    const dim3 bpg((g.nx + tpb.x - 1) / tpb.x, (g.ny + tpb.y - 1) / tpb.y, g.nz);
    solve_plain_kernel<<<bpg, tpb, 0, stream>>>(g, f, sc, pc, rk);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}
