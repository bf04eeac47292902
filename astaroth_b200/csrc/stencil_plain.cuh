/*
 * Stencils read straight from global memory (one __ldg per tap), for the
 * kernels that work cell by cell: the plain solve kernel, the adjoint kernels
 * and the CFL kernel.  6th-order central differences of
 * acc-runtime/stdlib/derivs.h:374-427,591-690 (host model
 * src/utils/modelsolver.cc:190-299): first, second and diagonal mixed
 * derivatives, with the grid spacing folded into the coefficients.
 */
#pragma once

#include "internal.h"
#include "mhd_rhs.cuh"

namespace {

template <typename T>
__device__ __forceinline__ T
ld(const T* p)
{
    return __ldg(p);
}

/* sum_k c_k (f[+ks] - f[-ks]) */
template <typename T>
__device__ __forceinline__ T
der1(const T* f, const long long s, const T* c)
{
    T r = c[0] * (ld(f + s) - ld(f - s));
    r   = fma(c[1], ld(f + 2 * s) - ld(f - 2 * s), r);
    r   = fma(c[2], ld(f + 3 * s) - ld(f - 3 * s), r);
    return r;
}

/* sum_k d_k (f[+ks] + f[-ks]), k = 1..3 (centre term excluded) */
template <typename T>
__device__ __forceinline__ T
der2_sides(const T* f, const long long s, const T* d)
{
    T r = d[1] * (ld(f + s) + ld(f - s));
    r   = fma(d[2], ld(f + 2 * s) + ld(f - 2 * s), r);
    r   = fma(d[3], ld(f + 3 * s) + ld(f - 3 * s), r);
    return r;
}

/* upwinding derivative: u_0 f + sum_k u_k (f[+ks] + f[-ks]), k = 1..3 */
template <typename T>
__device__ __forceinline__ T
der_up(const T* f, const long long s, const T* u)
{
    T r = u[0] * ld(f);
    r   = fma(u[1], ld(f + s) + ld(f - s), r);
    r   = fma(u[2], ld(f + 2 * s) + ld(f - 2 * s), r);
    r   = fma(u[3], ld(f + 3 * s) + ld(f - 3 * s), r);
    return r;
}

/* sum_k e_k (f(+k,+k) + f(-k,-k) - f(+k,-k) - f(-k,+k)) along strides a, b */
template <typename T>
__device__ __forceinline__ T
dermix(const T* f, const long long a, const long long b, const T* e)
{
    T r = 0;
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
        const T t = (ld(f + k * a + k * b) + ld(f - k * a - k * b)) -
                    (ld(f + k * a - k * b) + ld(f - k * a + k * b));
        r = k == 1 ? e[0] * t : fma(e[k - 1], t, r);
    }
    return r;
}

template <typename T>
__device__ __forceinline__ void
scal_derivs(const T* f, const long long* st, const StencilT<T>& sc, ScalD<T>& o)
{
    o.v = ld(f);
#pragma unroll
    for (int a = 0; a < 3; ++a)
        o.g[a] = der1(f, st[a], sc.d1[a]);
    T lap = (sc.d2[0][0] + sc.d2[1][0] + sc.d2[2][0]) * o.v;
#pragma unroll
    for (int a = 0; a < 3; ++a)
        lap += der2_sides(f, st[a], sc.d2[a]);
    o.lap = lap;
}

template <typename T>
__device__ __forceinline__ void
vec_derivs(const T* const* fc, const long long* st, const StencilT<T>& sc, VecD<T>& o)
{
    T diag[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const T* f = fc[c];
        o.v[c]     = ld(f);
#pragma unroll
        for (int a = 0; a < 3; ++a)
            o.g[c][a] = der1(f, st[a], sc.d1[a]);
        T side[3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
            side[a] = der2_sides(f, st[a], sc.d2[a]);
        diag[c]  = sc.d2[c][0] * o.v[c] + side[c];
        o.lap[c] = (sc.d2[0][0] + sc.d2[1][0] + sc.d2[2][0]) * o.v[c] + side[0] + side[1] +
                   side[2];
    }
    /* grad div: d_xx v_x + d_xy v_y + d_xz v_z, ... */
    const T mxy_y = dermix(fc[1], st[0], st[1], sc.mix[0]); /* d_xy v_y */
    const T mxz_z = dermix(fc[2], st[0], st[2], sc.mix[1]); /* d_xz v_z */
    const T mxy_x = dermix(fc[0], st[0], st[1], sc.mix[0]); /* d_xy v_x */
    const T myz_z = dermix(fc[2], st[1], st[2], sc.mix[2]); /* d_yz v_z */
    const T mxz_x = dermix(fc[0], st[0], st[2], sc.mix[1]); /* d_xz v_x */
    const T myz_y = dermix(fc[1], st[1], st[2], sc.mix[2]); /* d_yz v_y */
    o.gd[0]       = diag[0] + mxy_y + mxz_z;
    o.gd[1]       = mxy_x + diag[1] + myz_z;
    o.gd[2]       = mxz_x + myz_y + diag[2];
}


} // namespace
