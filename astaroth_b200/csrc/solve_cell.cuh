/*
 * One cell of the substep without tiling: every stencil tap an __ldg through
 * L1, the MHD right-hand side and the fused 2N RK3 update, for FP64 and
 * FP32-compensated meshes.  Shared by the plain single-mesh kernel (solve.cu)
 * and the persistent ensemble kernel (ensemble.cu), so both produce the same
 * bits for the same mesh.
 *
 * Reference: singlepass_solve, acc-runtime/samples/mhd_modular/mhdsolver.ac:524-549,
 * with the stencils of acc-runtime/stdlib/derivs.h:374-427,591-690 and rk3()
 * of acc-runtime/stdlib/integrators.h:11-29.
 */
#pragma once

#include "internal.h"
#include "mhd_rhs.cuh"
#include "stencil_plain.cuh"

/* Field arrays given as one base pointer per buffer and a field stride
 * (field q of a block at base + q * stride): the ensemble's layout, which
 * keeps two pointers in registers instead of 32. */
template <typename T>
struct BlockFieldsT {
    const T* in;
    const T* in_lo;
    T* out;
    T* out_lo;
    long long stride;
    __device__ __forceinline__ const T* in_p(const int q) const { return in + q * stride; }
    __device__ __forceinline__ const T* in_lo_p(const int q) const { return in_lo + q * stride; }
    __device__ __forceinline__ T* out_p(const int q) const { return out + q * stride; }
    __device__ __forceinline__ T* out_lo_p(const int q) const { return out_lo + q * stride; }
};

/* FieldsT seen through the same accessors. */
template <typename T>
struct PtrFieldsT {
    const FieldsT<T>& f;
    __device__ __forceinline__ const T* in_p(const int q) const { return f.in[q]; }
    __device__ __forceinline__ const T* in_lo_p(const int q) const { return f.in_lo[q]; }
    __device__ __forceinline__ T* out_p(const int q) const { return f.out[q]; }
    __device__ __forceinline__ T* out_lo_p(const int q) const { return f.out_lo[q]; }
};

/* One cell of the plain kernel; adds the cell's CFL quantities to cm when cfl
 * is set.  F gives the field arrays (BlockFieldsT or PtrFieldsT); UPWD adds
 * the upwinding terms (AC_upwind). */
template <typename T, bool COMP, bool UPWD = false, typename F>
static __device__ __forceinline__ void
plain_cell(const Geom& g, const F& f, const StencilT<T>& sc, const PhysConst& pc,
           const RkCoef& rk, const bool cfl, const int i, const int j, const int k, T cm[3])
{
    const long long idx   = geom_idx(g, i + NGHOST, j + NGHOST, k + NGHOST);
    const long long st[3] = {1, (long long)g.px, g.pxy};
    const bool use_prev   = rk.step > 0;
    /* previous-substep values (and the compensation terms), loaded before any
     * store so the loads overlap */
    T prev[AC_NF], prev_lo[AC_NF], lo[AC_NF];
#pragma unroll
    for (int q = 0; q < AC_NF; ++q) {
        prev[q]    = use_prev ? f.out_p(q)[idx] : T(0);
        prev_lo[q] = (COMP && use_prev) ? f.out_lo_p(q)[idx] : T(0);
        lo[q]      = COMP ? f.in_lo_p(q)[idx] : T(0);
    }

    ScalD<T> L, S;
    VecD<T> U, A;
    scal_derivs(f.in_p(VTXBUF_LNRHO) + idx, st, sc, L);
    scal_derivs(f.in_p(VTXBUF_ENTROPY) + idx, st, sc, S);
    {
        const T* uc[3] = {f.in_p(VTXBUF_UUX) + idx, f.in_p(VTXBUF_UUY) + idx,
                          f.in_p(VTXBUF_UUZ) + idx};
        vec_derivs(uc, st, sc, U);
        const T* ac[3] = {f.in_p(VTXBUF_AX) + idx, f.in_p(VTXBUF_AY) + idx, f.in_p(VTXBUF_AZ) + idx};
        vec_derivs(ac, st, sc, A);
    }
    const PhysT<T> p = phys_cast<T>(pc);
    T r[AC_NF];
    mhd_rates(L, S, U, A, p, r);
    if constexpr (UPWD) {
        T up_l[3], up_u[3][3], add[4];
        const T* lf = f.in_p(VTXBUF_LNRHO) + idx;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            up_l[a] = der_up(lf, st[a], sc.up[a]);
#pragma unroll
            for (int c = 0; c < 3; ++c)
                up_u[c][a] = der_up(f.in_p(VTXBUF_UUX + c) + idx, st[a], sc.up[a]);
        }
        upwind_terms(up_l, up_u, U.v, add);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            r[q] += add[q];
    }

    if (cfl) {
        const T Bx = A.g[2][1] - A.g[1][2], By = A.g[0][2] - A.g[2][0], Bz = A.g[1][0] - A.g[0][1];
        cfl_accumulate(U.v[0] * U.v[0] + U.v[1] * U.v[1] + U.v[2] * U.v[2],
                       Bx * Bx + By * By + Bz * Bz, ac_exp(-L.v), p.cs2_sound, cm,
                       pc.cfl_sum != 0);
    }

    const T val[AC_NF] = {L.v, U.v[0], U.v[1], U.v[2], A.v[0], A.v[1], A.v[2], S.v};
#pragma unroll
    for (int q = 0; q < AC_NF; ++q) {
        if constexpr (COMP) {
            const RkT32 c = {(float)rk.dt, (float)rk.beta, (float)rk.ab};
            float oh, ol;
            rk_update_comp(val[q], lo[q], prev[q], prev_lo[q], r[q], c, use_prev, oh, ol);
            f.out_p(q)[idx]    = oh;
            f.out_lo_p(q)[idx] = ol;
        }
        else {
            const RkT64 c = {rk.dt, rk.beta, rk.ab};
            double o;
            rk_update(val[q], prev[q], r[q], c, use_prev, o);
            f.out_p(q)[idx] = o;
        }
    }
}

