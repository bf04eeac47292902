/*
 * The MHD substep kernel without tiling ("plain"): one thread per cell,
 * every stencil tap an __ldg through L1, for FP64 and FP32-compensated
 * meshes.  It is the simple correctness baseline the tiled kernels
 * (solve_tiled.cu) are checked against, and the path for meshes the tiled
 * kernels do not support (nx < 32 or ny < 4, or an odd nx in FP64).
 *
 * Reference: twopass_solve_intermediate/final and singlepass_solve,
 * acc-runtime/samples/mhd_modular/mhdsolver.ac:524-636, with the stencils of
 * acc-runtime/stdlib/derivs.h:374-427,591-690 (host model
 * src/utils/modelsolver.cc:190-299) and rk3() of
 * acc-runtime/stdlib/integrators.h:11-29.
 */
#include "internal.h"
#include "mhd_rhs.cuh"
#include "stencil_plain.cuh"

namespace {

/* One cell of the plain kernel; adds the cell's CFL quantities to cm when cfl is set. */
template <typename T, bool COMP>
__device__ __forceinline__ void
plain_cell(const Geom& g, const FieldsT<T>& f, const StencilT<T>& sc, const PhysConst& pc,
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
        prev[q]    = use_prev ? f.out[q][idx] : T(0);
        prev_lo[q] = (COMP && use_prev) ? f.out_lo[q][idx] : T(0);
        lo[q]      = COMP ? f.in_lo[q][idx] : T(0);
    }

    ScalD<T> L, S;
    VecD<T> U, A;
    scal_derivs(f.in[VTXBUF_LNRHO] + idx, st, sc, L);
    scal_derivs(f.in[VTXBUF_ENTROPY] + idx, st, sc, S);
    {
        const T* uc[3] = {f.in[VTXBUF_UUX] + idx, f.in[VTXBUF_UUY] + idx,
                          f.in[VTXBUF_UUZ] + idx};
        vec_derivs(uc, st, sc, U);
        const T* ac[3] = {f.in[VTXBUF_AX] + idx, f.in[VTXBUF_AY] + idx, f.in[VTXBUF_AZ] + idx};
        vec_derivs(ac, st, sc, A);
    }
    const PhysT<T> p = phys_cast<T>(pc);
    T r[AC_NF];
    mhd_rates(L, S, U, A, p, r);

    if (cfl) {
        const T Bx = A.g[2][1] - A.g[1][2], By = A.g[0][2] - A.g[2][0], Bz = A.g[1][0] - A.g[0][1];
        cfl_accumulate(U.v[0] * U.v[0] + U.v[1] * U.v[1] + U.v[2] * U.v[2],
                       Bx * Bx + By * By + Bz * Bz, ac_exp(-L.v), p.cs2_sound, cm);
    }

    const T val[AC_NF] = {L.v, U.v[0], U.v[1], U.v[2], A.v[0], A.v[1], A.v[2], S.v};
#pragma unroll
    for (int q = 0; q < AC_NF; ++q) {
        if constexpr (COMP) {
            const RkT32 c = {(float)rk.dt, (float)rk.beta, (float)rk.ab};
            float oh, ol;
            rk_update_comp(val[q], lo[q], prev[q], prev_lo[q], r[q], c, use_prev, oh, ol);
            f.out[q][idx]    = oh;
            f.out_lo[q][idx] = ol;
        }
        else {
            const RkT64 c = {rk.dt, rk.beta, rk.ab};
            double o;
            rk_update(val[q], prev[q], r[q], c, use_prev, o);
            f.out[q][idx] = o;
        }
    }
}

/* Every thread reaches the single cfl_commit at the end (it uses full-warp
 * shuffles and a block barrier), so there is no early return. */
template <typename T, bool COMP>
__global__ void __launch_bounds__(128)
solve_plain_kernel(const Geom g, const FieldsT<T> f, const StencilT<T> sc, const PhysConst pc,
                   const RkCoef rk, unsigned long long* cfl)
{
    __shared__ T red[3 * 4];
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    const int j = threadIdx.y + blockIdx.y * blockDim.y;
    const int k = blockIdx.z;
    T cm[3]     = {0, 0, 0};
    if (i < g.nx && j < g.ny && k < g.nz)
        plain_cell<T, COMP>(g, f, sc, pc, rk, cfl != nullptr, i, j, k, cm);
    if (cfl)
        cfl_commit(cm, red, cfl);
}

template <typename T, bool COMP>
cudaError_t
launch_plain(const Geom& g, const FieldsT<T>& f, const StencilCoef& sc, const PhysConst& pc,
             const RkCoef& rk, unsigned long long* cfl, cudaStream_t stream,
             unsigned long long* launches)
{
    const dim3 tpb(32, 4, 1);
    const dim3 bpg((g.nx + tpb.x - 1) / tpb.x, (g.ny + tpb.y - 1) / tpb.y, g.nz);
    solve_plain_kernel<T, COMP><<<bpg, tpb, 0, stream>>>(g, f, stencil_cast<T>(sc), pc, rk, cfl);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

} // namespace

cudaError_t
ac_launch_solve_plain64(const Geom& g, const Fields64& f, const StencilCoef& sc,
                        const PhysConst& pc, const RkCoef& rk, unsigned long long* cfl,
                        cudaStream_t stream, unsigned long long* launches)
{
    return launch_plain<double, false>(g, f, sc, pc, rk, cfl, stream, launches);
}

cudaError_t
ac_launch_solve_plain32(const Geom& g, const Fields32& f, const StencilCoef& sc,
                        const PhysConst& pc, const RkCoef& rk, unsigned long long* cfl,
                        cudaStream_t stream, unsigned long long* launches)
{
    return launch_plain<float, true>(g, f, sc, pc, rk, cfl, stream, launches);
}
