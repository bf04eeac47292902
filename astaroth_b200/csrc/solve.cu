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
#include "solve_cell.cuh"

namespace {

/* Every thread reaches the single cfl_commit at the end (it uses full-warp
 * shuffles and a block barrier), so there is no early return. */
template <typename T, bool COMP, bool UPWD>
__global__ void __launch_bounds__(128)
solve_plain_kernel(const Geom g, const FieldsT<T> f, const StencilT<T> sc, const PhysConst pc,
                   const RkCoef rk, unsigned long long* cfl)
{
    __shared__ T red[3 * 4];
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    const int j = threadIdx.y + blockIdx.y * blockDim.y;
    const int k = pc.zlo + (int)blockIdx.z;
    T cm[3]     = {0, 0, 0};
    if (i < g.nx && j < g.ny && k < pc.zhi)
        plain_cell<T, COMP, UPWD>(g, PtrFieldsT<T>{f}, sc, pc, rk, cfl != nullptr, i, j, k, cm);
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
    const dim3 bpg((g.nx + tpb.x - 1) / tpb.x, (g.ny + tpb.y - 1) / tpb.y, pc.zhi - pc.zlo);
    if (pc.upwind)
        solve_plain_kernel<T, COMP, true><<<bpg, tpb, 0, stream>>>(g, f, stencil_cast<T>(sc), pc,
                                                                  rk, cfl);
    else
        solve_plain_kernel<T, COMP, false><<<bpg, tpb, 0, stream>>>(g, f, stencil_cast<T>(sc), pc,
                                                                   rk, cfl);
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
