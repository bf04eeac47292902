/*
 * Standalone CFL maxima of the current in-buffer: max |u|, max Alfven speed
 * |curl A| / sqrt(exp(lnrho)) and max |u| + sqrt(cs^2 + vA^2) over the
 * interior.  The substep-2 launch of the solve kernels computes the same
 * maxima on the fly; this kernel serves the first step of an adaptive run, as
 * the reference's separate calc_timestep launch does
 * (acc-runtime/samples/mhd_modular/mhdsolver.ac:551-583,
 *  samples/standalone_mpi/main.cc:396-441).  Halos must be filled.
 */
#include "internal.h"
#include "mhd_rhs.cuh"

namespace {

template <typename T>
__device__ __forceinline__ T
d1(const T* f, const long long s, const T* c)
{
    T r = c[0] * (__ldg(f + s) - __ldg(f - s));
    r   = fma(c[1], __ldg(f + 2 * s) - __ldg(f - 2 * s), r);
    r   = fma(c[2], __ldg(f + 3 * s) - __ldg(f - 3 * s), r);
    return r;
}

template <typename T>
__global__ void __launch_bounds__(128)
cfl_kernel(const Geom g, const FieldsT<T> f, const StencilT<T> sc, const T cs2_sound,
           unsigned long long* cfl)
{
    __shared__ T red[3 * 4];
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    const int j = threadIdx.y + blockIdx.y * blockDim.y;
    const int k = blockIdx.z;
    T cm[3]     = {0, 0, 0};
    if (i < g.nx && j < g.ny && k < g.nz) {
        const long long idx   = geom_idx(g, i + NGHOST, j + NGHOST, k + NGHOST);
        const long long st[3] = {1, (long long)g.px, g.pxy};
        const T* ax = f.in[VTXBUF_AX] + idx;
        const T* ay = f.in[VTXBUF_AY] + idx;
        const T* az = f.in[VTXBUF_AZ] + idx;
        const T Bx  = d1(az, st[1], sc.d1[1]) - d1(ay, st[2], sc.d1[2]);
        const T By  = d1(ax, st[2], sc.d1[2]) - d1(az, st[0], sc.d1[0]);
        const T Bz  = d1(ay, st[0], sc.d1[0]) - d1(ax, st[1], sc.d1[1]);
        const T ux = f.in[VTXBUF_UUX][idx], uy = f.in[VTXBUF_UUY][idx], uz = f.in[VTXBUF_UUZ][idx];
        cfl_accumulate(ux * ux + uy * uy + uz * uz, Bx * Bx + By * By + Bz * Bz,
                       ac_exp(-f.in[VTXBUF_LNRHO][idx]), cs2_sound, cm);
    }
    cfl_commit(cm, red, cfl);
}

} // namespace

template <typename T>
cudaError_t
ac_launch_cfl(const Geom& g, const FieldsT<T>& f, const StencilCoef& sc, const double cs2_sound,
              unsigned long long* cfl, cudaStream_t stream, unsigned long long* launches)
{
    const cudaError_t e = cudaMemsetAsync(cfl, 0, 3 * sizeof(unsigned long long), stream);
    if (e != cudaSuccess)
        return e;
    const dim3 tpb(32, 4, 1);
    const dim3 bpg((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz);
    cfl_kernel<T><<<bpg, tpb, 0, stream>>>(g, f, stencil_cast<T>(sc), (T)cs2_sound, cfl);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

template cudaError_t ac_launch_cfl<double>(const Geom&, const Fields64&, const StencilCoef&,
                                           const double, unsigned long long*, cudaStream_t,
                                           unsigned long long*);
template cudaError_t ac_launch_cfl<float>(const Geom&, const Fields32&, const StencilCoef&,
                                          const double, unsigned long long*, cudaStream_t,
                                          unsigned long long*);
