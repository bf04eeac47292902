/*
 * Helical forcing of the velocity after substep 2 (the reference's LFORCING
 * option): u_out += f(x) at every interior cell, with f the helical forcing of
 * mhdsolver.ac:286-331 (model src/utils/modelsolver.cc:1003-1076).  The
 * reference adds the force to the output of the third substep
 * (mhdsolver.ac:531-541, model :1162-1168); a separate pass over the three
 * velocity fields gives the same values and leaves the solve kernels as they
 * are when forcing is off.
 */
#include "internal.h"
#include "mhd_rhs.cuh"

namespace {

template <typename T, bool COMP>
__global__ void
forcing_kernel(const Geom g, T* __restrict__ ux, T* __restrict__ uy, T* __restrict__ uz,
               float* __restrict__ lx, float* __restrict__ ly, float* __restrict__ lz,
               const PhysConst pc)
{
    const long long n = (long long)g.nx * g.ny * (pc.zhi - pc.zlo);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int i         = (int)(t % g.nx);
        const int j         = (int)((t / g.nx) % g.ny);
        const int k         = pc.zlo + (int)(t / ((long long)g.nx * g.ny));
        const long long idx = geom_idx(g, i + NGHOST, j + NGHOST, k + NGHOST);
        T f[3];
        forcing_at(pc, i, j, k, f);
        T* u[3] = {ux, uy, uz};
        if constexpr (COMP) {
            float* l[3] = {lx, ly, lz};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float h = u[c][idx], lo = l[c][idx];
                comp_add(h, lo, f[c]);
                u[c][idx] = h;
                l[c][idx] = lo;
            }
        }
        else {
#pragma unroll
            for (int c = 0; c < 3; ++c)
                u[c][idx] += f[c];
        }
    }
}

} // namespace

cudaError_t
ac_launch_forcing(const Geom& g, void* const* u, float* const* lo, const int precision,
                  const PhysConst& pc, cudaStream_t stream, unsigned long long* launches)
{
    const long long n = (long long)g.nx * g.ny * (pc.zhi - pc.zlo);
    if (n <= 0)
        return cudaSuccess;
    long long blocks  = (n + 255) / 256;
    if (blocks > 148LL * 16)
        blocks = 148LL * 16;
    if (precision == 0)
        forcing_kernel<double, false><<<(unsigned)blocks, 256, 0, stream>>>(
            g, (double*)u[0], (double*)u[1], (double*)u[2], nullptr, nullptr, nullptr, pc);
    else
        forcing_kernel<float, true><<<(unsigned)blocks, 256, 0, stream>>>(
            g, (float*)u[0], (float*)u[1], (float*)u[2], lo[0], lo[1], lo[2], pc);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}
