/*
 * The auxiliary magnetic field B = curl A (the reference's LBFIELD option:
 * `write(BFIELD, curl(AA))` of acc-runtime/samples/mhd_modular/mhdsolver.ac:
 * 546-548 and 605-608).  After a whole RK3 step both reference forms leave
 * curl A of the input of substep 2, which this kernel computes when substep 2
 * is launched: 6th-order first derivatives of the in-buffer (the values hi of
 * FP32-compensated meshes), evaluated in double, written to three double
 * arrays in the host layout (x fastest, pitch mx, halos included and left 0).
 */
#include "internal.h"
#include "stencil_plain.cuh"

namespace {

template <typename T>
__global__ void
bfield_kernel(const Geom g, const T* __restrict__ ax, const T* __restrict__ ay,
              const T* __restrict__ az, double* __restrict__ bx, double* __restrict__ by,
              double* __restrict__ bz, const StencilCoef sc)
{
    const long long n = (long long)g.nx * g.ny * g.nz;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int i          = (int)(t % g.nx) + NGHOST;
        const int j          = (int)((t / g.nx) % g.ny) + NGHOST;
        const int k          = (int)(t / ((long long)g.nx * g.ny)) + NGHOST;
        const long long idx  = geom_idx(g, i, j, k);
        const long long st[3] = {1, (long long)g.px, g.pxy};
        /* d A_c / d x_a, with the taps converted to double */
        double d[3][3];
        const T* a[3] = {ax + idx, ay + idx, az + idx};
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                const T* f = a[c];
                const long long s = st[e];
                double r = sc.d1[e][0] * ((double)__ldg(f + s) - (double)__ldg(f - s));
                r        = fma(sc.d1[e][1], (double)__ldg(f + 2 * s) - (double)__ldg(f - 2 * s), r);
                r        = fma(sc.d1[e][2], (double)__ldg(f + 3 * s) - (double)__ldg(f - 3 * s), r);
                d[c][e]  = r;
            }
        const long long o = (long long)i + (long long)g.mx * (j + (long long)g.my * k);
        bx[o]             = d[2][1] - d[1][2];
        by[o]             = d[0][2] - d[2][0];
        bz[o]             = d[1][0] - d[0][1];
    }
}

} // namespace

cudaError_t
ac_launch_bfield(const Geom& g, const void* const* a, double* const* b, const int precision,
                 const StencilCoef& sc, cudaStream_t stream, unsigned long long* launches)
{
    const long long n = (long long)g.nx * g.ny * g.nz;
    long long blocks  = (n + 255) / 256;
    if (blocks > 148LL * 16)
        blocks = 148LL * 16;
    if (precision == 0)
        bfield_kernel<double><<<(unsigned)blocks, 256, 0, stream>>>(
            g, (const double*)a[0], (const double*)a[1], (const double*)a[2], b[0], b[1], b[2], sc);
    else
        bfield_kernel<float><<<(unsigned)blocks, 256, 0, stream>>>(
            g, (const float*)a[0], (const float*)a[1], (const float*)a[2], b[0], b[1], b[2], sc);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}
