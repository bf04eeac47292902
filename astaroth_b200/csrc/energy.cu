/*
 * The energy functional of the adjoint workloads and its gradient
 * (acEnergyFunctional).  The reference has no energy functional (its
 * reductions are RMS and exp^2 maps, acc-runtime/stdlib/map.h:40-46); this is
 * the objective of the differentiable integration:
 *
 *   J = sum over interior cells of ( (1/2) exp(lnrho) |u|^2 + |B|^2 / (2 mu0) ) dV,
 *   B = curl A with the solver's 6th-order first derivatives on the periodic
 *       interior (wrapped indices, so the halos of the input are not read),
 *
 *   dJ/dlnrho = (1/2) exp(lnrho) |u|^2 dV,  dJ/du = exp(lnrho) u dV,
 *   dJ/dA     = curl(B) / mu0 dV   (D1^T = -D1 on the periodic grid),
 *   dJ/ds     = 0.
 *
 * Two kernels: the first forms B (kept in caller scratch) and the per-cell
 * terms, with a deterministic sum (per-block double-double partials combined
 * in block order by the last block); the second forms curl B for the gradient.
 */
#include "internal.h"

namespace {

constexpr int kTpb = 256;

struct DD {
    double hi, lo;
};

__device__ __forceinline__ DD
dd_add(const DD a, const DD b)
{
    const double s  = a.hi + b.hi;
    const double bb = s - a.hi;
    const double e  = (a.hi - (s - bb)) + (b.hi - bb) + a.lo + b.lo;
    const double h  = s + e;
    return DD{h, e - (h - s)};
}

__device__ __forceinline__ int
wrap(const int i, const int n)
{
    return i < 0 ? i + n : i >= n ? i - n : i;
}

struct EGeom {
    int nx, ny, nz, mx, my;
    double inv[3]; /* 1 / ds per axis */
    double dV, inv_mu0;
};

__device__ __forceinline__ long long
eidx(const EGeom& g, const int i, const int j, const int k)
{
    return (long long)(i + NGHOST) + (long long)g.mx * ((j + NGHOST) + (long long)g.my * (k + NGHOST));
}

/* 6th-order first derivative along axis a at interior cell (i, j, k), wrapped */
__device__ __forceinline__ double
d1w(const double* f, const EGeom& g, const int a, const int i, const int j, const int k)
{
    const double c[3] = {3.0 / 4.0, -3.0 / 20.0, 1.0 / 60.0};
    double r          = 0;
#pragma unroll
    for (int s = 1; s <= 3; ++s) {
        double p, m;
        if (a == 0) {
            p = f[eidx(g, wrap(i + s, g.nx), j, k)];
            m = f[eidx(g, wrap(i - s, g.nx), j, k)];
        }
        else if (a == 1) {
            p = f[eidx(g, i, wrap(j + s, g.ny), k)];
            m = f[eidx(g, i, wrap(j - s, g.ny), k)];
        }
        else {
            p = f[eidx(g, i, j, wrap(k + s, g.nz))];
            m = f[eidx(g, i, j, wrap(k - s, g.nz))];
        }
        r = s == 1 ? c[0] * (p - m) : fma(c[s - 1], p - m, r);
    }
    return r * g.inv[a];
}

struct Ptr8 {
    const double* f[8];
    double* g[8];
};

/* B into scratch b[3] (host layout), the per-cell terms summed into J, and
 * (when grad) the lnrho and u gradients; s's gradient is zero. */
__global__ void __launch_bounds__(kTpb)
energy_kernel(const EGeom g, const Ptr8 p, double* __restrict__ b0, double* __restrict__ b1,
              double* __restrict__ b2, double* __restrict__ partials,
              unsigned int* __restrict__ counter, double* __restrict__ J, const int grad)
{
    __shared__ double s_hi[kTpb / 32], s_lo[kTpb / 32];
    __shared__ bool s_last;
    const long long n = (long long)g.nx * g.ny * g.nz;
    DD acc{0.0, 0.0};
    for (long long t = (long long)blockIdx.x * kTpb + threadIdx.x; t < n;
         t += (long long)gridDim.x * kTpb) {
        const int i          = (int)(t % g.nx);
        const int j          = (int)((t / g.nx) % g.ny);
        const int k          = (int)(t / ((long long)g.nx * g.ny));
        const long long idx  = eidx(g, i, j, k);
        const double lr      = p.f[0][idx];
        const double ux = p.f[1][idx], uy = p.f[2][idx], uz = p.f[3][idx];
        const double Bx = d1w(p.f[6], g, 1, i, j, k) - d1w(p.f[5], g, 2, i, j, k);
        const double By = d1w(p.f[4], g, 2, i, j, k) - d1w(p.f[6], g, 0, i, j, k);
        const double Bz = d1w(p.f[5], g, 0, i, j, k) - d1w(p.f[4], g, 1, i, j, k);
        b0[idx]         = Bx;
        b1[idx]         = By;
        b2[idx]         = Bz;
        const double er = exp(lr);
        const double u2 = ux * ux + uy * uy + uz * uz;
        const double ek = 0.5 * er * u2 * g.dV;
        const double em = (Bx * Bx + By * By + Bz * Bz) * (0.5 * g.inv_mu0) * g.dV;
        acc             = dd_add(acc, DD{ek + em, 0.0});
        if (grad) {
            p.g[0][idx] = ek;
            p.g[1][idx] = er * ux * g.dV;
            p.g[2][idx] = er * uy * g.dV;
            p.g[3][idx] = er * uz * g.dV;
            p.g[7][idx] = 0.0;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        acc = dd_add(acc, DD{__shfl_xor_sync(0xffffffffu, acc.hi, o),
                             __shfl_xor_sync(0xffffffffu, acc.lo, o)});
    if (lane == 0) {
        s_hi[warp] = acc.hi;
        s_lo[warp] = acc.lo;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        DD b{0.0, 0.0};
        for (int w = 0; w < kTpb / 32; ++w)
            b = dd_add(b, DD{s_hi[w], s_lo[w]});
        partials[2 * blockIdx.x]     = b.hi;
        partials[2 * blockIdx.x + 1] = b.lo;
        __threadfence();
        s_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0)
        return;
    __threadfence();
    /* the last block sums the partials in block order */
    const volatile double* vp = partials;
    DD t{0.0, 0.0};
    for (unsigned b = 0; b < gridDim.x; ++b)
        t = dd_add(t, DD{vp[2 * b], vp[2 * b + 1]});
    *J       = t.hi + t.lo;
    *counter = 0u;
}

/* dJ/dA = curl(B) / mu0 dV at the interior cells */
__global__ void __launch_bounds__(kTpb)
energy_grad_a_kernel(const EGeom g, const double* __restrict__ b0, const double* __restrict__ b1,
                     const double* __restrict__ b2, double* __restrict__ ga0,
                     double* __restrict__ ga1, double* __restrict__ ga2)
{
    const long long n = (long long)g.nx * g.ny * g.nz;
    const double s    = g.inv_mu0 * g.dV;
    for (long long t = (long long)blockIdx.x * kTpb + threadIdx.x; t < n;
         t += (long long)gridDim.x * kTpb) {
        const int i         = (int)(t % g.nx);
        const int j         = (int)((t / g.nx) % g.ny);
        const int k         = (int)(t / ((long long)g.nx * g.ny));
        const long long idx = eidx(g, i, j, k);
        ga0[idx] = (d1w(b2, g, 1, i, j, k) - d1w(b1, g, 2, i, j, k)) * s;
        ga1[idx] = (d1w(b0, g, 2, i, j, k) - d1w(b2, g, 0, i, j, k)) * s;
        ga2[idx] = (d1w(b1, g, 0, i, j, k) - d1w(b0, g, 1, i, j, k)) * s;
    }
}

} // namespace

extern "C" AcResult
acEnergyFunctional(const AcMeshInfo info, const AcReal* const* fields, AcReal* J,
                   AcReal* const* grad, AcReal* scratch, void* stream)
{
    if (!fields || !J || !scratch)
        return AC_FAILURE;
    for (int q = 0; q < AC_NF; ++q)
        if (!fields[q] || (grad && !grad[q]))
            return AC_FAILURE;
    const int3 n  = info.int3_params[AC_nlocal];
    const AcReal3 ds = info.real3_params[AC_ds];
    const double mu0 = info.real_params[AC_mu0];
    if (n.x < 4 || n.y < 4 || n.z < 4 || !(ds.x > 0) || !(ds.y > 0) || !(ds.z > 0) || !(mu0 > 0))
        return AC_FAILURE;
    EGeom g;
    g.nx = n.x;
    g.ny = n.y;
    g.nz = n.z;
    g.mx = n.x + 2 * NGHOST;
    g.my = n.y + 2 * NGHOST;
    g.inv[0]  = 1.0 / ds.x;
    g.inv[1]  = 1.0 / ds.y;
    g.inv[2]  = 1.0 / ds.z;
    g.dV      = ds.x * ds.y * ds.z;
    g.inv_mu0 = 1.0 / mu0;
    const long long cells = (long long)g.mx * g.my * (n.z + 2 * NGHOST);
    /* scratch: B (3 arrays of the mesh size), then 2 doubles per block and
     * the block counter */
    double* b0            = scratch;
    double* b1            = b0 + cells;
    double* b2            = b1 + cells;
    const int blocks      = 148 * 4;
    double* partials      = b2 + cells;
    unsigned int* counter = (unsigned int*)(partials + 2 * blocks);
    cudaStream_t st       = (cudaStream_t)stream;
    Ptr8 p;
    for (int q = 0; q < AC_NF; ++q) {
        p.f[q] = fields[q];
        p.g[q] = grad ? grad[q] : nullptr;
    }
    AC_CUDA_CHECK(cudaMemsetAsync(counter, 0, sizeof(unsigned int), st));
    energy_kernel<<<blocks, kTpb, 0, st>>>(g, p, b0, b1, b2, partials, counter, J, grad ? 1 : 0);
    AC_CUDA_CHECK(cudaGetLastError());
    if (grad) {
        energy_grad_a_kernel<<<blocks, kTpb, 0, st>>>(g, b0, b1, b2, grad[4], grad[5], grad[6]);
        AC_CUDA_CHECK(cudaGetLastError());
    }
    return AC_SUCCESS;
}

extern "C" size_t
acEnergyFunctionalScratchBytes(const AcMeshInfo info)
{
    const int3 n = info.int3_params[AC_nlocal];
    const size_t cells =
        (size_t)(n.x + 2 * NGHOST) * (size_t)(n.y + 2 * NGHOST) * (size_t)(n.z + 2 * NGHOST);
    return (3 * cells + 2 * 148 * 4) * sizeof(double) + 64;
}
