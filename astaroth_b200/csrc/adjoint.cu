/*
 * Discrete adjoint of one RK3 substep (acDeviceIntegrateSubstepAdjoint).
 *
 * The forward substep in 2N form (acc-runtime/stdlib/integrators.h:11-29,
 * host model src/utils/modelsolver.cc:1078-1175) is
 *     w_s     = alpha_s w_{s-1} + dt R(f_s)
 *     f_{s+1} = f_s + beta_s w_s
 * with R the 6th-order MHD right-hand side on the periodic mesh.  Its adjoint
 * maps the adjoints (lf, lw) of (f_{s+1}, w_s) to those of (f_s, w_{s-1}):
 *     lw <- lw + beta_s lf
 *     lf <- lf + dt J_R(f_s)^T lw
 *     lw <- alpha_s lw
 * and accumulates d/d(nu, eta) of dt lw . R.  J_R^T is applied in two
 * passes: adj_local_kernel evaluates, per cell, the reverse of the RHS into the
 * adjoints mu of the 46 derivative slots (mhd_rhs_adjoint.cuh); after a
 * periodic halo fill of mu, adj_gather_kernel applies the transposed stencils:
 * first derivatives are antisymmetric (D^T = -D), second, Laplacian and the
 * diagonal mixed stencils are symmetric, so the gather for a vector field is
 * value - div-like first-derivative terms + lap + grad div of the slot fields.
 */
#include "internal.h"
#include "mhd_rhs_adjoint.cuh"
#include "stencil_plain.cuh"

namespace {

__global__ void __launch_bounds__(128)
adj_local_kernel(const Geom g, const AdjointFields a, const StencilCoef sc, const PhysConst pc,
                 const double beta, const double dt, double* __restrict__ pgrad)
{
    __shared__ double red[2 * 4];
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    const int j = threadIdx.y + blockIdx.y * blockDim.y;
    const int k = blockIdx.z;
    double gnu = 0, geta = 0;
    if (i < g.nx && j < g.ny && k < g.nz) {
        const long long idx   = geom_idx(g, i + NGHOST, j + NGHOST, k + NGHOST);
        const long long st[3] = {1, (long long)g.px, g.pxy};
        double lam[AC_NF];
#pragma unroll
        for (int q = 0; q < AC_NF; ++q) {
            const double w = a.lw[q][idx] + beta * a.lf[q][idx];
            a.lw[q][idx]   = w;
            lam[q]         = dt * w;
        }
        ScalD<double> L, S;
        VecD<double> U, A;
        scal_derivs(a.f[VTXBUF_LNRHO] + idx, st, sc, L);
        scal_derivs(a.f[VTXBUF_ENTROPY] + idx, st, sc, S);
        {
            const double* uc[3] = {a.f[VTXBUF_UUX] + idx, a.f[VTXBUF_UUY] + idx,
                                   a.f[VTXBUF_UUZ] + idx};
            vec_derivs(uc, st, sc, U);
            const double* ac[3] = {a.f[VTXBUF_AX] + idx, a.f[VTXBUF_AY] + idx,
                                   a.f[VTXBUF_AZ] + idx};
            vec_derivs(ac, st, sc, A);
        }
        /* the rate order of mhd_rates: lnrho, ux, uy, uz, ax, ay, az, entropy */
        double mu[MU_COUNT];
        mhd_rates_adjoint(L, S, U, A, phys_cast<double>(pc), lam, mu, gnu, geta);
#pragma unroll
        for (int m = 0; m < MU_COUNT; ++m)
            a.mu[m][idx] = mu[m];
    }
    /* block sums of the parameter adjoints, one atomic per block and value */
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        gnu += __shfl_xor_sync(0xffffffffu, gnu, o);
        geta += __shfl_xor_sync(0xffffffffu, geta, o);
    }
    if (lane == 0) {
        red[2 * warp]     = gnu;
        red[2 * warp + 1] = geta;
    }
    __syncthreads();
    if (tid == 0) {
        double s0 = 0, s1 = 0;
        for (int w = 0; w < 4; ++w) {
            s0 += red[2 * w];
            s1 += red[2 * w + 1];
        }
        atomicAdd(pgrad, s0);
        atomicAdd(pgrad + 1, s1);
    }
}

/* lap of a slot field at idx */
__device__ __forceinline__ double
lap_of(const double* f, const long long* st, const StencilCoef& sc)
{
    return (sc.d2[0][0] + sc.d2[1][0] + sc.d2[2][0]) * __ldg(f) + der2_sides(f, st[0], sc.d2[0]) +
           der2_sides(f, st[1], sc.d2[1]) + der2_sides(f, st[2], sc.d2[2]);
}

/* value + sum_a D_a^T g_a + lap^T lap for a scalar slot block at base m */
__device__ __forceinline__ double
gather_scalar(const AdjointFields& a, const int m, const long long idx, const long long* st,
              const StencilCoef& sc)
{
    double acc = __ldg(a.mu[m + MU_SV] + idx);
#pragma unroll
    for (int ax = 0; ax < 3; ++ax)
        acc -= der1(a.mu[m + MU_SG + ax] + idx, st[ax], sc.d1[ax]);
    return acc + lap_of(a.mu[m + MU_SLAP] + idx, st, sc);
}

/* the same for component c of a vector slot block, plus grad div^T = grad div of
 * the three gd slots */
__device__ __forceinline__ void
gather_vector(const AdjointFields& a, const int m, const long long idx, const long long* st,
              const StencilCoef& sc, double out[3])
{
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double acc = __ldg(a.mu[m + MU_VV + c] + idx);
#pragma unroll
        for (int ax = 0; ax < 3; ++ax)
            acc -= der1(a.mu[m + MU_VG + 3 * c + ax] + idx, st[ax], sc.d1[ax]);
        out[c] = acc + lap_of(a.mu[m + MU_VLAP + c] + idx, st, sc);
    }
    const double* gd0 = a.mu[m + MU_VGD + 0] + idx;
    const double* gd1 = a.mu[m + MU_VGD + 1] + idx;
    const double* gd2 = a.mu[m + MU_VGD + 2] + idx;
    const double d00  = sc.d2[0][0] * __ldg(gd0) + der2_sides(gd0, st[0], sc.d2[0]);
    const double d11  = sc.d2[1][0] * __ldg(gd1) + der2_sides(gd1, st[1], sc.d2[1]);
    const double d22  = sc.d2[2][0] * __ldg(gd2) + der2_sides(gd2, st[2], sc.d2[2]);
    out[0] += d00 + dermix(gd1, st[0], st[1], sc.mix[0]) + dermix(gd2, st[0], st[2], sc.mix[1]);
    out[1] += dermix(gd0, st[0], st[1], sc.mix[0]) + d11 + dermix(gd2, st[1], st[2], sc.mix[2]);
    out[2] += dermix(gd0, st[0], st[2], sc.mix[1]) + dermix(gd1, st[1], st[2], sc.mix[2]) + d22;
}

__global__ void __launch_bounds__(128)
adj_gather_kernel(const Geom g, const AdjointFields a, const StencilCoef sc, const double alpha)
{
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    const int j = threadIdx.y + blockIdx.y * blockDim.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny || k >= g.nz)
        return;
    const long long idx   = geom_idx(g, i + NGHOST, j + NGHOST, k + NGHOST);
    const long long st[3] = {1, (long long)g.px, g.pxy};
    double add[AC_NF];
    add[VTXBUF_LNRHO]   = gather_scalar(a, MU_L, idx, st, sc);
    add[VTXBUF_ENTROPY] = gather_scalar(a, MU_S, idx, st, sc);
    gather_vector(a, MU_U, idx, st, sc, &add[VTXBUF_UUX]);
    gather_vector(a, MU_A, idx, st, sc, &add[VTXBUF_AX]);
#pragma unroll
    for (int q = 0; q < AC_NF; ++q) {
        a.lf[q][idx] += add[q];
        a.lw[q][idx] *= alpha;
    }
}

} // namespace

cudaError_t
ac_launch_adjoint_substep(const Geom& g, const AdjointFields& a, const StencilCoef& sc,
                          const PhysConst& pc, const double alpha, const double beta,
                          const double dt, double* pgrad, cudaStream_t stream,
                          unsigned long long* launches)
{
    const dim3 tpb(32, 4, 1);
    const dim3 bpg((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz);
    adj_local_kernel<<<bpg, tpb, 0, stream>>>(g, a, sc, pc, beta, dt, pgrad);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return e;
    const Volume m0 = {0, 0, 0};
    const Volume m1 = {(size_t)g.mx, (size_t)g.my, (size_t)g.mz};
    e = ac_launch_periodic<double>(g, a.mu, MU_COUNT, m0, m1, stream, launches);
    if (e != cudaSuccess)
        return e;
    adj_gather_kernel<<<bpg, tpb, 0, stream>>>(g, a, sc, alpha);
    if (launches)
        *launches += 2;
    return cudaGetLastError();
}
