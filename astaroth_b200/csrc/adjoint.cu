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
 * adjoints mu of the 46 derivative slots (mhd_rhs_adjoint.cuh), adds the 8
 * value slots to lf directly and stores the 38 others; adj_gather_kernel then
 * applies the transposed stencils at wrapped (periodic) interior indices, so
 * mu needs no halo fill: first derivatives are antisymmetric (D^T = -D),
 * second, Laplacian and the diagonal mixed stencils are symmetric, so the
 * gather for a vector field is - div-like first-derivative terms + lap + grad
 * div of the slot fields.  The gather runs one output field per block.
 */
#include "internal.h"
#include "mhd_rhs_adjoint.cuh"
#include "stencil_plain.cuh"

namespace {

/* z planes per thread of the gather.  Consecutive planes of one column share
 * most stencil taps through L1, but the kernel is latency-bound, and one plane
 * per thread (8x the blocks) measured 10% faster per adjoint substep at 64^3
 * than 2, 4 or 8 planes.  (The local kernel also keeps one plane per thread:
 * a loop there spills its 254 registers.) */
constexpr int KZ = 1;

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
        /* value slots need no stencil: their transpose is the identity */
        const int vslot[AC_NF] = {MU_L + MU_SV,     MU_U + MU_VV,     MU_U + MU_VV + 1,
                                  MU_U + MU_VV + 2, MU_A + MU_VV,     MU_A + MU_VV + 1,
                                  MU_A + MU_VV + 2, MU_S + MU_SV};
#pragma unroll
        for (int q = 0; q < AC_NF; ++q)
            a.lf[q][idx] += mu[vslot[q]];
#pragma unroll
        for (int m = 0; m < MU_COUNT; ++m) {
            const bool value_slot = m == MU_L + MU_SV || m == MU_S + MU_SV ||
                                    (m >= MU_U + MU_VV && m < MU_U + MU_VV + 3) ||
                                    (m >= MU_A + MU_VV && m < MU_A + MU_VV + 3);
            if (!value_slot)
                a.mu[m][idx] = mu[m];
        }
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

/* Periodic neighbour offsets of one interior cell: o[a][d + 3] is the index
 * offset of the interior cell d steps away along axis a, wrapped.  The slot
 * arrays mu are read only at interior cells, so they need no halo fill. */
struct Wrap {
    long long o[3][7];
};

__device__ __forceinline__ int
wrap(const int v, const int n)
{
    const int r = v % n;
    return r < 0 ? r + n : r;
}

__device__ __forceinline__ void
make_wrap(const Geom& g, const int i, const int j, const int k, Wrap& w)
{
#pragma unroll
    for (int d = -3; d <= 3; ++d) {
        w.o[0][d + 3] = (long long)(wrap(i + d, g.nx) - i);
        w.o[1][d + 3] = (long long)(wrap(j + d, g.ny) - j) * g.px;
        w.o[2][d + 3] = (long long)(wrap(k + d, g.nz) - k) * g.pxy;
    }
}

/* sum_k c_k (f[+k] - f[-k]) along axis A */
template <int A>
__device__ __forceinline__ double
wd1(const double* f, const Wrap& w, const double* c)
{
    double r = c[0] * (__ldg(f + w.o[A][4]) - __ldg(f + w.o[A][2]));
    r        = fma(c[1], __ldg(f + w.o[A][5]) - __ldg(f + w.o[A][1]), r);
    r        = fma(c[2], __ldg(f + w.o[A][6]) - __ldg(f + w.o[A][0]), r);
    return r;
}

/* sum_k d_k (f[+k] + f[-k]) along axis A (centre excluded) */
template <int A>
__device__ __forceinline__ double
wd2s(const double* f, const Wrap& w, const double* d)
{
    double r = d[1] * (__ldg(f + w.o[A][4]) + __ldg(f + w.o[A][2]));
    r        = fma(d[2], __ldg(f + w.o[A][5]) + __ldg(f + w.o[A][1]), r);
    r        = fma(d[3], __ldg(f + w.o[A][6]) + __ldg(f + w.o[A][0]), r);
    return r;
}

/* sum_k e_k (f(+k,+k) + f(-k,-k) - f(+k,-k) - f(-k,+k)) along axes A, B */
template <int A, int B>
__device__ __forceinline__ double
wmix(const double* f, const Wrap& w, const double* e)
{
    double r = 0;
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
        const double t = (__ldg(f + w.o[A][3 + k] + w.o[B][3 + k]) +
                          __ldg(f + w.o[A][3 - k] + w.o[B][3 - k])) -
                         (__ldg(f + w.o[A][3 + k] + w.o[B][3 - k]) +
                          __ldg(f + w.o[A][3 - k] + w.o[B][3 + k]));
        r = k == 1 ? e[0] * t : fma(e[k - 1], t, r);
    }
    return r;
}

__device__ __forceinline__ double
wlap(const double* f, const Wrap& w, const StencilCoef& sc)
{
    return (sc.d2[0][0] + sc.d2[1][0] + sc.d2[2][0]) * __ldg(f) + wd2s<0>(f, w, sc.d2[0]) +
           wd2s<1>(f, w, sc.d2[1]) + wd2s<2>(f, w, sc.d2[2]);
}

/* - sum_a D_a g_a + lap(l): the transposed first-derivative and Laplacian
 * terms of one output field (D1^T = -D1, the Laplacian is symmetric) */
__device__ __forceinline__ double
gather_gl(const AdjointFields& a, const int g0, const int l, const long long idx, const Wrap& w,
          const StencilCoef& sc)
{
    double acc = -wd1<0>(a.mu[g0] + idx, w, sc.d1[0]);
    acc -= wd1<1>(a.mu[g0 + 1] + idx, w, sc.d1[1]);
    acc -= wd1<2>(a.mu[g0 + 2] + idx, w, sc.d1[2]);
    return acc + wlap(a.mu[l] + idx, w, sc);
}

/* (grad div)^T = grad div of the three gd slots, component C */
template <int C>
__device__ __forceinline__ double
gather_gd(const AdjointFields& a, const int gd0, const long long idx, const Wrap& w,
          const StencilCoef& sc)
{
    const double* g0 = a.mu[gd0] + idx;
    const double* g1 = a.mu[gd0 + 1] + idx;
    const double* g2 = a.mu[gd0 + 2] + idx;
    if (C == 0)
        return (sc.d2[0][0] * __ldg(g0) + wd2s<0>(g0, w, sc.d2[0])) +
               wmix<0, 1>(g1, w, sc.mix[0]) + wmix<0, 2>(g2, w, sc.mix[1]);
    if (C == 1)
        return wmix<0, 1>(g0, w, sc.mix[0]) + (sc.d2[1][0] * __ldg(g1) + wd2s<1>(g1, w, sc.d2[1])) +
               wmix<1, 2>(g2, w, sc.mix[2]);
    return wmix<0, 2>(g0, w, sc.mix[1]) + wmix<1, 2>(g1, w, sc.mix[2]) +
           (sc.d2[2][0] * __ldg(g2) + wd2s<2>(g2, w, sc.d2[2]));
}

/* One output field per block (blockIdx.z = zblock * AC_NF + q), so a block
 * reads only the slot arrays of that field; KZ planes per thread. */
__global__ void __launch_bounds__(128)
adj_gather_kernel(const Geom g, const AdjointFields a, const StencilCoef sc, const double alpha)
{
    const int i = threadIdx.x + blockIdx.x * blockDim.x;
    const int j = threadIdx.y + blockIdx.y * blockDim.y;
    const int q = blockIdx.z % AC_NF;
    if (i >= g.nx || j >= g.ny)
        return;
    const int k1 = min((int)(blockIdx.z / AC_NF + 1) * KZ, g.nz);
    for (int k = blockIdx.z / AC_NF * KZ; k < k1; ++k) {
        const long long idx = geom_idx(g, i + NGHOST, j + NGHOST, k + NGHOST);
        Wrap w;
        make_wrap(g, i, j, k, w);
        double add;
        if (q == VTXBUF_LNRHO || q == VTXBUF_ENTROPY) {
            const int m = q == VTXBUF_LNRHO ? MU_L : MU_S;
            add         = gather_gl(a, m + MU_SG, m + MU_SLAP, idx, w, sc);
        }
        else {
            const int m = q <= VTXBUF_UUZ ? MU_U : MU_A;
            const int c = q <= VTXBUF_UUZ ? q - VTXBUF_UUX : q - VTXBUF_AX;
            add         = gather_gl(a, m + MU_VG + 3 * c, m + MU_VLAP + c, idx, w, sc);
            add += c == 0 ? gather_gd<0>(a, m + MU_VGD, idx, w, sc)
                          : c == 1 ? gather_gd<1>(a, m + MU_VGD, idx, w, sc)
                                   : gather_gd<2>(a, m + MU_VGD, idx, w, sc);
        }
        a.lf[q][idx] += add;
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
    const unsigned zb = (unsigned)((g.nz + KZ - 1) / KZ);
    if ((long long)zb * AC_NF > 65535)
        return cudaErrorInvalidConfiguration;
    const dim3 gpg(bpg.x, bpg.y, zb * AC_NF);
    adj_gather_kernel<<<gpg, tpb, 0, stream>>>(g, a, sc, alpha);
    if (launches)
        *launches += 2;
    return cudaGetLastError();
}
