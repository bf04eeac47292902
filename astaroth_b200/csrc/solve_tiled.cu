/*
 * The substep kernel, 2.5-D blocked (the production path on B200), for FP64
 * meshes and FP32-compensated meshes (the FP32 ring holds the hi parts; the
 * update works on (hi, lo) pairs, see rk_update_comp).
 *
 * Each CTA owns a 32 x 4 (x, y) tile of the interior and marches along z over
 * a chunk of up to ZCHUNK planes (fewer on small meshes, so that the grid
 * still covers the SMs; see zchunk_for).  A ring of RING = 8 shared-memory slots holds the
 * planes z-3 .. z+3 the stencils of plane z need plus one plane in flight.
 * One TMA instruction (cp.async.bulk.tensor.4d, CTA-local) brings a whole
 * plane of all 8 fields -- a (38 x 10 x 1 x 8) box of the in-buffer (40 wide
 * in FP32, where the box row must be a multiple of 16 bytes), halo
 * included -- into a slot and signals an mbarrier; every cell value is read
 * from HBM/L2 once per plane per CTA instead of once per stencil tap.
 *
 * Two warp groups share every cell (256 threads for 128 cells): warps 0-3
 * evaluate the stencils of lnrho and uu and the continuity and momentum
 * equations, warps 4-7 those of aa and entropy and the induction and entropy
 * equations; the two exchange 11 + 9 values per cell through shared memory
 * (6 + 9 in FP64, where the magnetic group reads u and forms exp(-lnrho) and
 * the sound-speed exponential itself)
 * between the halves of the RHS.  This doubles the warps per SM (the plane
 * ring fills the SM's shared memory, so one CTA fits) without extra loads.
 * The per-cell arithmetic is the one of the plain kernel in solve.cu.  Reference:
 * singlepass_solve / twopass_solve_intermediate,
 * acc-runtime/samples/mhd_modular/mhdsolver.ac:524-612 (the reference issues
 * every tap as a separate __ldg, acc-runtime/acc/stencilgen.c:2205).
 *
 * Waits on mbarriers are bounded: a wait that gives up sets *err and the
 * kernel still runs to completion (all threads take the same path, so no
 * __syncthreads is skipped); the host turns *err into AC_FAILURE.
 */
#include <cuda.h>

#include "internal.h"
#include "mhd_rhs.cuh"
#include "tma_ring.cuh"

namespace {

using namespace tma_ring;

constexpr int TX     = 32;
constexpr int TY     = 4;
constexpr int HY     = TY + 2 * NGHOST;
constexpr int RING   = 8;
constexpr int ZCHUNK = 64;
constexpr int NCELL  = TX * TY; /* cells per tile, one per thread of a group */
constexpr int XCHG   = (AC_H2M_COUNT + AC_M2H_COUNT) * NCELL; /* exchange entries */

template <typename T>
struct Tile;
template <>
struct Tile<double> {
    static constexpr int HXP  = TX + 2 * NGHOST; /* 38 x 8 B = 304 B rows */
    static constexpr int MINB = 1;
};
template <>
struct Tile<float> {
    static constexpr int HXP  = 40; /* 38 rounded up: 160 B rows */
    static constexpr int MINB = 2;
};

template <typename T>
struct Layout {
    static constexpr int HXP        = Tile<T>::HXP;
    static constexpr int PLANE      = HXP * HY;    /* elements per field per plane */
    static constexpr int SLOT       = AC_NF * PLANE; /* elements per ring slot */
    static constexpr unsigned SLOT_BYTES = SLOT * sizeof(T);
    static constexpr size_t SMEM_BYTES   = (size_t)RING * SLOT_BYTES + (size_t)XCHG * sizeof(T) +
                                         RING * sizeof(uint64_t);
};

/* Taps of field q at offset (dx, dy, dz) from this thread's cell. */
template <typename T>
struct Taps {
    const T* s;
    int off[7]; /* per dz = -3..3: slot base + this thread's (x, y) position */
    __device__ __forceinline__ T operator()(const int q, const int dx, const int dy,
                                            const int dz) const
    {
        return s[off[dz + 3] + q * Layout<T>::PLANE + dy * Layout<T>::HXP + dx];
    }
};

template <int A, typename T>
__device__ __forceinline__ T
tap1(const Taps<T>& t, const int q, const int k)
{
    return A == 0 ? t(q, k, 0, 0) : A == 1 ? t(q, 0, k, 0) : t(q, 0, 0, k);
}

template <int A, typename T>
__device__ __forceinline__ T
d1(const Taps<T>& t, const int q, const T* c)
{
    T r = c[0] * (tap1<A>(t, q, 1) - tap1<A>(t, q, -1));
    r   = fma(c[1], tap1<A>(t, q, 2) - tap1<A>(t, q, -2), r);
    r   = fma(c[2], tap1<A>(t, q, 3) - tap1<A>(t, q, -3), r);
    return r;
}

template <int A, typename T>
__device__ __forceinline__ T
d2_sides(const Taps<T>& t, const int q, const T* d)
{
    T r = d[1] * (tap1<A>(t, q, 1) + tap1<A>(t, q, -1));
    r   = fma(d[2], tap1<A>(t, q, 2) + tap1<A>(t, q, -2), r);
    r   = fma(d[3], tap1<A>(t, q, 3) + tap1<A>(t, q, -3), r);
    return r;
}

/* upwinding derivative along axis A: u_0 f + sum_k u_k (f[+k] + f[-k]) */
template <int A, typename T>
__device__ __forceinline__ T
dup(const Taps<T>& t, const int q, const T* u)
{
    T r = u[0] * t(q, 0, 0, 0);
    r   = fma(u[1], tap1<A>(t, q, 1) + tap1<A>(t, q, -1), r);
    r   = fma(u[2], tap1<A>(t, q, 2) + tap1<A>(t, q, -2), r);
    r   = fma(u[3], tap1<A>(t, q, 3) + tap1<A>(t, q, -3), r);
    return r;
}

/* tap at +a along axis A and +b along axis B (A < B) */
template <int A, int B, typename T>
__device__ __forceinline__ T
tap2(const Taps<T>& t, const int q, const int a, const int b)
{
    if (A == 0 && B == 1)
        return t(q, a, b, 0);
    if (A == 0 && B == 2)
        return t(q, a, 0, b);
    return t(q, 0, a, b);
}

template <int A, int B, typename T>
__device__ __forceinline__ T
dmix(const Taps<T>& t, const int q, const T* e)
{
    T r = 0;
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
        const T s = (tap2<A, B>(t, q, k, k) + tap2<A, B>(t, q, -k, -k)) -
                    (tap2<A, B>(t, q, k, -k) + tap2<A, B>(t, q, -k, k));
        r = k == 1 ? e[0] * s : fma(e[k - 1], s, r);
    }
    return r;
}

template <typename T>
__device__ __forceinline__ void
scal_derivs(const Taps<T>& t, const int q, const StencilT<T>& sc, ScalD<T>& o)
{
    o.v    = t(q, 0, 0, 0);
    o.g[0] = d1<0>(t, q, sc.d1[0]);
    o.g[1] = d1<1>(t, q, sc.d1[1]);
    o.g[2] = d1<2>(t, q, sc.d1[2]);
    o.lap  = (sc.d2[0][0] + sc.d2[1][0] + sc.d2[2][0]) * o.v + d2_sides<0>(t, q, sc.d2[0]) +
            d2_sides<1>(t, q, sc.d2[1]) + d2_sides<2>(t, q, sc.d2[2]);
}

/* scal_derivs with the z-line of the field (planes z-3 .. z+3 at this
 * thread's cell) from registers */
template <typename T>
__device__ __forceinline__ void
scal_derivs_zq(const Taps<T>& t, const int q, const StencilT<T>& sc, const T zq[7], ScalD<T>& o)
{
    o.v    = zq[3];
    o.g[0] = d1<0>(t, q, sc.d1[0]);
    o.g[1] = d1<1>(t, q, sc.d1[1]);
    {
        const T* c = sc.d1[2];
        T r = c[0] * (zq[4] - zq[2]);
        r   = fma(c[1], zq[5] - zq[1], r);
        r   = fma(c[2], zq[6] - zq[0], r);
        o.g[2] = r;
    }
    T s2;
    {
        const T* d = sc.d2[2];
        T r = d[1] * (zq[4] + zq[2]);
        r   = fma(d[2], zq[5] + zq[1], r);
        r   = fma(d[3], zq[6] + zq[0], r);
        s2 = r;
    }
    o.lap  = (sc.d2[0][0] + sc.d2[1][0] + sc.d2[2][0]) * o.v + d2_sides<0>(t, q, sc.d2[0]) +
            d2_sides<1>(t, q, sc.d2[1]) + s2;
}

template <typename T>
__device__ __forceinline__ void
vec_derivs(const Taps<T>& t, const int q0, const StencilT<T>& sc, VecD<T>& o)
{
    T diag[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int q = q0 + c;
        o.v[c]      = t(q, 0, 0, 0);
        o.g[c][0]   = d1<0>(t, q, sc.d1[0]);
        o.g[c][1]   = d1<1>(t, q, sc.d1[1]);
        o.g[c][2]   = d1<2>(t, q, sc.d1[2]);
        const T s0  = d2_sides<0>(t, q, sc.d2[0]);
        const T s1  = d2_sides<1>(t, q, sc.d2[1]);
        const T s2  = d2_sides<2>(t, q, sc.d2[2]);
        diag[c]     = sc.d2[c][0] * o.v[c] + (c == 0 ? s0 : c == 1 ? s1 : s2);
        o.lap[c]    = (sc.d2[0][0] + sc.d2[1][0] + sc.d2[2][0]) * o.v[c] + s0 + s1 + s2;
    }
    o.gd[0] = diag[0] + dmix<0, 1>(t, q0 + 1, sc.mix[0]) + dmix<0, 2>(t, q0 + 2, sc.mix[1]);
    o.gd[1] = dmix<0, 1>(t, q0, sc.mix[0]) + diag[1] + dmix<1, 2>(t, q0 + 2, sc.mix[2]);
    o.gd[2] = dmix<0, 2>(t, q0, sc.mix[1]) + dmix<1, 2>(t, q0 + 1, sc.mix[2]) + diag[2];
}

template <typename T, bool COMP, bool UPWD>
__global__ void __launch_bounds__(2 * TX * TY, Tile<T>::MINB)
solve_tiled_kernel(const __grid_constant__ CUtensorMap tmap, const Geom g, const FieldsT<T> f,
                   const StencilT<T> sc, const PhysConst pc, const RkCoef rk, int* err,
                   unsigned long long* cfl, const int zchunk)
{
    typedef Layout<T> L;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* smem        = reinterpret_cast<T*>(smem_raw);
    T* xh          = smem + (size_t)RING * L::SLOT;      /* hydro -> magnetic, [value][cell] */
    T* xm          = xh + (size_t)AC_H2M_COUNT * NCELL;  /* magnetic -> hydro */
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + (size_t)RING * L::SLOT_BYTES +
                                                 (size_t)XCHG * sizeof(T));
    const int lx    = threadIdx.x;
    const int ly    = threadIdx.y & (TY - 1);
    const int group = threadIdx.y / TY; /* 0: lnrho + uu, 1: aa + entropy (warp uniform) */
    const int tid   = threadIdx.y * TX + lx;
    const int cell  = ly * TX + lx;
    const int x0    = blockIdx.x * TX;
    const int y0    = blockIdx.y * TY;
    const int z0    = blockIdx.z * zchunk;
    const int z1    = min(z0 + zchunk, g.nz);
    const int pfirst = z0 - NGHOST;     /* first plane needed (interior z index) */
    const int plast  = z1 - 1 + NGHOST; /* last plane needed */

    if (tid == 0) {
        for (int s = 0; s < RING; ++s)
            mbar_init(&bars[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0) {
        const int pend = min(plast, pfirst + RING - 1);
        for (int p = pfirst; p <= pend; ++p) {
            const int s = (p - pfirst) & (RING - 1);
            mbar_arrive_expect_tx(&bars[s], L::SLOT_BYTES);
            tma_load_plane(smem + (size_t)s * L::SLOT, &tmap, &bars[s], x0, y0, p + NGHOST);
        }
    }

    const int x = x0 + lx, y = y0 + ly;
    const bool active  = x < g.nx && y < g.ny;
    const bool use_prev = rk.step > 0;
    const PhysT<T> p   = phys_cast<T>(pc);
    const int cell_off = (ly + NGHOST) * L::HXP + (lx + NGHOST);
    /* the 4 fields of this group, selected with constant indices (a runtime
     * index into the by-value parameter arrays would copy them to the stack) */
    T* outp[4];
    T* outl[4];
    const T* inl[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        outp[k] = group == 0 ? f.out[k] : f.out[4 + k];
        outl[k] = group == 0 ? f.out_lo[k] : f.out_lo[4 + k];
        inl[k]  = group == 0 ? f.in_lo[k] : f.in_lo[4 + k];
    }
    bool ok    = true;
    int waited = pfirst - 1;
    T cm[3]    = {0, 0, 0}; /* CFL maxima of this thread (substep 2 only) */
    /* the group's scalar field (lnrho or entropy) at this cell, planes z-3 ..
     * z+3, shifted by one plane per step: its z taps come from registers, 6
     * shared-memory loads fewer per cell and field */
    T zq[7];
    const int qs = group == 0 ? VTXBUF_LNRHO : VTXBUF_ENTROPY;

    for (int z = z0; z < z1; ++z) {
        const long long idx = geom_idx(g, x + NGHOST, y + NGHOST, z + NGHOST);
        /* previous-substep values (and compensation terms), loaded early so
         * their latency hides behind the stencils */
        T prev[4] = {0, 0, 0, 0}, prevl[4] = {0, 0, 0, 0}, lo[4] = {0, 0, 0, 0};
        if (active) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (use_prev)
                    prev[k] = outp[k][idx];
                if (COMP) {
                    lo[k] = inl[k][idx];
                    if (use_prev)
                        prevl[k] = outl[k][idx];
                }
            }
        }
        for (int q = waited + 1; q <= z + NGHOST; ++q) {
            const int s = (q - pfirst) & (RING - 1);
            /* after one failed wait the kernel stops waiting and only runs out */
            if (ok)
                ok = mbar_wait_bounded(&bars[s], (unsigned)(((q - pfirst) / RING) & 1));
        }
        waited = z + NGHOST;

        Taps<T> t;
        t.s = smem;
#pragma unroll
        for (int k = 0; k < 7; ++k)
            t.off[k] = ((z - NGHOST + k - pfirst) & (RING - 1)) * L::SLOT + cell_off;
        if (z == z0) {
#pragma unroll
            for (int k = 0; k < 7; ++k)
                zq[k] = t(qs, 0, 0, k - 3);
        }
        else {
#pragma unroll
            for (int k = 0; k < 6; ++k)
                zq[k] = zq[k + 1];
            zq[6] = t(qs, 0, 0, 3);
        }

        ScalD<T> sd;
        VecD<T> vd;
        HydroToMag<T> hx;
        MagToHydro<T> mx;
        Strain<T> st;
        T upr[4] = {0, 0, 0, 0}; /* upwinding terms of the hydro rates (UPWD) */
        if (active) {
            if (group == 0) {
                scal_derivs_zq(t, VTXBUF_LNRHO, sc, zq, sd);
                vec_derivs(t, VTXBUF_UUX, sc, vd);
                hydro_prepare(sd, t(VTXBUF_ENTROPY, 0, 0, 0), vd, p, hx, st);
                if constexpr (UPWD) {
                    const T up_l[3] = {dup<0>(t, VTXBUF_LNRHO, sc.up[0]),
                                       dup<1>(t, VTXBUF_LNRHO, sc.up[1]),
                                       dup<2>(t, VTXBUF_LNRHO, sc.up[2])};
                    T up_u[3][3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        up_u[c][0] = dup<0>(t, VTXBUF_UUX + c, sc.up[0]);
                        up_u[c][1] = dup<1>(t, VTXBUF_UUX + c, sc.up[1]);
                        up_u[c][2] = dup<2>(t, VTXBUF_UUX + c, sc.up[2]);
                    }
                    upwind_terms(up_l, up_u, vd.v, upr);
                }
                /* FP64: the magnetic group reads u and computes the two
                 * exponentials itself, so only entries H2M_GL .. H2M_DIVU cross */
                constexpr int k0 = sizeof(T) == 8 ? H2M_GL : 0;
                constexpr int k1 = sizeof(T) == 8 ? H2M_DIVU + 1 : AC_H2M_COUNT;
#pragma unroll
                for (int k = k0; k < k1; ++k)
                    xh[k * NCELL + cell] = hx.a[k];
            }
            else {
                scal_derivs_zq(t, VTXBUF_ENTROPY, sc, zq, sd);
                vec_derivs(t, VTXBUF_AX, sc, vd);
                mag_prepare(sd, vd, p, mx);
                if constexpr (sizeof(T) == 8) {
                    /* the expressions of hydro_prepare, so the bits are the same;
                     * fewer shared-memory accesses than the exchange (6 per cell),
                     * for two more exponentials on the FP64 pipe, which has room */
                    const T lv        = t(VTXBUF_LNRHO, 0, 0, 0);
                    const T arg       = p.gamma_inv_cp * sd.v + p.gamma_m1 * (lv - p.lnrho0);
                    hx.a[H2M_E]       = ac_exp(arg);
                    hx.a[H2M_INV_RHO] = ac_exp(-lv);
                    hx.a[H2M_U + 0]   = t(VTXBUF_UUX, 0, 0, 0);
                    hx.a[H2M_U + 1]   = t(VTXBUF_UUY, 0, 0, 0);
                    hx.a[H2M_U + 2]   = t(VTXBUF_UUZ, 0, 0, 0);
                }
#pragma unroll
                for (int k = 0; k < AC_M2H_COUNT; ++k)
                    xm[k * NCELL + cell] = mx.a[k];
            }
        }
        __syncthreads(); /* exchange records written */
        if (active) {
            T r[4], val[4];
            if (group == 0) {
#pragma unroll
                for (int k = 0; k < AC_M2H_COUNT; ++k)
                    mx.a[k] = xm[k * NCELL + cell];
                hydro_rates(sd, vd, st, hx, mx, p, r);
                if constexpr (UPWD) {
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        r[k] += upr[k];
                }
                val[0] = sd.v;
                val[1] = vd.v[0];
                val[2] = vd.v[1];
                val[3] = vd.v[2];
            }
            else {
                constexpr int k0 = sizeof(T) == 8 ? H2M_GL : 0;
                constexpr int k1 = sizeof(T) == 8 ? H2M_DIVU + 1 : AC_H2M_COUNT;
#pragma unroll
                for (int k = k0; k < k1; ++k)
                    hx.a[k] = xh[k * NCELL + cell];
                mag_rates(sd, vd, mx, hx, p, r);
                if (cfl) {
                    const T* u = &hx.a[H2M_U];
                    const T* B = &mx.a[M2H_B];
                    cfl_accumulate(u[0] * u[0] + u[1] * u[1] + u[2] * u[2],
                                   B[0] * B[0] + B[1] * B[1] + B[2] * B[2], hx.a[H2M_INV_RHO],
                                   p.cs2_sound, cm);
                }
                val[0] = vd.v[0];
                val[1] = vd.v[1];
                val[2] = vd.v[2];
                val[3] = sd.v;
            }
            /* group 0 writes lnrho, ux, uy, uz; group 1 writes ax, ay, az, entropy */
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if constexpr (COMP) {
                    const RkT32 c = {(float)rk.dt, (float)rk.beta, (float)rk.ab};
                    float oh, ol;
                    rk_update_comp(val[k], lo[k], prev[k], prevl[k], r[k], c, use_prev, oh, ol);
                    outp[k][idx] = oh;
                    outl[k][idx] = ol;
                }
                else {
                    const RkT64 c = {rk.dt, rk.beta, rk.ab};
                    double o;
                    rk_update(val[k], prev[k], r[k], c, use_prev, o);
                    outp[k][idx] = o;
                }
            }
        }
        __syncthreads(); /* every thread is done with plane z - 3 and the exchange */
        const int next = z - NGHOST + RING;
        if (tid == 0 && next <= plast) {
            const int s = (next - pfirst) & (RING - 1);
            mbar_arrive_expect_tx(&bars[s], L::SLOT_BYTES);
            tma_load_plane(smem + (size_t)s * L::SLOT, &tmap, &bars[s], x0, y0, next + NGHOST);
        }
    }
    if (cfl)
        cfl_commit(cm, xh, cfl); /* the exchange area is free after the last barrier */
    if (!ok)
        atomicExch(err, 1);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn
encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

/* Planes per CTA: ZCHUNK, halved (down to 8) while the grid would have fewer
 * than two CTAs per SM of the 148.  Every chunk reads 6 halo planes beyond its
 * own, so long chunks are cheaper where the grid is large enough. */
int
zchunk_for(const Geom& g)
{
    const long long tiles = (long long)((g.nx + TX - 1) / TX) * ((g.ny + TY - 1) / TY);
    int zc                = ZCHUNK;
    while (zc > 8 && tiles * ((g.nz + zc - 1) / zc) < 2 * 148)
        zc /= 2;
    return zc;
}

template <typename T, bool COMP>
cudaError_t
launch_tiled(const Geom& g, const void* tmap_in, const FieldsT<T>& f, const StencilCoef& sc,
             const PhysConst& pc, const RkCoef& rk, int* err, unsigned long long* cfl,
             cudaStream_t stream, unsigned long long* launches)
{
    const dim3 tpb(TX, 2 * TY, 1);
    const int zc = zchunk_for(g);
    const dim3 bpg((g.nx + TX - 1) / TX, (g.ny + TY - 1) / TY, (g.nz + zc - 1) / zc);
    if (pc.upwind)
        solve_tiled_kernel<T, COMP, true><<<bpg, tpb, Layout<T>::SMEM_BYTES, stream>>>(
            *(const CUtensorMap*)tmap_in, g, f, stencil_cast<T>(sc), pc, rk, err, cfl, zc);
    else
        solve_tiled_kernel<T, COMP, false><<<bpg, tpb, Layout<T>::SMEM_BYTES, stream>>>(
            *(const CUtensorMap*)tmap_in, g, f, stencil_cast<T>(sc), pc, rk, err, cfl, zc);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

} // namespace

bool
ac_tiled_supported(const Geom& g, const int precision)
{
    /* TMA: global strides must be multiples of 16 bytes and the box must not
     * exceed the tensor, whose rows are the px-element pitch (px >= box width,
     * my >= 10; an FP32 row of mx = 38 has px = 40, so 32^3 meshes qualify). */
    const int esz = precision == 0 ? 8 : 4;
    const int hxp = precision == 0 ? Tile<double>::HXP : Tile<float>::HXP;
    return ((long long)g.px * esz) % 16 == 0 && g.px >= hxp && g.my >= HY && g.nx >= TX &&
           g.ny >= TY;
}

bool
ac_encode_field_map(void* map_out, void* base, const Geom& g, const int precision,
                    const unsigned box_x, const unsigned box_y)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn)
        return false;
    const size_t esz            = precision == 0 ? sizeof(double) : sizeof(float);
    /* rows of px elements: the padding of FP32 rows (px - mx <= 3 elements,
     * allocated and never written) may be read into unused box columns */
    const cuuint64_t dims[4]    = {(cuuint64_t)g.px, (cuuint64_t)g.my, (cuuint64_t)g.mz,
                                   (cuuint64_t)AC_NF};
    const cuuint64_t strides[3] = {(cuuint64_t)g.px * esz, (cuuint64_t)g.pxy * esz,
                                   (cuuint64_t)g.cells * esz};
    const cuuint32_t box[4]     = {box_x, box_y, 1, AC_NF};
    const cuuint32_t estr[4]    = {1, 1, 1, 1};
    const CUresult r =
        fn((CUtensorMap*)map_out,
           precision == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
           base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool
ac_make_tensor_map(void* map_out, void* base, const Geom& g, const int precision)
{
    if (!ac_tiled_supported(g, precision))
        return false;
    const unsigned hxp = precision == 0 ? Tile<double>::HXP : Tile<float>::HXP;
    return ac_encode_field_map(map_out, base, g, precision, hxp, HY);
}

/* Opts the kernel in to its dynamic shared memory on the current device; called
 * by acDeviceCreate, outside any stream capture. */
cudaError_t
ac_solve_tiled_init(const int precision)
{
    /* both variants (with and without the upwinding terms) */
    if (precision == 0) {
        const cudaError_t e = cudaFuncSetAttribute(solve_tiled_kernel<double, false, false>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)Layout<double>::SMEM_BYTES);
        if (e != cudaSuccess)
            return e;
        return cudaFuncSetAttribute(solve_tiled_kernel<double, false, true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)Layout<double>::SMEM_BYTES);
    }
    const cudaError_t e = cudaFuncSetAttribute(solve_tiled_kernel<float, true, false>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)Layout<float>::SMEM_BYTES);
    if (e != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(solve_tiled_kernel<float, true, true>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)Layout<float>::SMEM_BYTES);
}

cudaError_t
ac_launch_solve_tiled64(const Geom& g, const void* tmap_in, const Fields64& f,
                        const StencilCoef& sc, const PhysConst& pc, const RkCoef& rk, int* err,
                        unsigned long long* cfl, cudaStream_t stream,
                        unsigned long long* launches)
{
    return launch_tiled<double, false>(g, tmap_in, f, sc, pc, rk, err, cfl, stream, launches);
}

cudaError_t
ac_launch_solve_tiled32(const Geom& g, const void* tmap_in, const Fields32& f,
                        const StencilCoef& sc, const PhysConst& pc, const RkCoef& rk, int* err,
                        unsigned long long* cfl, cudaStream_t stream,
                        unsigned long long* launches)
{
    return launch_tiled<float, true>(g, tmap_in, f, sc, pc, rk, err, cfl, stream, launches);
}
