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
#include "tmem.cuh"

namespace {

using namespace tma_ring;

constexpr int TX     = 32;
constexpr int TY     = 4;
constexpr int HY     = TY + 2 * NGHOST;
constexpr int RING   = 8;
constexpr int ZCHUNK = 512; /* the longest z chunk (zchunk_for) */
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

/* Number of plane loads issued into ring slot sl for the planes pfirst .. plast
 * (plane p goes to slot (p - pfirst) mod RING), without plast when skipped. */
__device__ __forceinline__ int
loads_into(const int sl, const int pfirst, const int plast, const bool skip_last)
{
    const int np = plast - pfirst + 1;
    int n        = sl < np ? (np - 1 - sl) / RING + 1 : 0;
    if (skip_last && ((plast - pfirst) & (RING - 1)) == sl)
        --n;
    return n;
}

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
    const int z0    = pc.zlo + (int)blockIdx.z * zchunk;
    const int z1    = min(z0 + zchunk, pc.zhi);
    const int pfirst = z0 - NGHOST;     /* first plane needed (interior z index) */
    const int plast  = z1 - 1 + NGHOST; /* last plane needed */

    if (tid == 0) {
        for (int s = 0; s < RING; ++s)
            mbar_init(&bars[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    /* the fault-path test switch skips the load of plane plast */
    const bool skip_last  = pc.debug_skip_load != 0;
    const long long wlim  = skip_last ? kDebugWaitLimit : kWaitLimit;
    if (tid == 0) {
        const int pend = min(plast, pfirst + RING - 1);
        for (int p = pfirst; p <= pend; ++p) {
            if (skip_last && p == plast)
                continue;
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
                ok = mbar_wait_bounded(&bars[s], (unsigned)(((q - pfirst) / RING) & 1), wlim);
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
                                   p.cs2_sound, cm, pc.cfl_sum != 0);
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
        if (tid == 0 && next <= plast && !(skip_last && next == plast)) {
            const int s = (next - pfirst) & (RING - 1);
            mbar_arrive_expect_tx(&bars[s], L::SLOT_BYTES);
            tma_load_plane(smem + (size_t)s * L::SLOT, &tmap, &bars[s], x0, y0, next + NGHOST);
        }
    }
    if (cfl)
        cfl_commit(cm, xh, cfl); /* the exchange area is free after the last barrier */
    if (!ok)
        atomicExch(err, 1);
    if (tid == 0)
        drain_ring(bars, RING, [&](const int sl) { return loads_into(sl, pfirst, plast, skip_last); });
}

/* ---------------------------------------------------------------------------
 * The leading-plane substep kernel: the production path for meshes without
 * the upwinding terms.
 *
 * Same tiles, plane ring, warp groups and RHS as solve_tiled_kernel, with the
 * stencils reorganised so that each in-plane tap is read from shared memory
 * once and serves every derivative that needs it:
 *
 * * When plane L arrives, each thread forms the x and y differences
 *   D^k f = f(+k) - f(-k) and sums S^k = f(+k) + f(-k) (k = 1..3) of its
 *   group's fields at its cell, and from them the in-plane first and second
 *   derivatives and the diagonal xy mixed derivatives of plane L.  These 17
 *   values per group (its record) go to tensor memory (TMEM), a 3-slot delay
 *   line in the thread's own lane, and come back when plane L is solved three
 *   planes later (the z stencils need planes up to z + 3 first).
 * * The xz and yz mixed derivatives use the separable form of the diagonal
 *   stencil (derivs.h:591-690):  D_az f(z) = sum_k e_k [D_a^k f(z+k) - D_a^k f(z-k)]
 *   with a = x or y.  The differences D_a^k at plane L are the ones just
 *   formed, so each mixed derivative costs no further shared-memory reads:
 *   plane L adds +e_k D^k to the sum of plane L-k and -e_k D^k to that of
 *   plane L+k, in seven running sums per mixed term held in registers.  Only
 *   the combinations grad(div) needs are formed: D_xz uz, D_yz uz and
 *   D_xz ux + D_yz uy (and the same for aa).
 * * The z lines: the scalar field's in registers; the vector components' in a
 *   TMEM queue of the last seven planes, written when a plane arrives (its
 *   value at the thread's cell, three values per group) and read back as
 *   planes z-3 .. z+2 in one load when z is solved.  The queue holds each plane
 *   twice, at entries e and e + 7 (e = plane mod 7), so that the window is
 *   always one contiguous run of entries and its register positions are fixed.
 *   The magnetic group reads u at plane z from the hydro group's queue.
 * * A plane is read from shared memory only in the step it arrives.
 *
 * Per cell and substep this reads ~155 values from shared memory instead of
 * ~320.  The arithmetic per cell is the same up to association (the mixed
 * derivatives are summed in a different order), so results agree with the
 * other kernels to rounding, not bit for bit.
 * ------------------------------------------------------------------------- */
template <typename T>
struct LeadTm;
template <>
struct LeadTm<double> {
    static constexpr uint32_t NCOLS = 512; /* 1 block per SM */
    static constexpr uint32_t GROUP = 256; /* columns per warp group */
};
template <>
struct LeadTm<float> {
    static constexpr uint32_t NCOLS = 256; /* 2 blocks per SM */
    static constexpr uint32_t GROUP = 128;
};

/* record of one plane and warp group (index: value) */
constexpr int NREC      = 17;
constexpr int REC_SD1X  = 0;  /* scalar d/dx */
constexpr int REC_SD1Y  = 1;  /* scalar d/dy */
constexpr int REC_SLAP  = 2;  /* scalar second-derivative side sums, x + y */
constexpr int REC_V     = 3;  /* + 4c + {0: d/dx, 1: d/dy, 2: x sides, 3: y sides} of component c */
constexpr int REC_DXY0  = 15; /* D_xy of component 0 (enters grad div, y) */
constexpr int REC_DXY1  = 16; /* D_xy of component 1 (enters grad div, x) */

/* A warp group's TMEM columns (32-bit words; WE per value), in its own lanes:
 *   records   3 slots (plane mod 3) of NREC values; the record of plane z is
 *             read back in the step that stores plane z + 3's into the same
 *             slot, after the read has completed;
 *   EXP       4 slots (plane mod 4) of the group's exponential (group 0:
 *             exp(-lnrho), group 1: exp(gamma s/cp + (gamma-1)(lnrho - lnrho0))),
 *             which the other group reads three planes later;
 *   XCH       the exchange between the groups, two buffers (plane parity) of up
 *             to nine values;
 *   ZQ        the z queue: 14 entries of the three vector components. */
template <typename T>
struct LeadCols {
    static constexpr uint32_t WE    = (uint32_t)sizeof(T) / 4;
    static constexpr uint32_t REC_W = NREC * WE;
    static constexpr uint32_t EXP0  = 3 * REC_W;
    static constexpr uint32_t XCH0  = EXP0 + 4 * WE;
    static constexpr uint32_t XCH_W = 9 * WE;
    static constexpr uint32_t ZQ0   = XCH0 + 2 * XCH_W;
    static constexpr uint32_t ZQ_E  = 3 * WE;
    static constexpr uint32_t END   = ZQ0 + 14 * ZQ_E;
    static_assert(END <= LeadTm<T>::GROUP, "TMEM columns of a warp group");
};

/* queue entry of plane p >= -NGHOST */
__device__ __forceinline__ uint32_t
zq_entry(const int p)
{
    return (uint32_t)(p + NGHOST) % 7u;
}

/* Shared memory of the leading-plane kernel: the plane ring, the group
 * exchange through shared memory in two buffers (alternate planes; none when
 * the exchange goes through TMEM), 256 B for the CFL commit, the ring's
 * mbarriers and the TMEM base address. */
constexpr int XROWS = 15; /* exchange rows: 6 hydro -> magnetic, 9 magnetic -> hydro */
template <typename T, bool XT>
struct LeadSmem {
    static constexpr size_t RING_B = (size_t)RING * Layout<T>::SLOT_BYTES;
    static constexpr size_t XCH_B  = XT ? 0 : 2 * (size_t)XROWS * NCELL * sizeof(T);
    static constexpr size_t RED_B  = 256;
    static constexpr size_t BAR_OFF = RING_B + XCH_B + RED_B;
    static constexpr size_t BYTES  = BAR_OFF + RING * sizeof(uint64_t) + 16;
};
template <typename T, bool XT>
constexpr size_t lead_smem_bytes()
{
    return LeadSmem<T, XT>::BYTES;
}

/* The exchange between the warp groups through tensor memory (the default):
 * group 0's six values (grad lnrho, lap lnrho, S:S, div u) and group 1's nine
 * (grad s, j, B), each group's in its own XCH columns. */

/* differences and sums of one field along x (or y) at this cell of a plane:
 * p points at the field's value there; step is 1 (x) or the row pitch (y) */
template <typename T>
__device__ __forceinline__ void
diffs(const T* p, const int step, T d[3])
{
#pragma unroll
    for (int k = 1; k <= 3; ++k)
        d[k - 1] = p[k * step] - p[-k * step];
}

template <typename T>
__device__ __forceinline__ void
diffs_sums(const T* p, const int step, T d[3], T s[3])
{
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
        const T a = p[k * step], b = p[-k * step];
        d[k - 1]  = a - b;
        s[k - 1]  = a + b;
    }
}

template <typename T>
__device__ __forceinline__ T
d1_from(const T d[3], const T* c)
{
    T r = c[0] * d[0];
    r   = fma(c[1], d[1], r);
    r   = fma(c[2], d[2], r);
    return r;
}

template <typename T>
__device__ __forceinline__ T
d2s_from(const T s[3], const T* c)
{
    T r = c[1] * s[0];
    r   = fma(c[2], s[1], r);
    r   = fma(c[3], s[2], r);
    return r;
}

/* diagonal xy mixed derivative at this cell of a plane (12 taps) */
template <typename T>
__device__ __forceinline__ T
dxy_at(const T* p, const T* e)
{
    constexpr int H = Layout<T>::HXP;
    T r             = 0;
#pragma unroll
    for (int k = 1; k <= 3; ++k) {
        const T s = (p[k + k * H] + p[-k - k * H]) - (p[k - k * H] + p[-k + k * H]);
        r         = k == 1 ? e[0] * s : fma(e[k - 1], s, r);
    }
    return r;
}

template <bool I, bool S>
struct LeadPhase {
    static constexpr bool interior = I; /* the plane arriving is interior: its record is kept */
    static constexpr bool solve    = S; /* plane lp - 3 is solved in this step */
};

/* The whole chunk for the threads of one warp group (GROUP 0: lnrho and uu,
 * GROUP 1: aa and entropy).  Both groups take the same barriers in the same
 * order. */
/* MODE: which of the substep's options are fixed at compile time.
 * MODE_FIRST is substep 0 (no previous state read, no CFL maxima); MODE_RUNTIME
 * takes both from rk.step and the cfl pointer.  (Forms fixed for substeps 1
 * and 2 were measured too: in FP64 they take 228-230 registers against 224
 * and ran 2-3% slower; in FP32 they were even.) */
enum {
    MODE_FIRST   = 0,
    MODE_PREV    = 1,
    MODE_PREVCFL = 2,
    MODE_RUNTIME = 3
};

template <typename T, bool COMP, int GROUP, bool XT, int MODE>
__device__ __forceinline__ void
lead_group(const CUtensorMap* tmap, const Geom& g, const FieldsT<T>& f, const StencilT<T>& sc,
           const PhysT<T>& p, const RkCoef& rk, int* err, unsigned long long* cfl, T* smem, T* xch,
           T* red, uint64_t* bars, const uint32_t tcol, const int zchunk, const int zlo,
           const int zhi, const bool skip_last, const bool cfl_sum)
{
    const long long wlim = skip_last ? kDebugWaitLimit : kWaitLimit;
    typedef Layout<T> L;
    typedef LeadTm<T> TM;
    typedef LeadCols<T> LC;
    constexpr int QS = GROUP == 0 ? VTXBUF_LNRHO : VTXBUF_ENTROPY;
    constexpr int Q0 = GROUP == 0 ? VTXBUF_UUX : VTXBUF_AX;
    /* the other group's columns in the same lanes */
    const uint32_t tother = GROUP == 0 ? tcol + TM::GROUP : tcol - TM::GROUP;
    const int lx     = threadIdx.x;
    const int ly     = threadIdx.y & (TY - 1);
    const int tid    = threadIdx.y * TX + lx;
    const int cell   = ly * TX + lx;
    const int x0     = blockIdx.x * TX;
    const int y0     = blockIdx.y * TY;
    const int z0     = zlo + (int)blockIdx.z * zchunk;
    const int z1     = min(z0 + zchunk, zhi);
    const int pfirst = z0 - NGHOST;
    const int plast  = z1 - 1 + NGHOST;
    const int x = x0 + lx, y = y0 + ly;
    const bool active   = x < g.nx && y < g.ny;
    const bool use_prev = MODE == MODE_RUNTIME ? rk.step > 0 : MODE != MODE_FIRST;
    const bool do_cfl   = MODE == MODE_RUNTIME ? cfl != nullptr : MODE == MODE_PREVCFL;
    const int cell_off  = (ly + NGHOST) * L::HXP + (lx + NGHOST);
    /* a cell outside the mesh (its stores are skipped) reads at the nearest cell
     * of the mesh, so that its loads need no branch */
    const int xg = min(x, g.nx - 1) + NGHOST, yg = min(y, g.ny - 1) + NGHOST;
    T* outp[4];
    T* outl[4];
    const T* inl[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        outp[k] = f.out[4 * GROUP + k];
        outl[k] = f.out_lo[4 * GROUP + k];
        inl[k]  = f.in_lo[4 * GROUP + k];
    }
    bool ok    = true;
    int waited = pfirst - 1;
    T cm[3]    = {0, 0, 0};
    T zq[7]    = {0, 0, 0, 0, 0, 0, 0}; /* the scalar field at this cell, planes z-3 .. z+3 */
    /* running sums of the z-coupled mixed terms of grad(div) of this group's
     * vector v for planes lp-3 .. lp+3: [0] D_xz v_z, [1] D_yz v_z,
     * [2] D_xz v_x + D_yz v_y */
    T acc[3][7];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int j = 0; j < 7; ++j)
            acc[a][j] = 0;
    /* the RK coefficients of the update, converted once */
    const RkT32 c32 = {(float)rk.dt, (float)rk.beta, (float)rk.ab};
    const RkT64 c64 = {rk.dt, rk.beta, rk.ab};
    /* plane lp mod 3 (record slot) and zq_entry(lp), stepped with lp (lp >= -3) */
    uint32_t r3 = (uint32_t)(pfirst + 3) % 3u;
    uint32_t q7 = zq_entry(pfirst);

    auto step = [&](auto ph, const int lp) {
        constexpr bool INTERIOR = decltype(ph)::interior;
        constexpr bool SOLVE    = decltype(ph)::solve;
        const int z             = lp - NGHOST; /* the plane solved in this step */
        const long long idx     = geom_idx(g, xg, yg, z + NGHOST);
        /* prev only after substep 0 */
        T prev[4], prevl[4], lo[4];
        if constexpr (SOLVE) {
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
        for (int q = waited + 1; q <= lp; ++q) {
            const int s = (q - pfirst) & (RING - 1);
            if (ok)
                ok = mbar_wait_bounded(&bars[s], (unsigned)(((q - pfirst) / RING) & 1), wlim);
        }
        waited = lp;
        __syncwarp(); /* tensor-memory accesses below are warp-collective */

        /* record of plane z, stored three steps ago, and the two groups'
         * exponentials of plane z */
        tmem::Words<T, NREC> rz;
        tmem::Words<T, 1> eo, ro;
        if constexpr (SOLVE) {
            rz.load(tcol + r3 * LC::REC_W); /* z mod 3 = lp mod 3 */
            eo.load(tcol + LC::EXP0 + (uint32_t)(z & 3) * LC::WE);
            ro.load(tother + LC::EXP0 + (uint32_t)(z & 3) * LC::WE);
        }

        /* ---- plane lp: the z lines, then (now or after the barrier) the
         * in-plane differences, record and running mixed sums ---- */
        const T* pl = smem + (size_t)((lp - pfirst) & (RING - 1)) * L::SLOT + cell_off;
#pragma unroll
        for (int k = 0; k < 6; ++k)
            zq[k] = zq[k + 1];
        zq[6] = pl[QS * L::PLANE];
        /* the vector at this cell of plane lp: into the z queue (both copies) */
        tmem::Words<T, 3> cur;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            cur.set(c, pl[(Q0 + c) * L::PLANE]);
        {
            const uint32_t qa = tcol + LC::ZQ0 + q7 * LC::ZQ_E;
            cur.store(qa);
            cur.store(qa + 7 * LC::ZQ_E);
        }
        /* In a solve step the hydro group forms plane lp's in-plane part after
         * the exchange barrier, in one basic block with its rates: its prepare
         * needs neither grad div u nor plane lp's record, so its shared-memory
         * reads overlap the rates' FP64 work, and on each SM sub-partition the
         * two groups' warps are in different phases before the barrier.  (The
         * magnetic group's prepare needs grad div A of plane z, complete only
         * with plane lp's differences: it keeps the in-plane part first.
         * Measured at 512^3, FP64: 31.2 against 33.6 ms per step with both
         * groups in-plane first, 36.1 with both late.) */
        constexpr bool LATE_NOW = SOLVE && GROUP == 0;
        auto inplane = [&]() {
        T dvx[3], dvy[3], dzx[3], dzy[3]; /* D_x^k v_x, D_y^k v_y, D_x^k v_z, D_y^k v_z */
        if constexpr (INTERIOR) {
            tmem::Words<T, NREC> r;
            {
                const T* ps = pl + QS * L::PLANE;
                T d[3], s[3], e[3], t[3];
                diffs_sums(ps, 1, d, s);
                diffs_sums(ps, L::HXP, e, t);
                r.set(REC_SD1X, d1_from(d, sc.d1[0]));
                r.set(REC_SD1Y, d1_from(e, sc.d1[1]));
                r.set(REC_SLAP, d2s_from(s, sc.d2[0]) + d2s_from(t, sc.d2[1]));
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T* pv = pl + (Q0 + c) * L::PLANE;
                T d[3], s[3], e[3], t[3];
                diffs_sums(pv, 1, d, s);
                diffs_sums(pv, L::HXP, e, t);
                r.set(REC_V + 4 * c + 0, d1_from(d, sc.d1[0]));
                r.set(REC_V + 4 * c + 1, d1_from(e, sc.d1[1]));
                r.set(REC_V + 4 * c + 2, d2s_from(s, sc.d2[0]));
                r.set(REC_V + 4 * c + 3, d2s_from(t, sc.d2[1]));
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    if (c == 0)
                        dvx[k] = d[k];
                    if (c == 1)
                        dvy[k] = e[k];
                    if (c == 2) {
                        dzx[k] = d[k];
                        dzy[k] = e[k];
                    }
                }
            }
            r.set(REC_DXY0, dxy_at(pl + Q0 * L::PLANE, sc.mix[0]));
            r.set(REC_DXY1, dxy_at(pl + (Q0 + 1) * L::PLANE, sc.mix[0]));
            /* the RHS's two exponentials (the expressions of hydro_prepare), one
             * per group, off the solve's critical path; each group reads the
             * other's from the shared lane */
            tmem::Words<T, 1> ex;
            if constexpr (GROUP == 0) {
                ex.set(0, ac_exp(-zq[6]));
            }
            else {
                const T lv  = pl[VTXBUF_LNRHO * L::PLANE];
                const T arg = p.gamma_inv_cp * zq[6] + p.gamma_m1 * (lv - p.lnrho0);
                ex.set(0, ac_exp(arg));
            }
            ex.store(tcol + LC::EXP0 + (uint32_t)(lp & 3) * LC::WE);
            if constexpr (SOLVE) {
                /* plane z's record, in the slot plane lp's takes, is in registers */
                tmem::wait_ld();
                rz.tie();
                eo.tie();
                ro.tie();
            }
            r.store(tcol + r3 * LC::REC_W);
        }
        else {
            /* halo planes only feed the mixed sums */
            diffs(pl + Q0 * L::PLANE, 1, dvx);
            diffs(pl + (Q0 + 1) * L::PLANE, L::HXP, dvy);
            diffs(pl + (Q0 + 2) * L::PLANE, 1, dzx);
            diffs(pl + (Q0 + 2) * L::PLANE, L::HXP, dzy);
        }
#pragma unroll
        for (int k = 1; k <= 3; ++k) {
            const T exz = sc.mix[1][k - 1], eyz = sc.mix[2][k - 1];
            const T a0  = exz * dzx[k - 1];
            const T a1  = eyz * dzy[k - 1];
            const T a2  = fma(exz, dvx[k - 1], eyz * dvy[k - 1]);
            acc[0][3 - k] += a0;
            acc[0][3 + k] -= a0;
            acc[1][3 - k] += a1;
            acc[1][3 + k] -= a1;
            acc[2][3 - k] += a2;
            acc[2][3 + k] -= a2;
        }
        };
        if constexpr (!LATE_NOW)
            inplane();

        /* ---- plane z = lp - 3: the RHS and the RK update ---- */
        if constexpr (SOLVE) {
            /* planes z-3 .. z+2 of the vector from the queue (z+3 = lp is cur);
             * the magnetic group also takes u at plane z from the hydro group's */
            tmem::Words<T, 18> win;
            /* zq_entry(z - 3) = zq_entry(lp) + 1, zq_entry(z) = zq_entry(lp) + 4 (mod 7) */
            const uint32_t qw = q7 == 6u ? 0u : q7 + 1u;
            win.load(tcol + LC::ZQ0 + qw * LC::ZQ_E);
            [[maybe_unused]] tmem::Words<T, 3> uz;
            if constexpr (GROUP == 1)
                uz.load(tother + LC::ZQ0 + (q7 >= 3u ? q7 - 3u : q7 + 4u) * LC::ZQ_E);
            T sz1, sz2;
            {
                const T* c = sc.d1[2];
                T a        = c[0] * (zq[4] - zq[2]);
                a          = fma(c[1], zq[5] - zq[1], a);
                sz1        = fma(c[2], zq[6] - zq[0], a);
                const T* d = sc.d2[2];
                T b        = d[1] * (zq[4] + zq[2]);
                b          = fma(d[2], zq[5] + zq[1], b);
                sz2        = fma(d[3], zq[6] + zq[0], b);
            }
            tmem::wait_ld();
            rz.tie();
            eo.tie();
            ro.tie();
            win.tie();
            if constexpr (GROUP == 1)
                uz.tie();
            ScalD<T> sd;
            VecD<T> vd;
            T s2z[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                /* window entry e is plane z - 3 + e */
                const T m3 = win.get(c), m2 = win.get(3 + c), m1 = win.get(6 + c);
                const T p1 = win.get(12 + c), p2 = win.get(15 + c), p3 = cur.get(c);
                const T* c1 = sc.d1[2];
                const T* c2 = sc.d2[2];
                vd.v[c]     = win.get(9 + c);
                T a         = c1[0] * (p1 - m1);
                a           = fma(c1[1], p2 - m2, a);
                vd.g[c][2]  = fma(c1[2], p3 - m3, a);
                T b         = c2[1] * (p1 + m1);
                b           = fma(c2[2], p2 + m2, b);
                s2z[c]      = fma(c2[3], p3 + m3, b);
            }
            /* E = exp(gamma s/cp + (gamma-1)(lnrho - lnrho0)) and 1/rho = exp(-lnrho) */
            const T e_cs  = GROUP == 0 ? ro.get(0) : eo.get(0);
            const T e_irh = GROUP == 0 ? eo.get(0) : ro.get(0);
            const T csum = sc.d2[0][0] + sc.d2[1][0] + sc.d2[2][0];
            sd.v         = zq[3];
            sd.g[0]      = rz.get(REC_SD1X);
            sd.g[1]      = rz.get(REC_SD1Y);
            sd.g[2]      = sz1;
            sd.lap       = csum * sd.v + rz.get(REC_SLAP) + sz2;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                vd.g[c][0] = rz.get(REC_V + 4 * c + 0);
                vd.g[c][1] = rz.get(REC_V + 4 * c + 1);
                vd.lap[c]  = csum * vd.v[c] + rz.get(REC_V + 4 * c + 2) +
                            rz.get(REC_V + 4 * c + 3) + s2z[c];
            }
            /* grad div v: the parts without the z-coupled mixed sums now, those
             * once plane lp's contributions are in (same association either way) */
            const T gd0 = sc.d2[0][0] * vd.v[0] + rz.get(REC_V + 2) + rz.get(REC_DXY1);
            const T gd1 = rz.get(REC_DXY0) + sc.d2[1][0] * vd.v[1] + rz.get(REC_V + 4 + 3);
            auto finish_gd = [&]() {
                vd.gd[0] = gd0 + acc[0][0];
                vd.gd[1] = gd1 + acc[1][0];
                vd.gd[2] = fma(sc.d2[2][0], vd.v[2], acc[2][0]) + s2z[2];
            };
            if constexpr (!LATE_NOW)
                finish_gd();

            HydroToMag<T> hx;
            MagToHydro<T> mx;
            [[maybe_unused]] Strain<T> st;
            /* group 0 sends grad lnrho, lap lnrho, S:S and div u; group 1 takes u
             * from the ring and the exponentials from group 0's record */
            constexpr int k0 = H2M_GL, k1 = H2M_DIVU + 1;
            /* the exchange alternates between two buffers by plane parity, so the
             * exchange barrier of the next plane also guards its reuse: in TMEM
             * the unused columns of record slots 0 and 1 of each group, in shared
             * memory two blocks of 15 rows */
            const uint32_t xslot  = LC::XCH0 + (uint32_t)(lp & 1) * LC::XCH_W;
            const uint32_t xmine  = tcol + xslot;
            const uint32_t xother = tother + xslot;
            T* xh = xch + (size_t)(lp & 1) * XROWS * NCELL; /* rows 0..5 */
            T* xm = xh + (size_t)(k1 - k0) * NCELL;         /* rows 6..14 */
            if constexpr (GROUP == 0) {
                hydro_prepare_exp(sd, vd, e_cs, e_irh, hx, st);
                if constexpr (XT) {
                    tmem::Words<T, 6> xw;
#pragma unroll
                    for (int k = k0; k < k1; ++k)
                        xw.set(k - k0, hx.a[k]);
                    __syncwarp();
                    xw.store(xmine);
                }
                else {
#pragma unroll
                    for (int k = k0; k < k1; ++k)
                        xh[(k - k0) * NCELL + cell] = hx.a[k];
                }
            }
            else {
                mag_prepare(sd, vd, p, mx);
                hx.a[H2M_E]       = e_cs;
                hx.a[H2M_INV_RHO] = e_irh;
                hx.a[H2M_U + 0]   = uz.get(0);
                hx.a[H2M_U + 1]   = uz.get(1);
                hx.a[H2M_U + 2]   = uz.get(2);
                if constexpr (XT) {
                    tmem::Words<T, 9> xw;
#pragma unroll
                    for (int k = 0; k < AC_M2H_COUNT; ++k)
                        xw.set(k, mx.a[k]);
                    __syncwarp();
                    xw.store(xmine);
                }
                else {
#pragma unroll
                    for (int k = 0; k < AC_M2H_COUNT; ++k)
                        xm[k * NCELL + cell] = mx.a[k];
                }
            }
            /* The step's one block barrier: the exchange values are written; no
             * thread reads a plane before lp any more (a plane is read in the
             * step it arrives; z taps come from the queue), so the ring slot of
             * plane lp - 6 takes plane lp + 2 next; the tensor-memory entries
             * stored before it are visible to the other group after it. */
            tmem::wait_st();
            tmem::fence_before_sync();
            __syncthreads();
            tmem::fence_after_sync();
            {
                const int next = lp + 2; /* = lp - 6 + RING */
                if (tid == 0 && next <= plast && !(skip_last && next == plast)) {
                    const int sl = (next - pfirst) & (RING - 1);
                    mbar_arrive_expect_tx(&bars[sl], L::SLOT_BYTES);
                    tma_load_plane(smem + (size_t)sl * L::SLOT, tmap, &bars[sl], x0, y0,
                                   next + NGHOST);
                }
            }
            if constexpr (XT) {
                __syncwarp();
                if constexpr (GROUP == 0) {
                    tmem::Words<T, 9> xw;
                    xw.load(xother);
                    tmem::wait_ld();
                    xw.tie();
#pragma unroll
                    for (int k = 0; k < AC_M2H_COUNT; ++k)
                        mx.a[k] = xw.get(k);
                }
                else {
                    tmem::Words<T, 6> xw;
                    xw.load(xother);
                    tmem::wait_ld();
                    xw.tie();
#pragma unroll
                    for (int k = k0; k < k1; ++k)
                        hx.a[k] = xw.get(k - k0);
                }
            }
            if constexpr (LATE_NOW) {
                inplane();
                finish_gd();
            }
            /* with the late in-plane part the rates are formed by every thread
             * (one basic block with it); a cell outside the mesh only skips its
             * stores */
            if (LATE_NOW || active) {
                T rr[4], val[4];
                if constexpr (GROUP == 0) {
                    if constexpr (!XT) {
#pragma unroll
                        for (int k = 0; k < AC_M2H_COUNT; ++k)
                            mx.a[k] = xm[k * NCELL + cell];
                    }
                    hydro_rates(sd, vd, st, hx, mx, p, rr);
                    val[0] = sd.v;
                    val[1] = vd.v[0];
                    val[2] = vd.v[1];
                    val[3] = vd.v[2];
                }
                else {
                    if constexpr (!XT) {
#pragma unroll
                        for (int k = k0; k < k1; ++k)
                            hx.a[k] = xh[(k - k0) * NCELL + cell];
                    }
                    mag_rates(sd, vd, mx, hx, p, rr);
                    if (do_cfl && active) {
                        const T* u = &hx.a[H2M_U];
                        const T* B = &mx.a[M2H_B];
                        cfl_accumulate(u[0] * u[0] + u[1] * u[1] + u[2] * u[2],
                                       B[0] * B[0] + B[1] * B[1] + B[2] * B[2],
                                       hx.a[H2M_INV_RHO], p.cs2_sound, cm, cfl_sum);
                    }
                    val[0] = vd.v[0];
                    val[1] = vd.v[1];
                    val[2] = vd.v[2];
                    val[3] = sd.v;
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if constexpr (COMP) {
                        float oh, ol;
                        rk_update_comp(val[k], lo[k], prev[k], prevl[k], rr[k], c32, use_prev, oh,
                                       ol);
                        if (active) {
                            outp[k][idx] = oh;
                            outl[k][idx] = ol;
                        }
                    }
                    else {
                        double o;
                        rk_update(val[k], prev[k], rr[k], c64, use_prev, o);
                        if (active)
                            outp[k][idx] = o;
                    }
                }
            }
        }
        /* the running sums move on by one plane (the first is complete and used) */
#pragma unroll
        for (int a = 0; a < 3; ++a) {
#pragma unroll
            for (int j = 0; j < 6; ++j)
                acc[a][j] = acc[a][j + 1];
            acc[a][6] = 0;
        }
        if constexpr (!SOLVE) {
            /* a step without a solve: the records stored are visible to the other
             * group after this barrier (no ring slot is freed before the first
             * solve) */
            tmem::wait_st();
            tmem::fence_before_sync();
            __syncthreads();
            tmem::fence_after_sync();
        }
        if constexpr (LATE_NOW)
            tmem::wait_st(); /* the queue entry of plane lp, read in the next step */
        r3 = r3 == 2u ? 0u : r3 + 1u;
        q7 = q7 == 6u ? 0u : q7 + 1u;
    };

    /* planes lp = pfirst .. plast in four phases (interior: lp in [z0, z1);
     * solve: lp >= z0 + 3) */
    int lp = pfirst;
    for (; lp < z0; ++lp)
        step(LeadPhase<false, false>{}, lp);
    for (; lp < min(z1, z0 + NGHOST); ++lp)
        step(LeadPhase<true, false>{}, lp);
    for (; lp < z1; ++lp)
        step(LeadPhase<true, true>{}, lp);
    for (; lp < z0 + NGHOST; ++lp) /* chunks shorter than three planes */
        step(LeadPhase<false, false>{}, lp);
    for (; lp <= plast; ++lp)
        step(LeadPhase<false, true>{}, lp);

    if (do_cfl) {
        __syncthreads(); /* every thread's last exchange reads are done */
        cfl_commit(cm, red, cfl);
    }
    if (!ok)
        atomicExch(err, 1);
}

template <typename T, bool COMP, bool XT, int MODE>
__global__ void __launch_bounds__(2 * TX * TY, Tile<T>::MINB)
solve_lead_kernel(const __grid_constant__ CUtensorMap tmap, const Geom g, const FieldsT<T> f,
                  const StencilT<T> sc, const PhysConst pc, const RkCoef rk, int* err,
                  unsigned long long* cfl, const int zchunk)
{
    typedef Layout<T> L;
    typedef LeadTm<T> TM;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    typedef LeadSmem<T, XT> LS;
    T* smem         = reinterpret_cast<T*>(smem_raw);
    T* xch          = reinterpret_cast<T*>(smem_raw + LS::RING_B);
    T* red          = reinterpret_cast<T*>(smem_raw + LS::RING_B + LS::XCH_B);
    uint64_t* bars  = reinterpret_cast<uint64_t*>(smem_raw + LS::BAR_OFF);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + RING);
    const int warp  = threadIdx.y; /* blockDim.x == 32 */
    const int group = threadIdx.y / TY;
    const int tid   = threadIdx.y * TX + threadIdx.x;
    const int z0    = pc.zlo + (int)blockIdx.z * zchunk;
    const int z1    = min(z0 + zchunk, pc.zhi);
    const int pfirst = z0 - NGHOST;
    const int plast  = z1 - 1 + NGHOST;

    if (tid == 0) {
        for (int s = 0; s < RING; ++s)
            mbar_init(&bars[s], 1);
        fence_barrier_init();
    }
    __syncwarp(); /* warp 0 reconverges after thread 0's barrier set-up */
    if (warp == 0)
        tmem::alloc(tslot, TM::NCOLS);
    tmem::fence_before_sync();
    __syncthreads();
    tmem::fence_after_sync();
    const uint32_t tbase = *tslot;
    /* this thread's lane (its cell; both groups share it) and its group's columns */
    const uint32_t tcol = tmem::lane_base(tbase, warp) + (uint32_t)group * TM::GROUP;
    /* the fault-path test switch skips the load of plane plast */
    const bool skip_last = pc.debug_skip_load != 0;
    if (tid == 0) {
        const int pend = min(plast, pfirst + RING - 1);
        for (int q = pfirst; q <= pend; ++q) {
            if (skip_last && q == plast)
                continue;
            const int s = (q - pfirst) & (RING - 1);
            mbar_arrive_expect_tx(&bars[s], L::SLOT_BYTES);
            tma_load_plane(smem + (size_t)s * L::SLOT, &tmap, &bars[s], blockIdx.x * TX,
                           blockIdx.y * TY, q + NGHOST);
        }
    }
    const PhysT<T> p        = phys_cast<T>(pc);
    const StencilT<T> scv   = sc;
    if (group == 0)
        lead_group<T, COMP, 0, XT, MODE>(&tmap, g, f, scv, p, rk, err, cfl, smem, xch, red, bars, tcol,
                               zchunk, pc.zlo, pc.zhi, skip_last, pc.cfl_sum != 0);
    else
        lead_group<T, COMP, 1, XT, MODE>(&tmap, g, f, scv, p, rk, err, cfl, smem, xch, red, bars, tcol,
                               zchunk, pc.zlo, pc.zhi, skip_last, pc.cfl_sum != 0);
    /* no copy into this block's shared memory is left in flight */
    if (tid == 0)
        drain_ring(bars, RING, [&](const int sl) { return loads_into(sl, pfirst, plast, skip_last); });

    /* every thread's tensor-memory accesses are complete before the columns are freed */
    __syncwarp();
    tmem::wait_st();
    tmem::fence_before_sync();
    __syncthreads();
    tmem::fence_after_sync();
    __syncwarp();
    if (warp == 0)
        tmem::dealloc(tbase, TM::NCOLS);
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

/* Planes per CTA.  Every chunk reads and forms 6 halo planes beyond its own,
 * so long chunks are cheaper, until the grid quantises badly into waves of
 * resident CTAs.  Among 512, 256, 128, 64 and 32 planes that keep at least two
 * CTAs per SM of the 148, the chunk with the least (waves of `per_sm` resident
 * CTAs per SM) x (planes a CTA steps through) is taken; the larger on a tie.
 * Smaller grids halve 32 down to 8 while there are fewer than two CTAs per SM.
 * (Measured at 512^3, FP64: 512 planes 28.9-29.1 ms per step against 29.2-29.3
 * with 256; earlier 256 planes 29.3, 128 planes 29.6-29.8, 64 planes 30.9; at
 * 256^3, 256-plane chunks would leave 512 CTAs, 3.5 waves.) */
int
zchunk_for(const Geom& g, const int nz, const int per_sm)
{
    const long long tiles = (long long)((g.nx + TX - 1) / TX) * ((g.ny + TY - 1) / TY);
    const long long slots = 148LL * per_sm;
    int best              = 0;
    long long best_cost   = 0;
    for (int zc = ZCHUNK; zc >= 32; zc /= 2) {
        const long long ctas = tiles * ((nz + zc - 1) / zc);
        if (ctas < 2 * 148)
            continue;
        const long long cost = (ctas + slots - 1) / slots * (long long)(min(zc, nz) + 2 * NGHOST);
        if (best == 0 || cost < best_cost) {
            best      = zc;
            best_cost = cost;
        }
    }
    if (best)
        return best;
    int zc = 32;
    while (zc > 8 && tiles * ((nz + zc - 1) / zc) < 2 * 148)
        zc /= 2;
    return zc;
}

template <typename T, bool COMP>
cudaError_t
launch_tiled(const Geom& g, const void* tmap_in, const FieldsT<T>& f, const StencilCoef& sc,
             const PhysConst& pc, const RkCoef& rk, int* err, unsigned long long* cfl,
             cudaStream_t stream, unsigned long long* launches, const int kernel)
{
    const dim3 tpb(TX, 2 * TY, 1);
    /* the planes [zlo, zhi) of this launch (all nz unless the caller solves the
     * interior in z boxes) */
    const int nzr = pc.zhi - pc.zlo;
    if (nzr <= 0)
        return cudaSuccess;
    const int per_sm = Tile<T>::MINB; /* resident CTAs per SM */
    const int zc     = zchunk_for(g, nzr, per_sm);
    const dim3 bpg((g.nx + TX - 1) / TX, (g.ny + TY - 1) / TY, (nzr + zc - 1) / zc);
    /* The leading-plane kernel forms stage 1 for the 6 halo planes of every z
     * chunk too; on short chunks (small meshes) that overhead loses to the
     * per-plane tap kernel, so the automatic choice takes it from 32 planes.
     * The choice follows the whole mesh, so that a substep solved in z boxes
     * gives the bits of the whole-interior launch (the results of either kernel
     * do not depend on where the z chunks start). */
    const int k = kernel == AC_SOLVE_TILED_AUTO
                      ? (zchunk_for(g, g.nz, per_sm) >= 32 ? AC_SOLVE_TILED_LEAD
                                                            : AC_SOLVE_TILED_TAPS)
                      : kernel;
    if (pc.upwind)
        solve_tiled_kernel<T, COMP, true><<<bpg, tpb, Layout<T>::SMEM_BYTES, stream>>>(
            *(const CUtensorMap*)tmap_in, g, f, stencil_cast<T>(sc), pc, rk, err, cfl, zc);
    else if (k == AC_SOLVE_TILED_LEAD || k == AC_SOLVE_TILED_LEAD_ALT) {
        /* the exchange between the warp groups goes through tensor memory; _ALT
         * takes shared memory instead (measured at 512^3: 28.5 against 29.5 ms
         * per FP64 step, and in FP32 the second shared-memory buffer costs the
         * second block per SM: 22.8 against 32.0 ms) */
        const bool xt = k != AC_SOLVE_TILED_LEAD_ALT;
        /* substep 0 of the default kernel reads no previous state: its own form
         * (measured at 512^3: 9.3 against 9.8 ms FP64, 6.2 against 6.7 ms FP32) */
        const size_t sb = lead_smem_bytes<T, true>();
        const CUtensorMap& tm = *(const CUtensorMap*)tmap_in;
        const StencilT<T> st  = stencil_cast<T>(sc);
        if (xt && rk.step == 0 && !cfl)
            solve_lead_kernel<T, COMP, true, MODE_FIRST><<<bpg, tpb, sb, stream>>>(
                tm, g, f, st, pc, rk, err, cfl, zc);
        else if (xt)
            solve_lead_kernel<T, COMP, true, MODE_RUNTIME><<<bpg, tpb, sb, stream>>>(
                tm, g, f, st, pc, rk, err, cfl, zc);
        else
            solve_lead_kernel<T, COMP, false, MODE_RUNTIME><<<bpg, tpb, lead_smem_bytes<T, false>(), stream>>>(
                *(const CUtensorMap*)tmap_in, g, f, stencil_cast<T>(sc), pc, rk, err, cfl, zc);
    }
    else
        solve_tiled_kernel<T, COMP, false><<<bpg, tpb, Layout<T>::SMEM_BYTES, stream>>>(
            *(const CUtensorMap*)tmap_in, g, f, stencil_cast<T>(sc), pc, rk, err, cfl, zc);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

template <typename T>
cudaError_t
set_smem(const void* fn, const size_t bytes)
{
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
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

/* Opts the kernels in to their dynamic shared memory on the current device;
 * called by acDeviceCreate, outside any stream capture. */
cudaError_t
ac_solve_tiled_init(const int precision)
{
    cudaError_t e;
    if (precision == 0) {
        typedef Layout<double> L;
        if ((e = set_smem<double>((const void*)solve_tiled_kernel<double, false, false>,
                                  L::SMEM_BYTES)) != cudaSuccess ||
            (e = set_smem<double>((const void*)solve_tiled_kernel<double, false, true>,
                                  L::SMEM_BYTES)) != cudaSuccess)
            return e;
        if ((e = set_smem<double>((const void*)solve_lead_kernel<double, false, true, MODE_FIRST>,
                                  lead_smem_bytes<double, true>())) != cudaSuccess ||
            (e = set_smem<double>(
                 (const void*)solve_lead_kernel<double, false, true, MODE_RUNTIME>,
                 lead_smem_bytes<double, true>())) != cudaSuccess)
            return e;
        return set_smem<double>((const void*)solve_lead_kernel<double, false, false, MODE_RUNTIME>,
                                lead_smem_bytes<double, false>());
    }
    typedef Layout<float> L;
    if ((e = set_smem<float>((const void*)solve_tiled_kernel<float, true, false>,
                             L::SMEM_BYTES)) != cudaSuccess ||
        (e = set_smem<float>((const void*)solve_tiled_kernel<float, true, true>, L::SMEM_BYTES)) !=
            cudaSuccess)
        return e;
    if ((e = set_smem<float>((const void*)solve_lead_kernel<float, true, true, MODE_FIRST>,
                             lead_smem_bytes<float, true>())) != cudaSuccess ||
        (e = set_smem<float>((const void*)solve_lead_kernel<float, true, true, MODE_RUNTIME>,
                             lead_smem_bytes<float, true>())) != cudaSuccess)
        return e;
    return set_smem<float>((const void*)solve_lead_kernel<float, true, false, MODE_RUNTIME>,
                           lead_smem_bytes<float, false>());
}

cudaError_t
ac_launch_solve_tiled64(const Geom& g, const void* tmap_in, const Fields64& f,
                        const StencilCoef& sc, const PhysConst& pc, const RkCoef& rk, int* err,
                        unsigned long long* cfl, cudaStream_t stream,
                        unsigned long long* launches, const int kernel)
{
    return launch_tiled<double, false>(g, tmap_in, f, sc, pc, rk, err, cfl, stream, launches,
                                       kernel);
}

cudaError_t
ac_launch_solve_tiled32(const Geom& g, const void* tmap_in, const Fields32& f,
                        const StencilCoef& sc, const PhysConst& pc, const RkCoef& rk, int* err,
                        unsigned long long* cfl, cudaStream_t stream,
                        unsigned long long* launches, const int kernel)
{
    return launch_tiled<float, true>(g, tmap_in, f, sc, pc, rk, err, cfl, stream, launches,
                                     kernel);
}
