/*
 * Index arithmetic of the periodic halo fill, shared by the single-mesh
 * kernels (boundconds.cu) and the ensemble's one-launch fill (ensemble.cu).
 *
 * Every ghost cell takes the value of the interior cell it wraps to
 * (host model src/utils/memory.cc:76-149).  The ghost cells of a whole mesh
 * are enumerated as z slabs (2*NGHOST full planes), then y slabs inside the
 * interior z range, then x slabs inside the interior y and z ranges, so a
 * launch spends no thread on the interior.
 */
#pragma once

#include "internal.h"

/* Number of ghost cells of g; *nzs and *nys receive the sizes of the z-slab
 * and y-slab groups. */
__host__ __device__ inline long long
halo_count(const Geom& g, long long* nzs, long long* nys)
{
    *nzs = 2LL * NGHOST * g.mx * g.my;
    *nys = 2LL * NGHOST * g.mx * g.nz;
    return *nzs + *nys + 2LL * NGHOST * g.ny * g.nz;
}

/* Coordinates (i, j, k) of ghost cell number t. */
__device__ __forceinline__ void
halo_cell(const Geom& g, const long long t, const long long nzs, const long long nys, int& i,
          int& j, int& k)
{
    const long long mxy = (long long)g.mx * g.my;
    if (t < nzs) { /* z slabs: 2*NGHOST full planes */
        i            = (int)(t % g.mx);
        j            = (int)((t / g.mx) % g.my);
        const int kk = (int)(t / mxy);
        k            = kk < NGHOST ? kk : g.nz + kk;
    }
    else if (t < nzs + nys) { /* y slabs inside the interior z range */
        const long long u = t - nzs;
        i                 = (int)(u % g.mx);
        const int jj      = (int)((u / g.mx) % (2 * NGHOST));
        k                 = NGHOST + (int)(u / ((long long)g.mx * 2 * NGHOST));
        j                 = jj < NGHOST ? jj : g.ny + jj;
    }
    else { /* x slabs inside the interior y and z ranges */
        const long long u = t - nzs - nys;
        const int ii      = (int)(u % (2 * NGHOST));
        j                 = NGHOST + (int)((u / (2 * NGHOST)) % g.ny);
        k                 = NGHOST + (int)(u / ((long long)2 * NGHOST * g.ny));
        i                 = ii < NGHOST ? ii : g.nx + ii;
    }
}

/* Linear index of the interior cell that ghost cell (i, j, k) wraps to. */
__device__ __forceinline__ long long
halo_source(const Geom& g, const int i, const int j, const int k)
{
    const int is = (i - NGHOST + g.nx) % g.nx + NGHOST;
    const int js = (j - NGHOST + g.ny) % g.ny + NGHOST;
    const int ks = (k - NGHOST + g.nz) % g.nz + NGHOST;
    return geom_idx(g, is, js, ks);
}
