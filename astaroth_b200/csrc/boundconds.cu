/*
 * Periodic halo fill and buffer fill kernels.
 *
 * Periodic boundconds: every ghost cell of [start, end) takes the value of
 * the interior cell it wraps to; interior cells are never written, so the
 * copy is in place and race free (sources are always interior).  Follows the
 * host model src/utils/memory.cc:76-149 (the oracle this is checked against
 * bit for bit).  The reference's device kernel BOUNDCOND_PERIODIC_DEVICE
 * (acc-runtime/built-in/kernels.h:17-42) adds AC_nlocal.x to the y and z
 * wraps, which differs from the host model on non-cubic grids; this file
 * follows the host model on all grids.
 *
 * One launch fills all requested fields (the reference launches once per
 * field, src/core/device.cc:999-1017).  For the whole-mesh box the threads
 * enumerate only the ghost cells (z slabs, then y slabs, then x slabs), so
 * no thread is spent on the interior.
 */
#include "internal.h"

namespace {

struct FieldList {
    double* p[AC_NF];
    int n;
};

__device__ __forceinline__ void
copy_wrapped(const Geom& g, const FieldList& fl, const int i, const int j, const int k)
{
    const int is = (i - NGHOST + g.nx) % g.nx + NGHOST;
    const int js = (j - NGHOST + g.ny) % g.ny + NGHOST;
    const int ks = (k - NGHOST + g.nz) % g.nz + NGHOST;
    const long long dst = (long long)i + (long long)j * g.mx + (long long)k * g.mxy;
    const long long src = (long long)is + (long long)js * g.mx + (long long)ks * g.mxy;
#pragma unroll
    for (int q = 0; q < AC_NF; ++q)
        if (q < fl.n)
            fl.p[q][dst] = fl.p[q][src];
}

/* Whole mesh: t enumerates the ghost cells only. */
__global__ void
periodic_halo_kernel(const Geom g, const FieldList fl, const long long nzs, const long long nys,
                     const long long total)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total)
        return;
    int i, j, k;
    if (t < nzs) { /* z slabs: 2*NGHOST full planes */
        i             = (int)(t % g.mx);
        j             = (int)((t / g.mx) % g.my);
        const int kk  = (int)(t / g.mxy);
        k             = kk < NGHOST ? kk : g.nz + kk;
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
    copy_wrapped(g, fl, i, j, k);
}

/* General box [start, end): interior cells are skipped. */
__global__ void
periodic_box_kernel(const Geom g, const FieldList fl, const int3 start, const int3 dims)
{
    const int i = start.x + (int)(threadIdx.x + blockIdx.x * blockDim.x);
    const int j = start.y + (int)(threadIdx.y + blockIdx.y * blockDim.y);
    const int k = start.z + (int)blockIdx.z;
    if (i >= start.x + dims.x || j >= start.y + dims.y)
        return;
    if (i >= NGHOST && i < g.nx + NGHOST && j >= NGHOST && j < g.ny + NGHOST && k >= NGHOST &&
        k < g.nz + NGHOST)
        return;
    copy_wrapped(g, fl, i, j, k);
}

__global__ void
fill_kernel(double* p, const long long count, const double value)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < count;
         t += (long long)gridDim.x * blockDim.x)
        p[t] = value;
}

} // namespace

cudaError_t
ac_launch_periodic(const Geom& g, double* const* fields, const int nfields, const Volume start,
                   const Volume end, cudaStream_t stream, unsigned long long* launches)
{
    if (nfields <= 0 || nfields > AC_NF)
        return cudaErrorInvalidValue;
    if (end.x > (size_t)g.mx || end.y > (size_t)g.my || end.z > (size_t)g.mz ||
        start.x >= end.x || start.y >= end.y || start.z >= end.z)
        return cudaErrorInvalidValue;
    FieldList fl;
    fl.n = nfields;
    for (int q = 0; q < AC_NF; ++q)
        fl.p[q] = q < nfields ? fields[q] : nullptr;

    const bool whole = start.x == 0 && start.y == 0 && start.z == 0 && end.x == (size_t)g.mx &&
                       end.y == (size_t)g.my && end.z == (size_t)g.mz;
    if (whole) {
        const long long nzs   = 2LL * NGHOST * g.mxy;
        const long long nys   = 2LL * NGHOST * g.mx * g.nz;
        const long long nxs   = 2LL * NGHOST * g.ny * g.nz;
        const long long total = nzs + nys + nxs;
        const int tpb         = 256;
        const long long bpg   = (total + tpb - 1) / tpb;
        periodic_halo_kernel<<<(unsigned)bpg, tpb, 0, stream>>>(g, fl, nzs, nys, total);
    }
    else {
        const int3 s  = make_int3((int)start.x, (int)start.y, (int)start.z);
        const int3 d  = make_int3((int)(end.x - start.x), (int)(end.y - start.y),
                                 (int)(end.z - start.z));
        const dim3 tpb(32, 8, 1);
        const dim3 bpg((d.x + 31) / 32, (d.y + 7) / 8, d.z);
        periodic_box_kernel<<<bpg, tpb, 0, stream>>>(g, fl, s, d);
    }
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

cudaError_t
ac_launch_fill(double* ptr, const long long count, const double value, cudaStream_t stream,
               unsigned long long* launches)
{
    if (count <= 0)
        return cudaSuccess;
    const int tpb      = 256;
    long long bpg      = (count + tpb - 1) / tpb;
    if (bpg > 148 * 32)
        bpg = 148 * 32;
    fill_kernel<<<(unsigned)bpg, tpb, 0, stream>>>(ptr, count, value);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}
