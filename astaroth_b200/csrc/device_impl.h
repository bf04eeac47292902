/*
 * Shared by the translation units of the device layer (device.cu: create,
 * configuration, host transfers, integration, reductions and the CFL
 * outputs; device_data.cu: ranges, transfers between devices, staged loads,
 * plane packing, snapshots; device_adjoint.cu: the discrete adjoint): buffer
 * access, argument checks, and the launch helpers of device.cu.
 */
#pragma once

#include "internal.h"

/* ---- buffer access ---- */

static inline size_t
elem_size(const Device d)
{
    return d->precision == 0 ? sizeof(double) : sizeof(float);
}

static inline double*
arr64(const Device d, const int b, const int q)
{
    return (double*)d->hi[b] + (size_t)q * d->geom.cells;
}

static inline float*
arr_hi(const Device d, const int b, const int q)
{
    return (float*)d->hi[b] + (size_t)q * d->geom.cells;
}

static inline float*
arr_lo(const Device d, const int b, const int q)
{
    return d->lo[b] + (size_t)q * d->geom.cells;
}

static inline Fields64
fields64(const Device d)
{
    Fields64 f;
    for (int q = 0; q < AC_NF; ++q) {
        f.in[q]     = arr64(d, d->in_idx[q], q);
        f.out[q]    = arr64(d, 1 - d->in_idx[q], q);
        f.in_lo[q]  = nullptr;
        f.out_lo[q] = nullptr;
    }
    return f;
}

static inline Fields32
fields32(const Device d)
{
    Fields32 f;
    for (int q = 0; q < AC_NF; ++q) {
        f.in[q]     = arr_hi(d, d->in_idx[q], q);
        f.out[q]    = arr_hi(d, 1 - d->in_idx[q], q);
        f.in_lo[q]  = arr_lo(d, d->in_idx[q], q);
        f.out_lo[q] = arr_lo(d, 1 - d->in_idx[q], q);
    }
    return f;
}

/* The block holding every field's in-buffer (0 or 1), or -1 when single
 * fields were swapped on their own. */
static inline int
in_block_index(const Device d)
{
    for (int q = 1; q < AC_NF; ++q)
        if (d->in_idx[q] != d->in_idx[0])
            return -1;
    return d->in_idx[0];
}

static inline bool
stream_ok(const Stream s)
{
    return (int)s >= 0 && (int)s < NUM_STREAMS;
}

static inline bool
host_matches(const Device d, const AcMeshInfo& host)
{
    AcMeshInfo h = host;
    if (acHostUpdateParams(&h) != AC_SUCCESS)
        return false;
    const int3 m = h.int3_params[AC_mlocal];
    return m.x == d->geom.mx && m.y == d->geom.my && m.z == d->geom.mz;
}

/* The result of a whole-mesh transfer from its per-field results: AC_FAILURE
 * if any field failed, else AC_NOT_ALLOCATED if any host field was NULL. */
static inline AcResult
worst(const AcResult a, const AcResult b)
{
    if (a == AC_FAILURE || b == AC_FAILURE)
        return AC_FAILURE;
    return a == AC_NOT_ALLOCATED || b == AC_NOT_ALLOCATED ? AC_NOT_ALLOCATED : AC_SUCCESS;
}

static inline bool
is_whole_interior(const Device d, const Volume start, const Volume end)
{
    return start.x == NGHOST && start.y == NGHOST && start.z == NGHOST &&
           end.x == (size_t)(d->geom.nx + NGHOST) && end.y == (size_t)(d->geom.ny + NGHOST) &&
           end.z == (size_t)(d->geom.nz + NGHOST);
}

/* A box of whole interior x-y planes: [nmin.z + zlo, nmin.z + zhi) in z. */
static inline bool
is_z_box(const Device d, const Volume start, const Volume end)
{
    return start.x == NGHOST && start.y == NGHOST && end.x == (size_t)(d->geom.nx + NGHOST) &&
           end.y == (size_t)(d->geom.ny + NGHOST) && start.z >= NGHOST && start.z < end.z &&
           end.z <= (size_t)(d->geom.nz + NGHOST);
}

/* device.cu; [zlo, zhi) are the interior z planes solved (zhi < 0: all) */
cudaError_t launch_substep(Device d, cudaStream_t st, const int step, const double dt,
                           unsigned long long* launches, const int zlo = 0, const int zhi = -1);
cudaError_t launch_periodic(Device d, cudaStream_t st, const int q0, const int nq,
                            const Volume start, const Volume end, unsigned long long* launches);
void invalidate_tape_graph(Device d);
