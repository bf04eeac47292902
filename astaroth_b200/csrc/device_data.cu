/*
 * The device layer's data movement beyond whole-mesh host transfers: linear
 * ranges between host and device and between devices (the reference's
 * *WithOffset and acDeviceTransfer* family), volume copies, pipelined staged
 * loads, transfers from and to caller-owned device arrays, whole-plane
 * packing for slab decompositions, box packing for decompositions in x, y and
 * z, snapshots, and the auxiliary B field.
 */
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include "internal.h"
#include "device_impl.h"

/* ---- linear ranges between meshes: the reference's *WithOffset family
 * (src/core/device.cc:666-698 and its store and transfer counterparts).
 * num_vertices consecutive values in host-layout linear order (x fastest,
 * rows of mx) move from position src of the source to position dst of the
 * target, into or out of the device's in-buffer.  FP32-compensated devices
 * split/join the range on the fly.  Ranges must lie inside both meshes. ---- */

static bool
mesh_dims(const AcMeshInfo& info, long long m[3])
{
    AcMeshInfo h = info;
    if (acHostUpdateParams(&h) != AC_SUCCESS)
        return false;
    const int3 v = h.int3_params[AC_mlocal];
    m[0]         = v.x;
    m[1]         = v.y;
    m[2]         = v.z;
    return v.x > 0 && v.y > 0 && v.z > 0;
}

/* linear index of p in a mesh of dims m, or -1 when p is outside or the n
 * values from it do not fit */
static long long
range_start(const int3 p, const long long m[3], const long long n)
{
    if (n < 0 || p.x < 0 || p.y < 0 || p.z < 0 || p.x >= m[0] || p.y >= m[1] || p.z >= m[2])
        return -1;
    const long long L = p.x + m[0] * (p.y + m[1] * (long long)p.z);
    return L + n <= m[0] * m[1] * m[2] ? L : -1;
}

static void
device_dims(const Device d, long long m[3])
{
    m[0] = d->geom.mx;
    m[1] = d->geom.my;
    m[2] = d->geom.mz;
}

extern "C" AcResult
acDeviceLoadVertexBufferWithOffset(const Device d, const Stream stream, const AcMesh host_mesh,
                                   const VertexBufferHandle h, const int3 src, const int3 dst,
                                   const int num_vertices)
{
    if (!d || !stream_ok(stream) || (int)h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    if (!host_mesh.vertex_buffer[h])
        return AC_NOT_ALLOCATED;
    long long hm[3], dm[3];
    device_dims(d, dm);
    if (!mesh_dims(host_mesh.info, hm))
        return AC_FAILURE;
    const long long n = num_vertices, s0 = range_start(src, hm, n), d0 = range_start(dst, dm, n);
    if (s0 < 0 || d0 < 0)
        return AC_FAILURE;
    if (n == 0)
        return AC_SUCCESS;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const int b       = d->in_idx[h];
    cudaStream_t st   = d->streams[stream];
    const double* hp  = host_mesh.vertex_buffer[h] + s0;
    if (d->precision == 0) {
        AC_CUDA_CHECK(cudaMemcpyAsync(arr64(d, b, h) + d0, hp, n * sizeof(double),
                                      cudaMemcpyHostToDevice, st));
        return AC_SUCCESS;
    }
    AC_CUDA_CHECK(cudaMemcpyAsync(d->staging + d0, hp, n * sizeof(double), cudaMemcpyHostToDevice,
                                  st));
    AC_CUDA_CHECK(ac_launch_split_range(d->geom, d->staging, arr_hi(d, b, h), arr_lo(d, b, h),
                                        d0, n, st, &d->launches));
    AC_CUDA_CHECK(cudaStreamSynchronize(st)); /* the staging field is shared */
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceLoadMeshWithOffset(const Device d, const Stream stream, const AcMesh host_mesh,
                           const int3 src, const int3 dst, const int num_vertices)
{
    AcResult res = AC_SUCCESS;
    for (int q = 0; q < AC_NF; ++q)
        res = worst(res, acDeviceLoadVertexBufferWithOffset(d, stream, host_mesh,
                                                            (VertexBufferHandle)q, src, dst,
                                                            num_vertices));
    return res;
}

extern "C" AcResult
acDeviceStoreVertexBufferWithOffset(const Device d, const Stream stream,
                                    const VertexBufferHandle h, const int3 src, const int3 dst,
                                    const int num_vertices, AcMesh* host_mesh)
{
    if (!d || !host_mesh || !stream_ok(stream) || (int)h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    if (!host_mesh->vertex_buffer[h])
        return AC_NOT_ALLOCATED;
    long long hm[3], dm[3];
    device_dims(d, dm);
    if (!mesh_dims(host_mesh->info, hm))
        return AC_FAILURE;
    const long long n = num_vertices, s0 = range_start(src, dm, n), d0 = range_start(dst, hm, n);
    if (s0 < 0 || d0 < 0)
        return AC_FAILURE;
    if (n == 0)
        return AC_SUCCESS;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const int b     = d->in_idx[h];
    cudaStream_t st = d->streams[stream];
    double* hp      = host_mesh->vertex_buffer[h] + d0;
    if (d->precision == 0) {
        AC_CUDA_CHECK(cudaMemcpyAsync(hp, arr64(d, b, h) + s0, n * sizeof(double),
                                      cudaMemcpyDeviceToHost, st));
    }
    else {
        AC_CUDA_CHECK(ac_launch_join_range(d->geom, arr_hi(d, b, h), arr_lo(d, b, h), d->staging,
                                           s0, n, st, &d->launches));
        AC_CUDA_CHECK(cudaMemcpyAsync(hp, d->staging + s0, n * sizeof(double),
                                      cudaMemcpyDeviceToHost, st));
    }
    AC_CUDA_CHECK(cudaStreamSynchronize(st)); /* the host range is ready on return */
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceStoreMeshWithOffset(const Device d, const Stream stream, const int3 src, const int3 dst,
                            const int num_vertices, AcMesh* host_mesh)
{
    AcResult res = AC_SUCCESS;
    for (int q = 0; q < AC_NF; ++q)
        res = worst(res, acDeviceStoreVertexBufferWithOffset(d, stream, (VertexBufferHandle)q, src,
                                                             dst, num_vertices, host_mesh));
    return res;
}

/* Device to device (the reference's acDeviceTransfer*, device.cc): on the source
 * device's stream, with a peer copy between GPUs.  Both devices must have the
 * same precision. */
extern "C" AcResult
acDeviceTransferVertexBufferWithOffset(const Device from, const Stream stream,
                                       const VertexBufferHandle h, const int3 src, const int3 dst,
                                       const int num_vertices, Device to)
{
    if (!from || !to || !stream_ok(stream) || (int)h < 0 || h >= NUM_VTXBUF_HANDLES ||
        from->precision != to->precision)
        return AC_FAILURE;
    long long fm[3], tm[3];
    device_dims(from, fm);
    device_dims(to, tm);
    const long long n = num_vertices, s0 = range_start(src, fm, n), d0 = range_start(dst, tm, n);
    if (s0 < 0 || d0 < 0)
        return AC_FAILURE;
    if (n == 0)
        return AC_SUCCESS;
    AC_CUDA_CHECK(cudaSetDevice(from->id));
    cudaStream_t st = from->streams[stream];
    const int fb = from->in_idx[h], tb = to->in_idx[h];
    if (from->precision == 0) {
        AC_CUDA_CHECK(cudaMemcpyPeerAsync(arr64(to, tb, h) + d0, to->id, arr64(from, fb, h) + s0,
                                          from->id, n * sizeof(double), st));
        return AC_SUCCESS;
    }
    /* FP32-compensated: join into the source's staging field, copy the doubles
     * to the target's staging field, split there */
    AC_CUDA_CHECK(ac_launch_join_range(from->geom, arr_hi(from, fb, h), arr_lo(from, fb, h),
                                       from->staging, s0, n, st, &from->launches));
    AC_CUDA_CHECK(cudaMemcpyPeerAsync(to->staging + d0, to->id, from->staging + s0, from->id,
                                      n * sizeof(double), st));
    AC_CUDA_CHECK(cudaStreamSynchronize(st));
    AC_CUDA_CHECK(cudaSetDevice(to->id));
    cudaStream_t tst = to->streams[stream];
    AC_CUDA_CHECK(ac_launch_split_range(to->geom, to->staging, arr_hi(to, tb, h),
                                        arr_lo(to, tb, h), d0, n, tst, &to->launches));
    AC_CUDA_CHECK(cudaStreamSynchronize(tst));
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceTransferMeshWithOffset(const Device from, const Stream stream, const int3 src,
                               const int3 dst, const int num_vertices, Device to)
{
    AcResult res = AC_SUCCESS;
    for (int q = 0; q < AC_NF; ++q)
        res = worst(res, acDeviceTransferVertexBufferWithOffset(from, stream, (VertexBufferHandle)q,
                                                                src, dst, num_vertices, to));
    return res;
}

extern "C" AcResult
acDeviceTransferVertexBuffer(const Device from, const Stream stream, const VertexBufferHandle h,
                             Device to)
{
    if (!from || !to || from->geom.mx != to->geom.mx || from->geom.my != to->geom.my ||
        from->geom.mz != to->geom.mz)
        return AC_FAILURE;
    const long long n = (long long)from->geom.mx * from->geom.my * from->geom.mz;
    if (n > 0x7fffffffLL)
        return AC_FAILURE;
    const int3 o = {0, 0, 0};
    return acDeviceTransferVertexBufferWithOffset(from, stream, h, o, o, (int)n, to);
}

extern "C" AcResult
acDeviceTransferMesh(const Device from, const Stream stream, Device to)
{
    AcResult res = AC_SUCCESS;
    for (int q = 0; q < AC_NF; ++q)
        res = worst(res, acDeviceTransferVertexBuffer(from, stream, (VertexBufferHandle)q, to));
    return res;
}

/* acDeviceUpdate / acDeviceGetLocalConfig (include/astaroth_device.h:217,246):
 * the same as acDeviceLoadMeshInfo / acDeviceGetConfig on one GPU. */
extern "C" AcResult
acDeviceUpdate(Device d, const AcMeshInfo info)
{
    return acDeviceLoadMeshInfo(d, info);
}

extern "C" AcMeshInfo
acDeviceGetLocalConfig(const Device d)
{
    return acDeviceGetConfig(d);
}

/* acDeviceVolumeCopy (include/astaroth_device.h:235, acc-runtime/api/
 * common_kernels.cc:143-155): copies the box min(in_volume, out_volume) from
 * in at in_offset to out at out_offset, both arrays laid out x fastest with
 * their volume's dims.  Unlike the reference, a box that would reach past
 * either array is refused. */
extern "C" AcResult
acDeviceVolumeCopy(const Device d, const Stream stream, const AcReal* in, const Volume in_offset,
                   const Volume in_volume, AcReal* out, const Volume out_offset,
                   const Volume out_volume)
{
    if (!d || !in || !out || !stream_ok(stream))
        return AC_FAILURE;
    const Volume nn = {in_volume.x < out_volume.x ? in_volume.x : out_volume.x,
                       in_volume.y < out_volume.y ? in_volume.y : out_volume.y,
                       in_volume.z < out_volume.z ? in_volume.z : out_volume.z};
    if (in_offset.x + nn.x > in_volume.x || in_offset.y + nn.y > in_volume.y ||
        in_offset.z + nn.z > in_volume.z || out_offset.x + nn.x > out_volume.x ||
        out_offset.y + nn.y > out_volume.y || out_offset.z + nn.z > out_volume.z)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    AC_CUDA_CHECK(ac_launch_volume_copy(in, in_offset, in_volume, out, out_offset, out_volume, nn,
                                        d->streams[stream], &d->launches));
    return AC_SUCCESS;
}

/* ---- pipelined loads of whole meshes ----
 * acDeviceLoadMeshStaged copies a host mesh into a device-side stage on
 * `stream` and returns at once; acDeviceCommitStagedMesh makes `stream` wait
 * for that copy and moves the stage into the in-buffer (a device copy, or the
 * hi/lo split of FP32-compensated meshes).  A caller that integrates on one
 * stream and stages the next input on another overlaps the host transfer
 * with the integration; the next staged load waits until the commit has read
 * the stage.  Host buffers must be page-locked for the copy to run
 * asynchronously. */
static cudaError_t
ensure_stage(Device d)
{
    if (d->stage)
        return cudaSuccess;
    const size_t n = (size_t)d->geom.mx * d->geom.my * d->geom.mz;
    cudaError_t e  = cudaMalloc((void**)&d->stage, AC_NF * n * sizeof(double));
    if (e != cudaSuccess)
        return e;
    e = cudaEventCreateWithFlags(&d->stage_loaded, cudaEventDisableTiming);
    if (e != cudaSuccess)
        return e;
    return cudaEventCreateWithFlags(&d->stage_read, cudaEventDisableTiming);
}

extern "C" AcResult
acDeviceLoadMeshStaged(const Device d, const Stream stream, const AcMesh host_mesh)
{
    if (!d || !stream_ok(stream))
        return AC_FAILURE;
    for (int q = 0; q < AC_NF; ++q)
        if (!host_mesh.vertex_buffer[q])
            return AC_NOT_ALLOCATED;
    if (!host_matches(d, host_mesh.info)) {
        fprintf(stderr, "astaroth_b200: host mesh dimensions differ from the device's\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const bool first = d->stage == nullptr;
    AC_CUDA_CHECK(ensure_stage(d));
    cudaStream_t st = d->streams[stream];
    if (!first) /* the previous commit has read the stage */
        AC_CUDA_CHECK(cudaStreamWaitEvent(st, d->stage_read, 0));
    const size_t n = (size_t)d->geom.mx * d->geom.my * d->geom.mz;
    for (int q = 0; q < AC_NF; ++q)
        AC_CUDA_CHECK(cudaMemcpyAsync(d->stage + q * n, host_mesh.vertex_buffer[q],
                                      n * sizeof(double), cudaMemcpyHostToDevice, st));
    AC_CUDA_CHECK(cudaEventRecord(d->stage_loaded, st));
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceCommitStagedMesh(const Device d, const Stream stream)
{
    if (!d || !stream_ok(stream) || !d->stage)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    cudaStream_t st = d->streams[stream];
    AC_CUDA_CHECK(cudaStreamWaitEvent(st, d->stage_loaded, 0));
    const size_t n = (size_t)d->geom.mx * d->geom.my * d->geom.mz;
    for (int q = 0; q < AC_NF; ++q) {
        const int b = d->in_idx[q];
        if (d->precision == 0)
            AC_CUDA_CHECK(ac_launch_copy(d->stage + q * n, arr64(d, b, q), (long long)n, st,
                                         &d->launches));
        else
            AC_CUDA_CHECK(ac_launch_split(d->geom, d->stage + q * n, arr_hi(d, b, q),
                                          arr_lo(d, b, q), st, &d->launches));
    }
    AC_CUDA_CHECK(cudaEventRecord(d->stage_read, st));
    return AC_SUCCESS;
}

/* ---- transfers from and to caller-owned device arrays ---- */

extern "C" AcResult
acDeviceLoadMeshDevice(const Device d, const Stream stream, const AcReal* const* src)
{
    if (!d || !src || !stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const size_t n = (size_t)d->geom.mx * d->geom.my * d->geom.mz;
    for (int q = 0; q < AC_NF; ++q) {
        if (!src[q])
            return AC_NOT_ALLOCATED;
        const int b = d->in_idx[q];
        if (d->precision == 0)
            AC_CUDA_CHECK(cudaMemcpyAsync(arr64(d, b, q), src[q], n * sizeof(double),
                                          cudaMemcpyDeviceToDevice, d->streams[stream]));
        else
            AC_CUDA_CHECK(ac_launch_split(d->geom, src[q], arr_hi(d, b, q), arr_lo(d, b, q),
                                          d->streams[stream], &d->launches));
    }
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceStoreMeshDevice(const Device d, const Stream stream, AcReal* const* dst)
{
    if (!d || !dst || !stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const size_t n = (size_t)d->geom.mx * d->geom.my * d->geom.mz;
    for (int q = 0; q < AC_NF; ++q) {
        if (!dst[q])
            return AC_NOT_ALLOCATED;
        const int b = d->in_idx[q];
        if (d->precision == 0)
            AC_CUDA_CHECK(cudaMemcpyAsync(dst[q], arr64(d, b, q), n * sizeof(double),
                                          cudaMemcpyDeviceToDevice, d->streams[stream]));
        else
            AC_CUDA_CHECK(ac_launch_join(d->geom, arr_hi(d, b, q), arr_lo(d, b, q), dst[q],
                                         d->streams[stream], &d->launches));
    }
    return AC_SUCCESS;
}

/* ---- whole-plane copies for a z-slab decomposition ----
 * The halo exchange of the reference's grid layer packs boundary slabs into
 * buffers and unpacks them into the neighbours' ghost zones
 * (src/core/kernels/packing.cuh:59-470, src/core/task.cc:1933-1993).  With a
 * decomposition along z only, a z halo is a run of whole xy planes, contiguous
 * in every field array, so packing is one copy per array: the buffer holds, for
 * each array (the 8 value arrays, then the 8 compensation arrays of FP32
 * meshes), `nplanes` planes of px*my elements. */
static bool
planes_ok(const Device d, const int z0, const int nplanes)
{
    return d && nplanes > 0 && z0 >= 0 && z0 + nplanes <= d->geom.mz;
}

static int
plane_arrays(const Device d)
{
    return d->precision == 0 ? AC_NF : 2 * AC_NF;
}

extern "C" size_t
acDevicePlaneBytes(const Device d)
{
    return d ? (size_t)d->geom.pxy * elem_size(d) * plane_arrays(d) : 0;
}

/* the in-buffer arrays in packing order: the 8 fields, then (FP32-compensated)
 * their 8 compensation arrays */
static void
packing_arrays(const Device d, void* arrays[2 * AC_NF])
{
    const size_t es = elem_size(d);
    for (int a = 0; a < plane_arrays(d); ++a) {
        const int q = a % AC_NF;
        arrays[a]   = a < AC_NF ? (void*)((char*)d->hi[d->in_idx[q]] + (size_t)q * d->geom.cells * es)
                                : (void*)arr_lo(d, d->in_idx[q], q);
    }
}

static AcResult
copy_planes(const Device d, const Stream stream, const int z0, const int nplanes, char* buffer,
            const bool pack)
{
    if (!planes_ok(d, z0, nplanes) || !buffer || !stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const size_t es = elem_size(d);
    void* arrays[2 * AC_NF];
    packing_arrays(d, arrays);
    /* one launch for all arrays (the buffer holds array a at a * bytes) */
    AC_CUDA_CHECK(ac_launch_planes(arrays, plane_arrays(d), (long long)z0 * d->geom.pxy * es,
                                   (long long)nplanes * d->geom.pxy * es, buffer, pack,
                                   d->streams[stream], &d->launches));
    return AC_SUCCESS;
}

extern "C" AcResult
acDevicePackPlanes(const Device d, const Stream stream, const int z0, const int nplanes,
                   void* buffer)
{
    return copy_planes(d, stream, z0, nplanes, (char*)buffer, true);
}

extern "C" AcResult
acDeviceUnpackPlanes(const Device d, const Stream stream, const int z0, const int nplanes,
                     const void* buffer)
{
    return copy_planes(d, stream, z0, nplanes, (char*)buffer, false);
}

/* ---- box copies for a decomposition in x, y and z ----
 * The faces of a decomposition in x or y are strided in every array: one
 * launch gathers the box [start, start + dims) (padded mesh indices) of every
 * array into the buffer, array by array, then z, y, x (x fastest), as the
 * reference's kernel_pack_data does (src/core/kernels/packing.cuh:59-90);
 * unpack scatters it back (kernel_unpack_data, packing.cuh:133-160). */
static bool
box_ok(const Device d, const int3 start, const int3 dims)
{
    const Geom& g = d->geom;
    return dims.x > 0 && dims.y > 0 && dims.z > 0 && start.x >= 0 && start.y >= 0 &&
           start.z >= 0 && (long long)start.x + dims.x <= g.mx &&
           (long long)start.y + dims.y <= g.my && (long long)start.z + dims.z <= g.mz;
}

extern "C" size_t
acDeviceBoxBytes(const Device d, const int3 dims)
{
    if (!d || dims.x <= 0 || dims.y <= 0 || dims.z <= 0)
        return 0;
    return (size_t)dims.x * dims.y * dims.z * elem_size(d) * plane_arrays(d);
}

static AcResult
copy_box(const Device d, const Stream stream, const int3 start, const int3 dims, void* buffer,
         const bool pack)
{
    if (!d || !box_ok(d, start, dims) || !buffer || !stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    void* arrays[2 * AC_NF];
    packing_arrays(d, arrays);
    AC_CUDA_CHECK(ac_launch_box(arrays, plane_arrays(d), elem_size(d), d->geom, start, dims,
                                buffer, pack, d->streams[stream], &d->launches));
    return AC_SUCCESS;
}

extern "C" AcResult
acDevicePackBox(const Device d, const Stream stream, const int3 start, const int3 dims,
                void* buffer)
{
    return copy_box(d, stream, start, dims, buffer, true);
}

extern "C" AcResult
acDeviceUnpackBox(const Device d, const Stream stream, const int3 start, const int3 dims,
                  const void* buffer)
{
    return copy_box(d, stream, start, dims, (void*)buffer, false);
}

/* ---- snapshots of the computational domain: src/core/grid.cc:3792-3935 ----
 * One raw file per field holding the interior nx*ny*nz values (x fastest):
 * <dir>/<field name>-<label>.mesh, or with `segmented`,
 * <dir>/<field name>-segment-<ox>-<oy>-<oz>-<label>.mesh where (ox, oy, oz) is
 * AC_multigpu_offset ((0, 0, 0) on one GPU), the names the reference's grid
 * layer writes without and with distributed I/O.  FP32-compensated meshes are
 * written as the double values hi + lo. */
static const char* const kSnapNames[NUM_VTXBUF_HANDLES] = {
    "VTXBUF_LNRHO", "VTXBUF_UUX", "VTXBUF_UUY", "VTXBUF_UUZ",
    "VTXBUF_AX",    "VTXBUF_AY",  "VTXBUF_AZ",  "VTXBUF_ENTROPY"};

static bool
snapshot_path(const Device d, const char* dir, const char* label, const int segmented,
              const int q, char* out, const size_t len)
{
    const int3 o = d->config.int3_params[AC_multigpu_offset];
    const int n  = segmented ? snprintf(out, len, "%s/%s-segment-%d-%d-%d-%s.mesh", dir,
                                        kSnapNames[q], o.x, o.y, o.z, label)
                             : snprintf(out, len, "%s/%s-%s.mesh", dir, kSnapNames[q], label);
    return n >= 0 && (size_t)n < len;
}

extern "C" AcResult
acDeviceWriteMeshToDisk(const Device d, const char* dir, const char* label, const int segmented)
{
    if (!d || !dir || !label)
        return AC_FAILURE;
    if (mkdir(dir, 0755) != 0 && errno != EEXIST) {
        fprintf(stderr, "astaroth_b200: cannot create %s\n", dir);
        return AC_FAILURE;
    }
    const Geom& g   = d->geom;
    const size_t nm = (size_t)g.mx * g.my * g.mz;
    double* buf     = (double*)malloc(nm * sizeof(double));
    if (!buf)
        return AC_FAILURE;
    AcResult res = AC_SUCCESS;
    for (int q = 0; q < AC_NF && res == AC_SUCCESS; ++q) {
        AcMesh m;
        memset(&m, 0, sizeof(m));
        m.info            = d->config;
        m.vertex_buffer[q] = buf;
        res = acDeviceStoreVertexBuffer(d, STREAM_DEFAULT, (VertexBufferHandle)q, &m);
        if (res != AC_SUCCESS)
            break;
        char path[4096];
        FILE* fp = NULL;
        if (!snapshot_path(d, dir, label, segmented, q, path, sizeof(path)) ||
            !(fp = fopen(path, "wb"))) {
            res = AC_FAILURE;
            break;
        }
        for (int k = 0; k < g.nz && res == AC_SUCCESS; ++k)
            for (int j = 0; j < g.ny; ++j) {
                const double* row = buf + NGHOST + (size_t)g.mx * ((j + NGHOST) +
                                                                  (size_t)g.my * (k + NGHOST));
                if (fwrite(row, sizeof(double), g.nx, fp) != (size_t)g.nx) {
                    res = AC_FAILURE;
                    break;
                }
            }
        if (fclose(fp) != 0)
            res = AC_FAILURE;
    }
    free(buf);
    return res;
}

extern "C" AcResult
acDeviceReadMeshFromDisk(const Device d, const char* dir, const char* label, const int segmented)
{
    if (!d || !dir || !label)
        return AC_FAILURE;
    const Geom& g   = d->geom;
    const size_t nm = (size_t)g.mx * g.my * g.mz;
    double* buf     = (double*)calloc(nm, sizeof(double));
    if (!buf)
        return AC_FAILURE;
    AcResult res = AC_SUCCESS;
    for (int q = 0; q < AC_NF && res == AC_SUCCESS; ++q) {
        char path[4096];
        FILE* fp = NULL;
        if (!snapshot_path(d, dir, label, segmented, q, path, sizeof(path)) ||
            !(fp = fopen(path, "rb"))) {
            fprintf(stderr, "astaroth_b200: cannot open snapshot field %d in %s\n", q, dir);
            res = AC_FAILURE;
            break;
        }
        for (int k = 0; k < g.nz && res == AC_SUCCESS; ++k)
            for (int j = 0; j < g.ny; ++j) {
                double* row = buf + NGHOST + (size_t)g.mx * ((j + NGHOST) +
                                                            (size_t)g.my * (k + NGHOST));
                if (fread(row, sizeof(double), g.nx, fp) != (size_t)g.nx) {
                    res = AC_FAILURE;
                    break;
                }
            }
        /* the file must hold exactly the interior */
        if (res == AC_SUCCESS && fgetc(fp) != EOF)
            res = AC_FAILURE;
        fclose(fp);
        if (res != AC_SUCCESS)
            break;
        AcMesh m;
        memset(&m, 0, sizeof(m));
        m.info            = d->config;
        m.vertex_buffer[q] = buf;
        res = acDeviceLoadVertexBuffer(d, STREAM_DEFAULT, m, (VertexBufferHandle)q);
        if (res == AC_SUCCESS && cudaStreamSynchronize(d->streams[STREAM_DEFAULT]) != cudaSuccess)
            res = AC_FAILURE;
    }
    free(buf);
    if (res != AC_SUCCESS)
        return res;
    /* the halos follow from the interior by the periodic fill */
    const Volume m0 = {0, 0, 0};
    const Volume m1 = {(size_t)g.mx, (size_t)g.my, (size_t)g.mz};
    res = acDevicePeriodicBoundconds(d, STREAM_DEFAULT, m0, m1);
    if (res == AC_SUCCESS)
        res = acDeviceSynchronizeStream(d, STREAM_DEFAULT);
    return res;
}

extern "C" AcResult
acDeviceStoreBfield(const Device d, const Stream stream, AcReal* bx, AcReal* by, AcReal* bz)
{
    if (!d || !stream_ok(stream) || !bx || !by || !bz)
        return AC_FAILURE;
    if (!d->config.int_params[AC_lbfield] || !d->bfield) {
        fprintf(stderr, "astaroth_b200: acDeviceStoreBfield needs AC_lbfield\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const size_t nm = (size_t)d->geom.mx * d->geom.my * d->geom.mz;
    AcReal* out[3]  = {bx, by, bz};
    for (int c = 0; c < 3; ++c)
        AC_CUDA_CHECK(cudaMemcpyAsync(out[c], d->bfield + c * nm, nm * sizeof(double),
                                      cudaMemcpyDeviceToHost, d->streams[stream]));
    AC_CUDA_CHECK(cudaStreamSynchronize(d->streams[stream]));
    return AC_SUCCESS;
}

