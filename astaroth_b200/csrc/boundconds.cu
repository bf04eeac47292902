/*
 * Periodic halo fill, buffer fills and the FP64 <-> FP32-compensated
 * conversions of one field.
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
 * One launch fills all requested arrays (the reference launches once per
 * field, src/core/device.cc:999-1017).  The whole-mesh fill works by rows
 * (x lines): a row with a ghost y or z index is copied whole, by one warp with
 * coalesced accesses, from the row it wraps to, with the x wrap at both ends;
 * a row of the interior (y, z) gets its six x ghosts from one thread.
 * Every source is an interior cell, so no ghost reads another ghost and the
 * order does not matter.  Index arithmetic is 32-bit without divisions by a
 * 64-bit value.
 */
#include "internal.h"
#include "halo.cuh"

namespace {

/* FP32 compensated meshes fill hi and lo of 8 fields (16 arrays); the adjoint
 * fills its 46 derivative-slot arrays. */
constexpr int kMaxArrays = 48;

template <typename T>
struct ArrayList {
    T* p[kMaxArrays];
    int n;
};

template <typename T>
__device__ __forceinline__ void
copy_wrapped(const Geom& g, const ArrayList<T>& fl, const int i, const int j, const int k)
{
    const long long dst = geom_idx(g, i, j, k);
    const long long src = halo_source(g, i, j, k);
#pragma unroll
    for (int q = 0; q < kMaxArrays; ++q)
        if (q < fl.n)
            fl.p[q][dst] = fl.p[q][src];
}

/* Whole mesh by rows.  Blocks [0, blocks_rows) copy the ghost rows, one warp
 * per row; the others fill the six x ghosts of the interior rows, one thread
 * per row.  Sources (interior cells) and destinations (ghost cells) never
 * overlap, so each thread issues its loads before its stores.  blockIdx.y is
 * the array.
 *
 * VEC (every row and array 16-byte aligned): the ghost rows move as 16-byte
 * vectors of the row pitch, a vector inside the x interior straight from the
 * same place of the source row, one with x ghosts (or FP32 row padding, which
 * takes the source row's) element by element; in FP64 with nx even the x
 * ghosts of an interior row move as two 16-byte pairs and two single cells.
 * Half the memory instructions of the 8-byte form (the kernel is bound by the
 * queue of outstanding memory instructions). */
template <typename T, bool VEC>
__global__ void __launch_bounds__(256)
periodic_rows_kernel(const Geom g, const ArrayList<T> fl, const int blocks_rows)
{
    T* a         = fl.p[blockIdx.y];
    const int nx = g.nx, ny = g.ny, nz = g.nz, mx = g.mx, my = g.my;
    constexpr int W = 16 / (int)sizeof(T); /* elements per 16-byte vector */
    union Vec {
        uint4 u;
        T v[W];
    };
    if ((int)blockIdx.x < blocks_rows) {
        /* ghost rows: the 6 ghost z planes (my rows each), then the 6 ghost y
         * rows of each interior z plane */
        const int r    = (int)blockIdx.x * 8 + (int)(threadIdx.x >> 5);
        const int lane = threadIdx.x & 31;
        if (r >= 6 * (my + nz))
            return;
        int j, k;
        if (r < 6 * my) {
            const int kk = r / my;
            j            = r - kk * my;
            k            = kk < NGHOST ? kk : nz + kk;
        }
        else {
            const int u  = r - 6 * my;
            const int jj = u % 6;
            k            = NGHOST + u / 6;
            j            = jj < NGHOST ? jj : ny + jj;
        }
        const int js = (j - NGHOST + ny) % ny + NGHOST;
        const int ks = (k - NGHOST + nz) % nz + NGHOST;
        T* dst       = a + geom_idx(g, 0, j, k);
        const T* src = a + geom_idx(g, 0, js, ks);
        if constexpr (VEC) {
            constexpr int U = 4; /* vectors in flight per lane */
            const int nv    = g.px / W;
            for (int v0 = lane; v0 < nv; v0 += 32 * U) {
                Vec w[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int v = v0 + 32 * u;
                    if (v >= nv)
                        continue;
                    const int e = v * W;
                    if (e >= NGHOST && e + W <= nx + NGHOST) {
                        w[u].u = *reinterpret_cast<const uint4*>(src + e);
                    }
                    else {
#pragma unroll
                        for (int i = 0; i < W; ++i) {
                            const int x  = e + i;
                            const int xs = x < NGHOST ? x + nx : x >= nx + NGHOST && x < mx ? x - nx : x;
                            w[u].v[i]    = src[xs];
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int v = v0 + 32 * u;
                    if (v < nv)
                        *reinterpret_cast<uint4*>(dst + v * W) = w[u].u;
                }
            }
            return;
        }
        constexpr int B = 8; /* loads in flight per lane */
        for (int x0 = lane; x0 < mx; x0 += 32 * B) {
            T v[B];
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const int x  = x0 + 32 * u;
                const int xs = x < NGHOST ? x + nx : x >= nx + NGHOST ? x - nx : x;
                v[u]         = x < mx ? src[xs] : T(0);
            }
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const int x = x0 + 32 * u;
                if (x < mx)
                    dst[x] = v[u];
            }
        }
    }
    else {
        /* the six x ghosts of interior row (j, k): x = 0..2 <- nx..nx+2 and
         * x = nx+3..nx+5 <- 3..5 */
        const int row = ((int)blockIdx.x - blocks_rows) * 256 + (int)threadIdx.x;
        if (row >= ny * nz)
            return;
        const int k = NGHOST + row / ny;
        const int j = NGHOST + row - (row / ny) * ny;
        T* rp       = a + geom_idx(g, 0, j, k);
        if constexpr (VEC && sizeof(T) == 8) {
            if ((nx & 1) == 0) {
                /* (0, 1) <- (nx, nx + 1), 2 <- nx + 2, nx + 3 <- 3,
                 * (nx + 4, nx + 5) <- (4, 5): the pairs 16-byte aligned */
                const uint4 lo = *reinterpret_cast<const uint4*>(rp + nx);
                const T s2     = rp[nx + 2];
                const T s3     = rp[NGHOST];
                const uint4 hi = *reinterpret_cast<const uint4*>(rp + NGHOST + 1);
                *reinterpret_cast<uint4*>(rp) = lo;
                rp[2]                         = s2;
                rp[nx + NGHOST]               = s3;
                *reinterpret_cast<uint4*>(rp + nx + NGHOST + 1) = hi;
                return;
            }
        }
        T v[6];
#pragma unroll
        for (int c = 0; c < NGHOST; ++c) {
            v[c]          = rp[nx + c];
            v[NGHOST + c] = rp[NGHOST + c];
        }
#pragma unroll
        for (int c = 0; c < NGHOST; ++c) {
            rp[c]               = v[c];
            rp[nx + NGHOST + c] = v[NGHOST + c];
        }
    }
}

/* General box [start, end): interior cells are skipped. */
template <typename T>
__global__ void
periodic_box_kernel(const Geom g, const ArrayList<T> fl, const int3 start, const int3 dims)
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

__global__ void
fill_comp_kernel(float* hi, float* lo, const long long count, const float h, const float l)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < count;
         t += (long long)gridDim.x * blockDim.x) {
        hi[t] = h;
        lo[t] = l;
    }
}

/* One field: double (host layout, pitch mx) -> (hi, lo) with pitch px. */
__global__ void
split_kernel(const Geom g, const double* __restrict__ src, float* __restrict__ hi,
             float* __restrict__ lo)
{
    const long long rows = (long long)g.my * g.mz;
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        const double* s = src + r * g.mx;
        float* h        = hi + r * g.px;
        float* l        = lo + r * g.px;
        for (int i = threadIdx.x; i < g.mx; i += blockDim.x) {
            const double v = s[i];
            const float vh = (float)v;
            h[i]           = vh;
            l[i]           = (float)(v - (double)vh);
        }
    }
}

__global__ void
join_kernel(const Geom g, const float* __restrict__ hi, const float* __restrict__ lo,
            double* __restrict__ dst)
{
    const long long rows = (long long)g.my * g.mz;
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        double* d       = dst + r * g.mx;
        const float* h  = hi + r * g.px;
        const float* l  = lo + r * g.px;
        for (int i = threadIdx.x; i < g.mx; i += blockDim.x)
            d[i] = (double)h[i] + (double)l[i];
    }
}

/* A range [first, first + count) of host-layout linear indices (pitch mx) of
 * one field, between doubles at those indices and the (hi, lo) pair of the
 * device layout (pitch px); the same arithmetic as split_kernel / join_kernel. */
__device__ __forceinline__ long long
range_dev_idx(const Geom& g, const long long L)
{
    const long long i = L % g.mx;
    const long long j = (L / g.mx) % g.my;
    const long long k = L / ((long long)g.mx * g.my);
    return i + j * g.px + k * g.pxy;
}

__global__ void
split_range_kernel(const Geom g, const double* __restrict__ src, float* __restrict__ hi,
                   float* __restrict__ lo, const long long first, const long long count)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < count;
         t += (long long)gridDim.x * blockDim.x) {
        const long long L = first + t;
        const long long d = range_dev_idx(g, L);
        const double v    = src[L];
        const float vh    = (float)v;
        hi[d]             = vh;
        lo[d]             = (float)(v - (double)vh);
    }
}

__global__ void
join_range_kernel(const Geom g, const float* __restrict__ hi, const float* __restrict__ lo,
                  double* __restrict__ dst, const long long first, const long long count)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < count;
         t += (long long)gridDim.x * blockDim.x) {
        const long long L = first + t;
        const long long d = range_dev_idx(g, L);
        dst[L]            = (double)hi[d] + (double)lo[d];
    }
}

/* out[(p + out_offset) in out_volume] = in[(p + in_offset) in in_volume] for p
 * in the box nn, x fastest (the reference's AC_VOLUME_COPY,
 * acc-runtime/built-in/kernels.h:43-67). */
__global__ void
volume_copy_kernel(const double* __restrict__ in, const Volume in_offset, const Volume in_volume,
                   double* __restrict__ out, const Volume out_offset, const Volume out_volume,
                   const Volume nn)
{
    const long long total = (long long)nn.x * nn.y * nn.z;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const long long x = t % nn.x, y = (t / nn.x) % nn.y, z = t / ((long long)nn.x * nn.y);
        const long long si = (x + in_offset.x) + (long long)(y + in_offset.y) * in_volume.x +
                             (long long)(z + in_offset.z) * in_volume.x * in_volume.y;
        const long long di = (x + out_offset.x) + (long long)(y + out_offset.y) * out_volume.x +
                             (long long)(z + out_offset.z) * out_volume.x * out_volume.y;
        out[di] = in[si];
    }
}

/* Plane ranges of up to 16 arrays to or from one contiguous buffer, in 8-byte
 * words: word w of array a is arrays[a][offset + w] and buffer[a * count + w]
 * (pack) or the reverse (unpack); grid-stride over all arrays' words. */
struct PlaneArrays {
    unsigned long long* a[2 * AC_NF];
};

__global__ void
planes_kernel(const PlaneArrays arr, const int narrays, const long long offset,
              const long long count, unsigned long long* __restrict__ buffer, const bool pack)
{
    const long long total = (long long)narrays * count;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int a         = (int)(t / count);
        const long long w   = t - (long long)a * count;
        unsigned long long* f = arr.a[a] + offset + w;
        if (pack)
            buffer[t] = *f;
        else
            *f = buffer[t];
    }
}

/* A box of every array <-> the packed buffer (array-major, then z, y, x), the
 * reference's kernel_pack_data / kernel_unpack_data
 * (src/core/kernels/packing.cuh:59-90,133-160) for one element type E. */
template <typename E>
__global__ void
box_kernel(const PlaneArrays arr, const int narrays, const long long px, const long long pxy,
           const int3 start, const int3 dims, E* __restrict__ buffer, const bool pack)
{
    const long long row   = dims.x;
    const long long cells = row * dims.y * dims.z;
    const long long total = (long long)narrays * cells;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int a         = (int)(t / cells);
        const long long c   = t - (long long)a * cells;
        const long long r   = c / row; /* row index within the box: j + dims.y * k */
        const int i         = (int)(c - r * row);
        const int j         = (int)(r % dims.y);
        const int k         = (int)(r / dims.y);
        E* f = reinterpret_cast<E*>(arr.a[a]) + (start.x + i) + (long long)(start.y + j) * px +
               (long long)(start.z + k) * pxy;
        if (pack)
            buffer[t] = *f;
        else
            *f = buffer[t];
    }
}

/* dst = src for n2 double2 pairs (both 16-byte aligned), grid-stride */
__global__ void
copy2_kernel(const double2* __restrict__ src, double2* __restrict__ dst, const long long n2)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n2;
         t += (long long)gridDim.x * blockDim.x)
        dst[t] = src[t];
}

int
grid_for(const long long work, const int tpb)
{
    long long bpg = (work + tpb - 1) / tpb;
    if (bpg > 148LL * 32)
        bpg = 148LL * 32;
    return (int)(bpg > 0 ? bpg : 1);
}

} // namespace

template <typename T>
cudaError_t
ac_launch_periodic(const Geom& g, T* const* arrays, const int n, const Volume start,
                   const Volume end, cudaStream_t stream, unsigned long long* launches)
{
    if (n <= 0 || n > kMaxArrays)
        return cudaErrorInvalidValue;
    if (end.x > (size_t)g.mx || end.y > (size_t)g.my || end.z > (size_t)g.mz ||
        start.x >= end.x || start.y >= end.y || start.z >= end.z)
        return cudaErrorInvalidValue;
    ArrayList<T> fl;
    fl.n = n;
    for (int q = 0; q < kMaxArrays; ++q)
        fl.p[q] = q < n ? arrays[q] : nullptr;

    const bool whole = start.x == 0 && start.y == 0 && start.z == 0 && end.x == (size_t)g.mx &&
                       end.y == (size_t)g.my && end.z == (size_t)g.mz;
    if (whole) {
        const long long ghost_rows = 6LL * (g.my + g.nz);
        const long long irows      = (long long)g.ny * g.nz;
        const long long b_rows     = (ghost_rows + 7) / 8;
        const long long b_cells    = (irows + 255) / 256;
        if (b_rows + b_cells > 0x7fffffffLL)
            return cudaErrorInvalidValue;
        /* the 16-byte form needs every row (pitch) and array 16-byte aligned */
        bool vec = ((long long)g.px * (long long)sizeof(T)) % 16 == 0;
        for (int q = 0; q < n; ++q)
            vec = vec && ((uintptr_t)arrays[q] & 15) == 0;
        if (vec)
            periodic_rows_kernel<T, true><<<dim3((unsigned)(b_rows + b_cells), (unsigned)n), 256,
                                            0, stream>>>(g, fl, (int)b_rows);
        else
            periodic_rows_kernel<T, false><<<dim3((unsigned)(b_rows + b_cells), (unsigned)n), 256,
                                             0, stream>>>(g, fl, (int)b_rows);
    }
    else {
        const int3 s = make_int3((int)start.x, (int)start.y, (int)start.z);
        const int3 d = make_int3((int)(end.x - start.x), (int)(end.y - start.y),
                                 (int)(end.z - start.z));
        const dim3 tpb(32, 8, 1);
        const dim3 bpg((d.x + 31) / 32, (d.y + 7) / 8, d.z);
        periodic_box_kernel<T><<<bpg, tpb, 0, stream>>>(g, fl, s, d);
    }
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

template cudaError_t ac_launch_periodic<double>(const Geom&, double* const*, const int,
                                                const Volume, const Volume, cudaStream_t,
                                                unsigned long long*);
template cudaError_t ac_launch_periodic<float>(const Geom&, float* const*, const int,
                                               const Volume, const Volume, cudaStream_t,
                                               unsigned long long*);

cudaError_t
ac_launch_fill(double* ptr, const long long count, const double value, cudaStream_t stream,
               unsigned long long* launches)
{
    if (count <= 0)
        return cudaSuccess;
    fill_kernel<<<grid_for(count, 256), 256, 0, stream>>>(ptr, count, value);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

cudaError_t
ac_launch_fill_comp(float* hi, float* lo, const long long count, const double value,
                    cudaStream_t stream, unsigned long long* launches)
{
    if (count <= 0)
        return cudaSuccess;
    const float h = (float)value;
    const float l = (float)(value - (double)h);
    fill_comp_kernel<<<grid_for(count, 256), 256, 0, stream>>>(hi, lo, count, h, l);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

cudaError_t
ac_launch_copy(const double* src, double* dst, const long long count, cudaStream_t stream,
               unsigned long long* launches)
{
    if (count <= 0)
        return cudaSuccess;
    if ((count & 1) || ((uintptr_t)src & 15) || ((uintptr_t)dst & 15))
        return cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyDeviceToDevice,
                               stream);
    copy2_kernel<<<grid_for(count / 2, 256), 256, 0, stream>>>((const double2*)src,
                                                              (double2*)dst, count / 2);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

cudaError_t
ac_launch_planes(void* const* arrays, const int narrays, const long long offset_bytes,
                 const long long bytes, void* buffer, const bool pack, cudaStream_t stream,
                 unsigned long long* launches)
{
    if (narrays < 1 || narrays > 2 * AC_NF || (offset_bytes & 7) || (bytes & 7) ||
        ((uintptr_t)buffer & 7))
        return cudaErrorInvalidValue;
    PlaneArrays arr;
    for (int a = 0; a < narrays; ++a) {
        if ((uintptr_t)arrays[a] & 7)
            return cudaErrorInvalidValue;
        arr.a[a] = (unsigned long long*)arrays[a];
    }
    const long long count = bytes / 8;
    planes_kernel<<<grid_for((long long)narrays * count, 256), 256, 0, stream>>>(
        arr, narrays, offset_bytes / 8, count, (unsigned long long*)buffer, pack);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

cudaError_t
ac_launch_box(void* const* arrays, const int narrays, const size_t elem, const Geom& g,
              const int3 start, const int3 dims, void* buffer, const bool pack,
              cudaStream_t stream, unsigned long long* launches)
{
    if (narrays < 1 || narrays > 2 * AC_NF || (elem != 4 && elem != 8) ||
        ((uintptr_t)buffer & (elem - 1)) || dims.x < 1 || dims.y < 1 || dims.z < 1 ||
        start.x < 0 || start.y < 0 || start.z < 0 || start.x + dims.x > g.mx ||
        start.y + dims.y > g.my || start.z + dims.z > g.mz)
        return cudaErrorInvalidValue;
    PlaneArrays arr;
    for (int a = 0; a < narrays; ++a) {
        if ((uintptr_t)arrays[a] & (elem - 1))
            return cudaErrorInvalidValue;
        arr.a[a] = (unsigned long long*)arrays[a];
    }
    const long long total = (long long)narrays * dims.x * dims.y * dims.z;
    if (elem == 8)
        box_kernel<unsigned long long><<<grid_for(total, 256), 256, 0, stream>>>(
            arr, narrays, g.px, g.pxy, start, dims, (unsigned long long*)buffer, pack);
    else
        box_kernel<unsigned int><<<grid_for(total, 256), 256, 0, stream>>>(
            arr, narrays, g.px, g.pxy, start, dims, (unsigned int*)buffer, pack);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

cudaError_t
ac_launch_split_range(const Geom& g, const double* src, float* hi, float* lo,
                      const long long first, const long long count, cudaStream_t stream,
                      unsigned long long* launches)
{
    if (count <= 0)
        return cudaSuccess;
    split_range_kernel<<<grid_for(count, 256), 256, 0, stream>>>(g, src, hi, lo, first, count);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

cudaError_t
ac_launch_join_range(const Geom& g, const float* hi, const float* lo, double* dst,
                     const long long first, const long long count, cudaStream_t stream,
                     unsigned long long* launches)
{
    if (count <= 0)
        return cudaSuccess;
    join_range_kernel<<<grid_for(count, 256), 256, 0, stream>>>(g, hi, lo, dst, first, count);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

cudaError_t
ac_launch_volume_copy(const double* in, const Volume in_offset, const Volume in_volume,
                      double* out, const Volume out_offset, const Volume out_volume,
                      const Volume nn, cudaStream_t stream, unsigned long long* launches)
{
    const long long total = (long long)nn.x * nn.y * nn.z;
    if (total <= 0)
        return cudaSuccess;
    volume_copy_kernel<<<grid_for(total, 256), 256, 0, stream>>>(in, in_offset, in_volume, out,
                                                                out_offset, out_volume, nn);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

cudaError_t
ac_launch_split(const Geom& g, const double* src, float* hi, float* lo, cudaStream_t stream,
                unsigned long long* launches)
{
    split_kernel<<<grid_for((long long)g.my * g.mz * 256, 256), 256, 0, stream>>>(g, src, hi, lo);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

cudaError_t
ac_launch_join(const Geom& g, const float* hi, const float* lo, double* dst, cudaStream_t stream,
               unsigned long long* launches)
{
    join_kernel<<<grid_for((long long)g.my * g.mz * 256, 256), 256, 0, stream>>>(g, hi, lo, dst);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}
