/*
 * Scalar / vector / vector+scalar reductions over the interior, fused in one
 * launch: map -> per-thread accumulate -> warp shuffle -> block -> one atomic
 * ticket per block; the last block to finish combines the per-block partials
 * in a fixed order and writes the single result.
 *
 * Reference: acKernelReduceScal/Vec/VecScal, src/core/kernels/reductions.cu:95-170
 * (a map kernel writing an N^3 scratch array, then cub::DeviceReduce), map
 * kernels acc-runtime/stdlib/map.h:29-150, reduction types stdlib/reduction.h:1-8.
 * Here the map never goes through memory and the traffic is one read of the
 * fields.  Sums are accumulated as double-double (error-free two-sum), so the
 * result is the correctly rounded sum up to the map's own rounding; the
 * order is fixed by the grid, so repeated calls give identical bits.
 */
#include <climits>
#include <mutex>

#include "internal.h"

namespace {

constexpr int kTpb = 256;

struct DD {
    double hi, lo;
};

__device__ __forceinline__ DD
dd_add(const DD x, const double y)
{
    const double s  = x.hi + y;
    const double bb = s - x.hi;
    double e        = (x.hi - (s - bb)) + (y - bb);
    e += x.lo;
    const double hi = s + e;
    return DD{hi, e - (hi - s)};
}

__device__ __forceinline__ DD
dd_add(const DD x, const DD y)
{
    const double s  = x.hi + y.hi;
    const double bb = s - x.hi;
    double e        = (x.hi - (s - bb)) + (y.hi - bb);
    e += x.lo + y.lo;
    const double hi = s + e;
    return DD{hi, e - (hi - s)};
}

/* Reads the value of field q at idx: FP64 arrays, or hi + lo of the FP32
 * compensated representation (exact in double). */
struct Reader64 {
    const double* p[4];
    __device__ __forceinline__ double operator()(const int q, const long long idx) const
    {
        return p[q][idx];
    }
};
struct ReaderComp {
    const float* hi[4];
    const float* lo[4];
    __device__ __forceinline__ double operator()(const int q, const long long idx) const
    {
        return (double)hi[q][idx] + (double)lo[q][idx];
    }
};

template <typename R>
__device__ __forceinline__ double
map_value(const int map, const R& f, const long long idx)
{
    const double a = f(0, idx);
    switch (map) {
    case AC_MAP_VTXBUF:
        return a;
    case AC_MAP_VTXBUF_SQUARE:
        return a * a;
    case AC_MAP_VTXBUF_EXP_SQUARE: {
        const double e = exp(a);
        return e * e;
    }
    default:
        break;
    }
    const double b  = f(1, idx);
    const double c  = f(2, idx);
    const double sq = a * a + b * b + c * c;
    switch (map) {
    case AC_MAP_VTXBUF3_NORM:
        return sqrt(sq);
    case AC_MAP_VTXBUF3_SQUARE:
        return sq;
    case AC_MAP_VTXBUF3_EXP_SQUARE: {
        const double ea = exp(a), eb = exp(b), ec = exp(c);
        return ea * ea + eb * eb + ec * ec;
    }
    case AC_MAP_VTXBUF4_ALFVEN_NORM:
        return sqrt(sq) / sqrt(exp(f(3, idx)));
    case AC_MAP_VTXBUF4_ALFVEN_SQUARE:
        return sq / exp(f(3, idx));
    default:
        return 0;
    }
}

__device__ __forceinline__ double
combine(const int op, const double a, const double b)
{
    return op == AC_REDUCE_OP_MAX ? fmax(a, b) : fmin(a, b);
}

/* nonfinite (optional): set to 1 when a mapped value is NaN or infinite, which a
 * maximum or minimum would otherwise hide (fmax and fmin drop NaN) */
template <typename R>
__global__ void __launch_bounds__(kTpb)
reduce_kernel(const Geom g, const R f, const int map, const int op,
              double* __restrict__ partials, unsigned int* __restrict__ counter,
              double* __restrict__ result, unsigned int* __restrict__ nonfinite)
{
    __shared__ double s_hi[kTpb / 32];
    __shared__ double s_lo[kTpb / 32];
    __shared__ bool s_last;
    const bool is_sum  = op == AC_REDUCE_OP_SUM;
    const double ident = op == AC_REDUCE_OP_MAX ? -INFINITY : INFINITY;

    DD acc{0.0, 0.0};
    double ext          = ident;
    bool bad            = false;
    const long long rows = (long long)g.ny * g.nz;
    for (long long r = blockIdx.x; r < rows; r += gridDim.x) {
        const int j          = (int)(r % g.ny);
        const int k          = (int)(r / g.ny);
        const long long base = geom_idx(g, NGHOST, j + NGHOST, k + NGHOST);
        for (int i = threadIdx.x; i < g.nx; i += kTpb) {
            const double v = map_value(map, f, base + i);
            bad |= !isfinite(v);
            if (is_sum)
                acc = dd_add(acc, v);
            else
                ext = combine(op, ext, v);
        }
    }
    if (__syncthreads_or(bad) && nonfinite && threadIdx.x == 0)
        atomicOr(nonfinite, 1u);
    /* warp */
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        if (is_sum) {
            DD other{__shfl_xor_sync(0xffffffffu, acc.hi, o),
                     __shfl_xor_sync(0xffffffffu, acc.lo, o)};
            acc = dd_add(acc, other);
        }
        else {
            ext = combine(op, ext, __shfl_xor_sync(0xffffffffu, ext, o));
        }
    }
    if (lane == 0) {
        s_hi[warp] = is_sum ? acc.hi : ext;
        s_lo[warp] = is_sum ? acc.lo : 0.0;
    }
    __syncthreads();
    /* block */
    if (threadIdx.x == 0) {
        DD b{0.0, 0.0};
        double e = ident;
        for (int w = 0; w < kTpb / 32; ++w) {
            if (is_sum)
                b = dd_add(b, DD{s_hi[w], s_lo[w]});
            else
                e = combine(op, e, s_hi[w]);
        }
        partials[2 * blockIdx.x]     = is_sum ? b.hi : e;
        partials[2 * blockIdx.x + 1] = is_sum ? b.lo : 0.0;
        __threadfence();
        const unsigned int ticket = atomicAdd(counter, 1u);
        s_last                    = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last)
        return;
    /* last block: combine the partials in block order */
    __threadfence();
    DD t{0.0, 0.0};
    double e = ident;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kTpb) {
        const volatile double* vp = partials;
        if (is_sum)
            t = dd_add(t, DD{vp[2 * b], vp[2 * b + 1]});
        else
            e = combine(op, e, vp[2 * b]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        if (is_sum) {
            DD other{__shfl_xor_sync(0xffffffffu, t.hi, o), __shfl_xor_sync(0xffffffffu, t.lo, o)};
            t = dd_add(t, other);
        }
        else {
            e = combine(op, e, __shfl_xor_sync(0xffffffffu, e, o));
        }
    }
    if (lane == 0) {
        s_hi[warp] = is_sum ? t.hi : e;
        s_lo[warp] = is_sum ? t.lo : 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        DD b{0.0, 0.0};
        double x = ident;
        for (int w = 0; w < kTpb / 32; ++w) {
            if (is_sum)
                b = dd_add(b, DD{s_hi[w], s_lo[w]});
            else
                x = combine(op, x, s_hi[w]);
        }
        *result  = is_sum ? b.hi + b.lo : x;
        *counter = 0u;
    }
}

} // namespace

int
ac_reduce_blocks(const Geom& g)
{
    const long long rows = (long long)g.ny * g.nz;
    const long long cap  = 148LL * 8;
    return (int)(rows < cap ? rows : cap);
}

cudaError_t
ac_launch_reduce(const Geom& g, const void* const* fields, const float* const* lo,
                 const int nfields, const int precision, const int map, const int op,
                 const ReduceScratch& scratch, cudaStream_t stream, unsigned long long* launches)
{
    if (nfields < 1 || nfields > 4)
        return cudaErrorInvalidValue;
    if (op != AC_REDUCE_OP_SUM && op != AC_REDUCE_OP_MAX && op != AC_REDUCE_OP_MIN)
        return cudaErrorInvalidValue;
    const int blocks = ac_reduce_blocks(g);
    if (blocks > scratch.max_blocks)
        return cudaErrorInvalidValue;
    if (precision == 0) {
        Reader64 f;
        for (int q = 0; q < 4; ++q)
            f.p[q] = (const double*)fields[q < nfields ? q : 0];
        reduce_kernel<<<blocks, kTpb, 0, stream>>>(g, f, map, op, scratch.partials,
                                                   scratch.counter, scratch.result,
                                                   scratch.nonfinite);
    }
    else {
        ReaderComp f;
        for (int q = 0; q < 4; ++q) {
            f.hi[q] = (const float*)fields[q < nfields ? q : 0];
            f.lo[q] = lo[q < nfields ? q : 0];
        }
        reduce_kernel<<<blocks, kTpb, 0, stream>>>(g, f, map, op, scratch.partials,
                                                   scratch.counter, scratch.result,
                                                   scratch.nonfinite);
    }
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

/* ------------------------------------------------------------------------
 * Reduction without any allocation (acReduceNoAlloc).
 *
 * For callers that must not allocate device memory: an application or
 * framework that owns all of the GPU's memory through its own pool or arena
 * (where a cudaMalloc outside the pool can fail once the pool has reserved the
 * memory, and where cudaFree would synchronize the whole device), or a coupled
 * code that runs under a fixed memory budget.  Such a caller keeps its fields
 * in its own buffers and only wants the reduced value.
 *
 * The per-block partials and the block-completion counter of the reduction
 * kernel above live in this file-scope device array instead of in memory that
 * acDeviceCreate allocated.  Every GPU that loads the library holds one copy
 * (33 KB) until the process exits.  The array is shared by all calls on a
 * device: calls that overlap on the GPU (for example on two streams) race on
 * it and must be ordered by the caller.
 * ---------------------------------------------------------------------- */
namespace {

constexpr int kNoAllocMaxBlocks = AC_REDUCE_NOALLOC_MAX_BLOCKS;
/* [2 * kNoAllocMaxBlocks partials][counter word] */
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxBlocks + 32];

constexpr int kMaxDevicesNoAlloc = 64;
double* g_noalloc_ptr[kMaxDevicesNoAlloc]; /* device address of the array, per device */
std::mutex g_noalloc_mutex;                /* guards the one-time fill of g_noalloc_ptr */

} // namespace

extern "C" AcResult
acReduceNoAlloc(const AcReal* const* fields, const int nfields, const int nx, const int ny,
                const int nz, const AcReduction reduction, AcReal* result, const int blocks,
                void* stream)
{
    if (!fields || !result || nx <= 0 || ny <= 0 || nz <= 0) {
        fprintf(stderr, "acReduceNoAlloc: null pointer or empty mesh\n");
        return AC_FAILURE;
    }
    /* the padded extents n + 6 must fit an int (the kernel's row indices) */
    if (nx > INT_MAX - 2 * NGHOST || ny > INT_MAX - 2 * NGHOST || nz > INT_MAX - 2 * NGHOST) {
        fprintf(stderr, "acReduceNoAlloc: mesh extent too large (%d, %d, %d)\n", nx, ny, nz);
        return AC_FAILURE;
    }
    if (blocks < 0) {
        fprintf(stderr, "acReduceNoAlloc: negative block count %d\n", blocks);
        return AC_FAILURE;
    }
    if (nfields != 1 && nfields != 3 && nfields != 4) {
        fprintf(stderr, "acReduceNoAlloc: nfields must be 1, 3 or 4 (got %d)\n", nfields);
        return AC_FAILURE;
    }
    for (int q = 0; q < nfields; ++q)
        if (!fields[q]) {
            fprintf(stderr, "acReduceNoAlloc: fields[%d] is NULL\n", q);
            return AC_FAILURE;
        }
    const int map = nfields == 1 ? reduction.map_vtxbuf_single
                    : nfields == 3 ? reduction.map_vtxbuf_vec
                                   : reduction.map_vtxbuf_vec_scal;
    const bool map_ok = nfields == 1 ? (map >= AC_MAP_VTXBUF && map <= AC_MAP_VTXBUF_EXP_SQUARE)
                        : nfields == 3 ? (map >= AC_MAP_VTXBUF3_NORM &&
                                          map <= AC_MAP_VTXBUF3_EXP_SQUARE)
                                       : (map >= AC_MAP_VTXBUF4_ALFVEN_NORM &&
                                          map <= AC_MAP_VTXBUF4_ALFVEN_SQUARE);
    const int op = reduction.reduce_op;
    if (!map_ok || (op != AC_REDUCE_OP_SUM && op != AC_REDUCE_OP_MAX && op != AC_REDUCE_OP_MIN)) {
        fprintf(stderr, "acReduceNoAlloc: reduction type does not fit %d field(s)\n", nfields);
        return AC_FAILURE;
    }

    Geom g;
    g.nx    = nx;
    g.ny    = ny;
    g.nz    = nz;
    g.mx    = nx + 2 * NGHOST;
    g.my    = ny + 2 * NGHOST;
    g.mz    = nz + 2 * NGHOST;
    g.px    = g.mx;
    g.pxy   = (long long)g.px * g.my;
    g.cells = g.pxy * g.mz;

    const int nb = blocks > 0 ? blocks : ac_reduce_blocks(g);
    if (nb > kNoAllocMaxBlocks) {
        fprintf(stderr,
                "acReduceNoAlloc: %d blocks requested, the static scratch holds at most %d\n",
                nb, kNoAllocMaxBlocks);
        return AC_FAILURE;
    }

    /* One-time set-up per device, on the first call with that device current:
     * the device address of the scratch array.  In host code the array's name
     * stands for a host-side shadow, not a device address. */
    int dev = 0;
    AC_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevicesNoAlloc) {
        fprintf(stderr, "acReduceNoAlloc: device %d beyond the supported %d\n", dev,
                kMaxDevicesNoAlloc);
        return AC_FAILURE;
    }
    double* partials = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            AC_CUDA_CHECK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
            g_noalloc_ptr[dev] = (double*)p;
        }
        partials = g_noalloc_ptr[dev];
    }
    unsigned int* counter = (unsigned int*)(partials + 2 * kNoAllocMaxBlocks);
    cudaStream_t st       = (cudaStream_t)stream;

    /* the completion counter must start at zero; the partials need no clearing */
    AC_CUDA_CHECK(cudaMemsetAsync(counter, 0, sizeof(unsigned int), st));
    Reader64 f;
    for (int q = 0; q < 4; ++q)
        f.p[q] = fields[q < nfields ? q : 0];
    reduce_kernel<<<nb, kTpb, 0, st>>>(g, f, map, op, partials, counter, result, nullptr);
    AC_CUDA_CHECK(cudaGetLastError());
    return AC_SUCCESS;
}
