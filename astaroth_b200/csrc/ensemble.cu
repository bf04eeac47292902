/*
 * Ensembles of independent meshes on one GPU (acEnsemble*; no counterpart in
 * the reference, whose device layer integrates one mesh per Device,
 * src/core/device.cc:941-997).
 *
 * Layout: one allocation holds every member's two buffers (in/out), each a
 * block of 8 fields in the single-mesh layout (x fastest, 3-cell halos; FP32
 * rows padded to a multiple of 4 elements, plus the 8 compensation arrays).
 * A device table of member records holds each member's geometry, field
 * pointers for both buffer parities, stencil coefficients and physics
 * constants; the member timesteps live in a device array, so a captured step
 * reads the current values.
 *
 * A step is 3 x [halo fill, solve, swap]:
 *  - the halo fill is one launch over the ghost cells of all members (a
 *    prefix sum of the members' ghost-cell counts maps a thread to a member);
 *  - the solve is one persistent launch: a grid of (SMs x resident blocks)
 *    walks a work list of tiles (member, x0, y0, z0) of tx * ty cells and zb
 *    planes; a block copies the record of an item's member into shared memory
 *    and computes each cell with plain_cell, the per-cell function of the
 *    single-mesh plain kernel, so a member's result is bit-identical to a
 *    Device of that member without tiling;
 *  - the whole step is captured once per buffer parity as a CUDA graph.
 * acEnsembleAutotune times the solve over a fixed set of tile shapes and
 * keeps the fastest.
 */
#include <algorithm>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <vector>

#include "halo.cuh"
#include "internal.h"
#include "solve_cell.cuh"

namespace {

template <typename T>
struct EnsMember {
    Geom g;
    FieldsT<T> f[2];       /* f[p]: the fields with the in-buffer in block p */
    BlockFieldsT<T> bf[2]; /* the same as block bases and a field stride */
    StencilT<T> sc;
    PhysConst pc;
    long long halo_nzs, halo_nys;
};

/* Cooperative copy of a record (a multiple of 4 bytes) into shared memory. */
__device__ __forceinline__ void
copy_words(void* dst, const void* src, const int bytes)
{
    const unsigned* s = (const unsigned*)src;
    unsigned* d       = (unsigned*)dst;
    for (int w = threadIdx.x; w < bytes / 4; w += blockDim.x)
        d[w] = s[w];
}

/* Persistent solve: block b takes items b, b + grid, b + 2 grid, ...  All
 * control flow around the barriers depends only on the item, so it is uniform
 * across the block. */
template <typename T, bool COMP>
__global__ void __launch_bounds__(256)
ens_solve_kernel(const EnsMember<T>* __restrict__ mem, const int4* __restrict__ items,
                 const int nitems, const double* __restrict__ dts, const int parity,
                 const RkCoef rk, const int tx, const int zb)
{
    __shared__ Geom g;
    __shared__ BlockFieldsT<T> f;
    __shared__ StencilT<T> sc;
    __shared__ PhysConst pc;
    __shared__ double dt;
    const int lx = threadIdx.x % tx, ly = threadIdx.x / tx;
    int cur      = -1;
    for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
        const int4 it = items[w];
        if (it.x != cur) {
            __syncthreads(); /* the previous member's record is no longer read */
            const EnsMember<T>* m = mem + it.x;
            copy_words(&g, &m->g, sizeof(Geom));
            copy_words(&f, &m->bf[parity], sizeof(BlockFieldsT<T>));
            copy_words(&sc, &m->sc, sizeof(StencilT<T>));
            copy_words(&pc, &m->pc, sizeof(PhysConst));
            if (threadIdx.x == 0)
                dt = dts[it.x];
            __syncthreads();
            cur = it.x;
        }
        RkCoef r = rk;
        r.dt     = dt;
        const BlockFieldsT<T> bf = f;
        const int i = it.y + lx, j = it.z + ly;
        if (i < g.nx && j < g.ny) {
            const int k1 = min(it.w + zb, g.nz);
            T cm[3];
            for (int k = it.w; k < k1; ++k)
                plain_cell<T, COMP>(g, bf, sc, pc, r, false, i, j, k, cm);
        }
    }
}

/* Halo fill of every member's in-buffer: thread t handles ghost cell t of the
 * concatenation of all members' ghost cells; prefix[m] is the first ghost
 * cell of member m, prefix[n] the total. */
template <typename T, bool COMP>
__global__ void
ens_halo_kernel(const EnsMember<T>* __restrict__ mem, const long long* __restrict__ prefix,
                const int n, const int parity, const long long total)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = n; /* prefix[lo] <= t < prefix[hi] */
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (prefix[mid] <= t)
                lo = mid;
            else
                hi = mid;
        }
        const EnsMember<T>* m = mem + lo;
        const Geom g          = m->g;
        int i, j, k;
        halo_cell(g, t - prefix[lo], m->halo_nzs, m->halo_nys, i, j, k);
        const long long dst = geom_idx(g, i, j, k);
        const long long src = halo_source(g, i, j, k);
#pragma unroll
        for (int q = 0; q < AC_NF; ++q) {
            T* a   = const_cast<T*>(m->f[parity].in[q]);
            a[dst] = a[src];
            if constexpr (COMP) {
                T* l   = const_cast<T*>(m->f[parity].in_lo[q]);
                l[dst] = l[src];
            }
        }
    }
}

size_t
align_up(const size_t v, const size_t a)
{
    return (v + a - 1) / a * a;
}

} // namespace

struct ensemble_s {
    int id, n, precision;
    int parity; /* block holding every member's in-buffer */
    int sms;
    std::vector<AcMeshInfo> info;
    std::vector<Geom> geom;
    std::vector<StencilCoef> sc; /* double coefficients, for the sequential launches */
    std::vector<PhysConst> pc;
    std::vector<double> dts;
    std::vector<size_t> offset; /* byte offset of each member's buffers in the pool */
    void* hmem;                 /* host EnsMember<T>[n] */
    void* dmem;                 /* device copy */
    char* pool;
    double* d_dts;
    long long* halo_prefix;
    long long halo_total;
    long long cells;
    int4* items;
    int nitems, items_cap;
    AcEnsembleTiles tiles;
    int grid;
    cudaStream_t stream;
    cudaGraphExec_t graph[2];
    int graph_valid[2];
    double* staging;
    ReduceScratch red;
    double* host_result;
    unsigned long long launches;
    /* mode 1: per-member tensor maps of both buffer parities, branch streams */
    std::vector<CUtensorMap> tmaps; /* 2 per member: [2 m + parity] */
    std::vector<char> tiled;        /* member fits the tiled kernel (else: plain) */
    std::vector<cudaStream_t> branches;
    std::vector<cudaEvent_t> joins;
    cudaEvent_t fork;
    int* err;
};

namespace {

template <typename T>
const EnsMember<T>*
members(const Ensemble e)
{
    return (const EnsMember<T>*)e->hmem;
}

void
invalidate(Ensemble e)
{
    for (int p = 0; p < 2; ++p) {
        if (e->graph_valid[p])
            cudaGraphExecDestroy(e->graph[p]);
        e->graph_valid[p] = 0;
    }
}

void
destroy(Ensemble e)
{
    if (!e)
        return;
    cudaSetDevice(e->id);
    if (e->stream)
        cudaStreamSynchronize(e->stream);
    invalidate(e);
    cudaFree(e->pool);
    cudaFree(e->dmem);
    cudaFree(e->d_dts);
    cudaFree(e->halo_prefix);
    cudaFree(e->items);
    cudaFree(e->staging);
    cudaFree(e->red.partials);
    cudaFree(e->err);
    cudaFreeHost(e->host_result);
    for (cudaStream_t b : e->branches)
        cudaStreamDestroy(b);
    for (cudaEvent_t j : e->joins)
        cudaEventDestroy(j);
    if (e->fork)
        cudaEventDestroy(e->fork);
    if (e->stream)
        cudaStreamDestroy(e->stream);
    free(e->hmem);
    delete e;
}

template <typename T, bool COMP>
void
fill_members(Ensemble e)
{
    EnsMember<T>* hm = (EnsMember<T>*)e->hmem;
    for (int m = 0; m < e->n; ++m) {
        EnsMember<T>& r = hm[m];
        memset(&r, 0, sizeof(r));
        r.g              = e->geom[m];
        const size_t fb  = (size_t)r.g.cells * sizeof(T);
        char* base       = e->pool + e->offset[m];
        /* block b: [hi of 8 fields][lo of 8 fields (FP32)] */
        const size_t blk = align_up((size_t)AC_NF * fb * (COMP ? 2 : 1), 256);
        for (int p = 0; p < 2; ++p)
            for (int q = 0; q < AC_NF; ++q) {
                T* in_hi     = (T*)(base + p * blk + q * fb);
                T* out_hi    = (T*)(base + (1 - p) * blk + q * fb);
                r.f[p].in[q]  = in_hi;
                r.f[p].out[q] = out_hi;
                if (COMP) {
                    r.f[p].in_lo[q]  = (T*)(base + p * blk + (AC_NF + q) * fb);
                    r.f[p].out_lo[q] = (T*)(base + (1 - p) * blk + (AC_NF + q) * fb);
                }
            }
        for (int p = 0; p < 2; ++p) {
            r.bf[p].in     = r.f[p].in[0];
            r.bf[p].in_lo  = r.f[p].in_lo[0];
            r.bf[p].out    = r.f[p].out[0];
            r.bf[p].out_lo = r.f[p].out_lo[0];
            r.bf[p].stride = r.g.cells;
        }
        r.sc = stencil_cast<T>(e->sc[m]);
        r.pc = e->pc[m];
        halo_count(r.g, &r.halo_nzs, &r.halo_nys);
    }
}

size_t
member_bytes(const Geom& g, const int precision)
{
    const size_t fb = (size_t)g.cells * (precision == 0 ? sizeof(double) : sizeof(float));
    return 2 * align_up((size_t)AC_NF * fb * (precision == 0 ? 1 : 2), 256);
}

cudaError_t
build_items(Ensemble e, const AcEnsembleTiles t)
{
    /* largest members first, so the last wave holds the small items */
    std::vector<int> order(e->n);
    for (int m = 0; m < e->n; ++m)
        order[m] = m;
    std::stable_sort(order.begin(), order.end(), [&](const int a, const int b) {
        return e->geom[a].nx * (long long)e->geom[a].ny * e->geom[a].nz >
               e->geom[b].nx * (long long)e->geom[b].ny * e->geom[b].nz;
    });
    std::vector<int4> items;
    for (const int m : order) {
        const Geom& g = e->geom[m];
        for (int z = 0; z < g.nz; z += t.zb)
            for (int y = 0; y < g.ny; y += t.ty)
                for (int x = 0; x < g.nx; x += t.tx)
                    items.push_back(make_int4(m, x, y, z));
    }
    if ((int)items.size() > e->items_cap) {
        cudaFree(e->items);
        e->items     = nullptr;
        e->items_cap = 0;
        cudaError_t err = cudaMalloc((void**)&e->items, items.size() * sizeof(int4));
        if (err != cudaSuccess)
            return err;
        e->items_cap = (int)items.size();
    }
    cudaError_t err = cudaMemcpyAsync(e->items, items.data(), items.size() * sizeof(int4),
                                      cudaMemcpyHostToDevice, e->stream);
    if (err != cudaSuccess)
        return err;
    err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess)
        return err;
    e->nitems = (int)items.size();

    const int threads = t.tx * t.ty;
    int occ           = 0;
    err = e->precision == 0
              ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &occ, ens_solve_kernel<double, false>, threads, 0)
              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &occ, ens_solve_kernel<float, true>, threads, 0);
    if (err != cudaSuccess)
        return err;
    if (occ < 1)
        return cudaErrorInvalidConfiguration;
    const int bps = t.blocks_per_sm > 0 ? std::min(t.blocks_per_sm, occ) : occ;
    e->grid       = std::max(1, std::min(e->nitems, e->sms * bps));
    e->tiles      = t;
    invalidate(e);
    return cudaSuccess;
}

bool
tiles_ok(const AcEnsembleTiles t)
{
    const int threads = t.tx * t.ty;
    return t.tx >= 1 && t.ty >= 1 && t.zb >= 1 && threads <= 256 && threads % 32 == 0 &&
           t.blocks_per_sm >= 0 && (t.mode == 0 || t.mode == 1);
}

cudaError_t
launch_solve(Ensemble e, const int step, unsigned long long* launches)
{
    const RkCoef rk = ac_rk_coef(step, 0.0); /* dt comes from the device array */
    const int threads = e->tiles.tx * e->tiles.ty;
    if (e->precision == 0)
        ens_solve_kernel<double, false><<<e->grid, threads, 0, e->stream>>>(
            (const EnsMember<double>*)e->dmem, e->items, e->nitems, e->d_dts, e->parity, rk,
            e->tiles.tx, e->tiles.zb);
    else
        ens_solve_kernel<float, true><<<e->grid, threads, 0, e->stream>>>(
            (const EnsMember<float>*)e->dmem, e->items, e->nitems, e->d_dts, e->parity, rk,
            e->tiles.tx, e->tiles.zb);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

cudaError_t
launch_halo(Ensemble e, unsigned long long* launches)
{
    const int tpb         = 256;
    const long long need  = (e->halo_total + tpb - 1) / tpb;
    const int blocks      = (int)std::min<long long>(need, (long long)e->sms * 8);
    if (e->precision == 0)
        ens_halo_kernel<double, false><<<blocks, tpb, 0, e->stream>>>(
            (const EnsMember<double>*)e->dmem, e->halo_prefix, e->n, e->parity, e->halo_total);
    else
        ens_halo_kernel<float, true><<<blocks, tpb, 0, e->stream>>>(
            (const EnsMember<float>*)e->dmem, e->halo_prefix, e->n, e->parity, e->halo_total);
    if (launches)
        ++*launches;
    return cudaGetLastError();
}

/* Mode 1: the substeps [s0, s1) of every member as tiled single-mesh launches,
 * member chains spread over the branch streams, which fork from and join into
 * the ensemble stream (so a capture of the ensemble stream records them as
 * concurrent branches).  The in-block parity of substep s is parity ^ (s & 1)
 * relative to s0. */
template <typename T, bool COMP>
cudaError_t
record_members(Ensemble e, const int s0, const int s1, unsigned long long* launches,
               const bool halo = true)
{
    cudaError_t err = cudaEventRecord(e->fork, e->stream);
    if (err != cudaSuccess)
        return err;
    const int nb = (int)e->branches.size();
    for (int b = 0; b < nb; ++b) {
        err = cudaStreamWaitEvent(e->branches[b], e->fork, 0);
        if (err != cudaSuccess)
            return err;
    }
    const Volume m0 = {0, 0, 0};
    for (int m = 0; m < e->n; ++m) {
        cudaStream_t st       = e->branches[m % nb];
        const EnsMember<T>& r = members<T>(e)[m];
        const Volume m1       = {(size_t)r.g.mx, (size_t)r.g.my, (size_t)r.g.mz};
        for (int s = s0; s < s1; ++s) {
            const int p         = e->parity ^ ((s - s0) & 1);
            const FieldsT<T>& f = r.f[p];
            T* arr[2 * AC_NF];
            for (int q = 0; q < AC_NF; ++q) {
                arr[q]         = const_cast<T*>(f.in[q]);
                arr[AC_NF + q] = COMP ? const_cast<T*>(f.in_lo[q]) : nullptr;
            }
            if (halo) {
                err = ac_launch_periodic<T>(r.g, arr, COMP ? 2 * AC_NF : AC_NF, m0, m1, st,
                                            launches);
                if (err != cudaSuccess)
                    return err;
            }
            const RkCoef rk     = ac_rk_coef(s, e->dts[m]);
            const void* tmap    = &e->tmaps[2 * m + p];
            /* the kernel a Device of this member would use */
            if constexpr (COMP)
                err = e->tiled[m] ? ac_launch_solve_tiled32(r.g, tmap, f, e->sc[m], e->pc[m], rk,
                                                            e->err, nullptr, st, launches,
                                                            AC_SOLVE_TILED_AUTO)
                                  : ac_launch_solve_plain32(r.g, f, e->sc[m], e->pc[m], rk, nullptr,
                                                            st, launches);
            else
                err = e->tiled[m] ? ac_launch_solve_tiled64(r.g, tmap, f, e->sc[m], e->pc[m], rk,
                                                            e->err, nullptr, st, launches,
                                                            AC_SOLVE_TILED_AUTO)
                                  : ac_launch_solve_plain64(r.g, f, e->sc[m], e->pc[m], rk, nullptr,
                                                            st, launches);
            if (err != cudaSuccess)
                return err;
        }
    }
    for (int b = 0; b < nb; ++b) {
        err = cudaEventRecord(e->joins[b], e->branches[b]);
        if (err != cudaSuccess)
            return err;
        err = cudaStreamWaitEvent(e->stream, e->joins[b], 0);
        if (err != cudaSuccess)
            return err;
    }
    return cudaSuccess;
}

cudaError_t
record_step(Ensemble e, unsigned long long* launches)
{
    if (e->tiles.mode == 1) {
        const cudaError_t err = e->precision == 0 ? record_members<double, false>(e, 0, 3, launches)
                                                  : record_members<float, true>(e, 0, 3, launches);
        if (err == cudaSuccess)
            e->parity ^= 1; /* three swaps */
        return err;
    }
    for (int s = 0; s < 3; ++s) {
        cudaError_t err = launch_halo(e, launches);
        if (err != cudaSuccess)
            return err;
        err = launch_solve(e, s, launches);
        if (err != cudaSuccess)
            return err;
        e->parity ^= 1;
    }
    return cudaSuccess;
}

template <typename T, bool COMP>
cudaError_t
sequential_step(Ensemble e)
{
    const Volume m0 = {0, 0, 0};
    for (int s = 0; s < 3; ++s) {
        for (int m = 0; m < e->n; ++m) {
            const EnsMember<T>& r = members<T>(e)[m];
            const FieldsT<T>& f   = r.f[e->parity];
            T* arr[2 * AC_NF];
            for (int q = 0; q < AC_NF; ++q) {
                arr[q]         = const_cast<T*>(f.in[q]);
                arr[AC_NF + q] = COMP ? const_cast<T*>(f.in_lo[q]) : nullptr;
            }
            const Volume m1 = {(size_t)r.g.mx, (size_t)r.g.my, (size_t)r.g.mz};
            cudaError_t err = ac_launch_periodic<T>(r.g, arr, COMP ? 2 * AC_NF : AC_NF, m0, m1,
                                                    e->stream, &e->launches);
            if (err != cudaSuccess)
                return err;
            const RkCoef rk = ac_rk_coef(s, e->dts[m]);
            if constexpr (COMP)
                err = ac_launch_solve_plain32(r.g, f, e->sc[m], e->pc[m], rk, nullptr, e->stream,
                                              &e->launches);
            else
                err = ac_launch_solve_plain64(r.g, f, e->sc[m], e->pc[m], rk, nullptr, e->stream,
                                              &e->launches);
            if (err != cudaSuccess)
                return err;
        }
        e->parity ^= 1;
    }
    return cudaSuccess;
}

bool
member_ok(const Ensemble e, const int m)
{
    return e && m >= 0 && m < e->n;
}

bool
host_matches(const Ensemble e, const int m, const AcMeshInfo& host)
{
    AcMeshInfo h = host;
    if (acHostUpdateParams(&h) != AC_SUCCESS)
        return false;
    const int3 mm = h.int3_params[AC_mlocal];
    const Geom& g = e->geom[m];
    return mm.x == g.mx && mm.y == g.my && mm.z == g.mz;
}

/* pointers of field q of member m's in-buffer */
void
member_arrays(const Ensemble e, const int m, const int q, void** hi, float** lo)
{
    if (e->precision == 0) {
        const EnsMember<double>& r = members<double>(e)[m];
        *hi                        = const_cast<double*>(r.f[e->parity].in[q]);
        *lo                        = nullptr;
    }
    else {
        const EnsMember<float>& r = members<float>(e)[m];
        *hi                       = const_cast<float*>(r.f[e->parity].in[q]);
        *lo                       = const_cast<float*>(r.f[e->parity].in_lo[q]);
    }
}

AcResult
reduce_member(const Ensemble e, const int m, const AcReduction r, const int kind,
              const VertexBufferHandle* h, AcReal* result)
{
    if (!member_ok(e, m) || !result)
        return AC_FAILURE;
    for (int q = 0; q < kind; ++q)
        if ((int)h[q] < 0 || h[q] >= NUM_VTXBUF_HANDLES)
            return AC_NOT_ALLOCATED;
    const int map = kind == 1 ? r.map_vtxbuf_single : r.map_vtxbuf_vec;
    const bool ok = kind == 1 ? (map >= AC_MAP_VTXBUF && map <= AC_MAP_VTXBUF_EXP_SQUARE)
                              : (map >= AC_MAP_VTXBUF3_NORM && map <= AC_MAP_VTXBUF3_EXP_SQUARE);
    if (!ok) {
        fprintf(stderr, "astaroth_b200: invalid reduction type for this call\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(e->id));
    const void* fp[4];
    const float* lo[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int q = 0; q < kind; ++q) {
        void* hi;
        float* l;
        member_arrays(e, m, h[q], &hi, &l);
        fp[q] = hi;
        lo[q] = l;
    }
    const Geom& g = e->geom[m];
    AC_CUDA_CHECK(ac_launch_reduce(g, fp, lo, kind, e->precision, map, r.reduce_op, e->red,
                                   e->stream, &e->launches));
    AC_CUDA_CHECK(cudaMemcpyAsync(e->host_result, e->red.result, sizeof(double),
                                  cudaMemcpyDeviceToHost, e->stream));
    AC_CUDA_CHECK(cudaStreamSynchronize(e->stream));
    double v = *e->host_result;
    if (r.post_processing_op == AC_RMS)
        v = sqrt(v / ((double)g.nx * (double)g.ny * (double)g.nz));
    *result = v;
    return AC_SUCCESS;
}

} // namespace

extern "C" AcResult
acEnsembleCreate(const int device_id, const int n, const AcMeshInfo* member_infos, Ensemble* out)
{
    if (!out)
        return AC_FAILURE;
    *out = NULL;
    if (n < 1 || !member_infos)
        return AC_FAILURE;
    int count = 0;
    AC_CUDA_CHECK(cudaGetDeviceCount(&count));
    if (device_id < 0 || device_id >= count)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(device_id));

    Ensemble e = new ensemble_s();
    e->id      = device_id;
    e->n       = n;
#define ENS_CHECK(call)                                                                       \
    do {                                                                                      \
        const cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                              \
            fprintf(stderr, "astaroth_b200: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
            destroy(e);                                                                       \
            return AC_FAILURE;                                                                \
        }                                                                                     \
    } while (0)
    for (int m = 0; m < n; ++m) {
        AcMeshInfo info = member_infos[m];
        if (acHostUpdateParams(&info) != AC_SUCCESS) {
            fprintf(stderr, "astaroth_b200: ensemble member %d: invalid AcMeshInfo\n", m);
            destroy(e);
            return AC_FAILURE;
        }
        const int p = info.int_params[AC_precision];
        if ((p != 0 && p != 1) || (m > 0 && p != e->precision)) {
            fprintf(stderr, "astaroth_b200: ensemble members need one precision (0 or 1)\n");
            destroy(e);
            return AC_FAILURE;
        }
        if (info.int_params[AC_upwind] || info.int_params[AC_lforcing]) {
            fprintf(stderr, "astaroth_b200: ensemble members without AC_upwind and "
                            "AC_lforcing only\n");
            destroy(e);
            return AC_FAILURE;
        }
        e->precision = p;
        e->info.push_back(info);
        e->geom.push_back(ac_make_geom(info, p));
        StencilCoef sc;
        PhysConst pc;
        ac_make_stencil(info, &sc);
        ac_make_phys(info, &pc);
        e->sc.push_back(sc);
        e->pc.push_back(pc);
        e->dts.push_back(0.0);
    }
    size_t total = 0, max_mesh = 0;
    int max_blocks = 1;
    e->cells       = 0;
    for (int m = 0; m < n; ++m) {
        const Geom& g = e->geom[m];
        e->offset.push_back(total);
        total += member_bytes(g, e->precision);
        max_mesh   = std::max(max_mesh, (size_t)g.mx * g.my * g.mz);
        max_blocks = std::max(max_blocks, ac_reduce_blocks(g));
        e->cells += (long long)g.nx * g.ny * g.nz;
    }
    ENS_CHECK(cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, device_id));
    ENS_CHECK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    ENS_CHECK(cudaMalloc((void**)&e->pool, total));
    /* zero-filled in and out, as a Device */
    ENS_CHECK(cudaMemsetAsync(e->pool, 0, total, e->stream));

    const size_t rec = e->precision == 0 ? sizeof(EnsMember<double>) : sizeof(EnsMember<float>);
    e->hmem          = calloc(n, rec);
    if (!e->hmem) {
        destroy(e);
        return AC_FAILURE;
    }
    if (e->precision == 0)
        fill_members<double, false>(e);
    else
        fill_members<float, true>(e);
    ENS_CHECK(cudaMalloc(&e->dmem, n * rec));
    ENS_CHECK(cudaMemcpyAsync(e->dmem, e->hmem, n * rec, cudaMemcpyHostToDevice, e->stream));
    ENS_CHECK(cudaMalloc((void**)&e->d_dts, n * sizeof(double)));
    ENS_CHECK(cudaMemsetAsync(e->d_dts, 0, n * sizeof(double), e->stream));

    std::vector<long long> prefix(n + 1, 0);
    for (int m = 0; m < n; ++m) {
        long long a, b;
        prefix[m + 1] = prefix[m] + halo_count(e->geom[m], &a, &b);
    }
    e->halo_total = prefix[n];
    ENS_CHECK(cudaMalloc((void**)&e->halo_prefix, (n + 1) * sizeof(long long)));
    ENS_CHECK(cudaMemcpyAsync(e->halo_prefix, prefix.data(), (n + 1) * sizeof(long long),
                              cudaMemcpyHostToDevice, e->stream));
    if (e->precision == 1)
        ENS_CHECK(cudaMalloc((void**)&e->staging, max_mesh * sizeof(double)));

    e->red.max_blocks   = max_blocks;
    const size_t rbytes = (2 * (size_t)max_blocks + 2) * sizeof(double) + 64;
    ENS_CHECK(cudaMalloc((void**)&e->red.partials, rbytes));
    ENS_CHECK(cudaMemsetAsync(e->red.partials, 0, rbytes, e->stream));
    e->red.result  = e->red.partials + 2 * (size_t)max_blocks;
    e->red.counter = (unsigned int*)(e->red.result + 2);
    e->red.nonfinite = nullptr;
    ENS_CHECK(cudaMallocHost((void**)&e->host_result, sizeof(double)));
    ENS_CHECK(cudaStreamSynchronize(e->stream));
    const AcEnsembleTiles def = {32, 4, 8, 0, 0};
    ENS_CHECK(build_items(e, def));
    /* mode 1: tensor maps of both buffer blocks of every member, branch streams */
    ENS_CHECK(cudaMalloc((void**)&e->err, sizeof(int)));
    ENS_CHECK(cudaMemset(e->err, 0, sizeof(int)));
    e->tmaps.resize(2 * (size_t)n);
    e->tiled.assign(n, 1);
    for (int m = 0; m < n; ++m)
        for (int p = 0; p < 2; ++p) {
            void* base = e->precision == 0 ? (void*)members<double>(e)[m].f[p].in[0]
                                           : (void*)members<float>(e)[m].f[p].in[0];
            if (!ac_make_tensor_map(&e->tmaps[2 * m + p], base, e->geom[m], e->precision))
                e->tiled[m] = 0;
        }
    ENS_CHECK(ac_solve_tiled_init(e->precision));
    const int nb = std::min(n, 16);
    e->branches.assign(nb, nullptr);
    e->joins.assign(nb, nullptr);
    for (int b = 0; b < nb; ++b) {
        ENS_CHECK(cudaStreamCreateWithFlags(&e->branches[b], cudaStreamNonBlocking));
        ENS_CHECK(cudaEventCreateWithFlags(&e->joins[b], cudaEventDisableTiming));
    }
    ENS_CHECK(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
#undef ENS_CHECK
    *out = e;
    return AC_SUCCESS;
}

extern "C" AcResult
acEnsembleDestroy(Ensemble* e)
{
    if (!e)
        return AC_FAILURE;
    destroy(*e);
    *e = NULL;
    return AC_SUCCESS;
}

extern "C" AcResult
acEnsembleLoadMember(const Ensemble e, const int m, const AcMesh host)
{
    if (!member_ok(e, m))
        return AC_FAILURE;
    if (!host_matches(e, m, host.info)) {
        fprintf(stderr, "astaroth_b200: host mesh dimensions differ from ensemble member %d\n", m);
        return AC_FAILURE;
    }
    for (int q = 0; q < AC_NF; ++q)
        if (!host.vertex_buffer[q])
            return AC_NOT_ALLOCATED;
    AC_CUDA_CHECK(cudaSetDevice(e->id));
    const Geom& g  = e->geom[m];
    const size_t n = (size_t)g.mx * g.my * g.mz;
    for (int q = 0; q < AC_NF; ++q) {
        void* hi;
        float* lo;
        member_arrays(e, m, q, &hi, &lo);
        if (e->precision == 0) {
            AC_CUDA_CHECK(cudaMemcpyAsync(hi, host.vertex_buffer[q], n * sizeof(double),
                                          cudaMemcpyHostToDevice, e->stream));
        }
        else {
            AC_CUDA_CHECK(cudaMemcpyAsync(e->staging, host.vertex_buffer[q], n * sizeof(double),
                                          cudaMemcpyHostToDevice, e->stream));
            AC_CUDA_CHECK(ac_launch_split(g, e->staging, (float*)hi, lo, e->stream, &e->launches));
        }
    }
    AC_CUDA_CHECK(cudaStreamSynchronize(e->stream));
    return AC_SUCCESS;
}

extern "C" AcResult
acEnsembleStoreMember(const Ensemble e, const int m, AcMesh* host)
{
    if (!member_ok(e, m) || !host)
        return AC_FAILURE;
    if (!host_matches(e, m, host->info)) {
        fprintf(stderr, "astaroth_b200: host mesh dimensions differ from ensemble member %d\n", m);
        return AC_FAILURE;
    }
    for (int q = 0; q < AC_NF; ++q)
        if (!host->vertex_buffer[q])
            return AC_NOT_ALLOCATED;
    AC_CUDA_CHECK(cudaSetDevice(e->id));
    const Geom& g  = e->geom[m];
    const size_t n = (size_t)g.mx * g.my * g.mz;
    for (int q = 0; q < AC_NF; ++q) {
        void* hi;
        float* lo;
        member_arrays(e, m, q, &hi, &lo);
        if (e->precision == 0) {
            AC_CUDA_CHECK(cudaMemcpyAsync(host->vertex_buffer[q], hi, n * sizeof(double),
                                          cudaMemcpyDeviceToHost, e->stream));
        }
        else {
            AC_CUDA_CHECK(ac_launch_join(g, (const float*)hi, lo, e->staging, e->stream,
                                         &e->launches));
            AC_CUDA_CHECK(cudaMemcpyAsync(host->vertex_buffer[q], e->staging, n * sizeof(double),
                                          cudaMemcpyDeviceToHost, e->stream));
            /* the staging field is reused by the next field */
            AC_CUDA_CHECK(cudaStreamSynchronize(e->stream));
        }
    }
    AC_CUDA_CHECK(cudaStreamSynchronize(e->stream));
    return AC_SUCCESS;
}

extern "C" AcResult
acEnsembleSetTimesteps(const Ensemble e, const AcReal* dts)
{
    if (!e || !dts)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(e->id));
    for (int m = 0; m < e->n; ++m)
        e->dts[m] = dts[m];
    /* pageable source: the copy is complete when the call returns */
    AC_CUDA_CHECK(cudaMemcpyAsync(e->d_dts, e->dts.data(), e->n * sizeof(double),
                                  cudaMemcpyHostToDevice, e->stream));
    AC_CUDA_CHECK(cudaStreamSynchronize(e->stream));
    invalidate(e); /* mode 1 launches take dt as a parameter */
    return AC_SUCCESS;
}

extern "C" AcResult
acEnsembleIntegrateStep(const Ensemble e)
{
    if (!e)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(e->id));
    const int p = e->parity;
    /* capture the graphs of both buffer parities at the first step, so later
     * steps (which alternate parities) never capture */
    for (int c = 0; c < 2; ++c) {
        const int pc = p ^ c;
        if (e->graph_valid[pc])
            continue;
        e->parity = pc;
        cudaGraph_t graph;
        AC_CUDA_CHECK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        const cudaError_t rec = record_step(e, NULL);
        const cudaError_t end = cudaStreamEndCapture(e->stream, &graph);
        e->parity             = p; /* undo the capture's swaps */
        AC_CUDA_CHECK(rec);
        AC_CUDA_CHECK(end);
        const cudaError_t inst = cudaGraphInstantiate(&e->graph[pc], graph, 0);
        cudaGraphDestroy(graph);
        AC_CUDA_CHECK(inst);
        e->graph_valid[pc] = 1;
    }
    AC_CUDA_CHECK(cudaGraphLaunch(e->graph[p], e->stream));
    e->launches += e->tiles.mode == 1 ? 6ull * e->n : 6ull; /* halo + solve, 3 substeps */
    e->parity ^= 1; /* three swaps */
    return AC_SUCCESS;
}

extern "C" AcResult
acEnsembleIntegrateStepSequential(const Ensemble e)
{
    if (!e)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(e->id));
    const cudaError_t err = e->precision == 0 ? sequential_step<double, false>(e)
                                              : sequential_step<float, true>(e);
    AC_CUDA_CHECK(err);
    return AC_SUCCESS;
}

extern "C" AcResult
acEnsembleSetTiles(const Ensemble e, const AcEnsembleTiles t)
{
    if (!e || !tiles_ok(t)) {
        fprintf(stderr, "astaroth_b200: invalid ensemble tiles (tx*ty a multiple of 32, "
                        "at most 256; zb >= 1)\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(e->id));
    AC_CUDA_CHECK(build_items(e, t));
    return AC_SUCCESS;
}

extern "C" AcResult
acEnsembleGetTiles(const Ensemble e, AcEnsembleTiles* t)
{
    if (!e || !t)
        return AC_FAILURE;
    *t = e->tiles;
    return AC_SUCCESS;
}

extern "C" AcResult
acEnsembleAutotune(const Ensemble e, AcEnsembleTiles* best, double* best_ms)
{
    if (!e)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(e->id));
    static const int shapes[][2] = {{32, 2}, {32, 4}, {32, 8}, {16, 4}, {16, 8},
                                    {16, 16}, {8, 8}, {8, 16}, {64, 2}, {64, 4}};
    static const int zbs[]       = {4, 8, 16, 32};
    std::vector<AcEnsembleTiles> cand;
    for (const auto& s : shapes)
        for (const int zb : zbs)
            cand.push_back({s[0], s[1], zb, 0, 0});
    cudaEvent_t t0, t1;
    AC_CUDA_CHECK(cudaEventCreate(&t0));
    AC_CUDA_CHECK(cudaEventCreate(&t1));
    AcEnsembleTiles win = e->tiles;
    double win_ms       = 1e300;
    /* Substep 0 reads the in-buffers and writes the out-buffers only, which the
     * next step overwrites before reading: timing it leaves the state as it was. */
    auto time_tiles = [&](const AcEnsembleTiles t, double* ms) -> cudaError_t {
        cudaError_t err = build_items(e, t);
        if (err != cudaSuccess)
            return err;
        const int reps = 5;
        err            = launch_solve(e, 0, &e->launches);
        if (err != cudaSuccess)
            return err;
        cudaEventRecord(t0, e->stream);
        for (int r = 0; r < reps && err == cudaSuccess; ++r)
            err = launch_solve(e, 0, &e->launches);
        cudaEventRecord(t1, e->stream);
        if (err != cudaSuccess)
            return err;
        err = cudaEventSynchronize(t1);
        if (err != cudaSuccess)
            return err;
        float f = 0;
        cudaEventElapsedTime(&f, t0, t1);
        *ms = f / reps;
        return cudaSuccess;
    };
    cudaError_t err = cudaSuccess;
    for (const AcEnsembleTiles& t : cand) {
        double ms = 0;
        err       = time_tiles(t, &ms);
        if (err != cudaSuccess)
            break;
        if (ms < win_ms) {
            win_ms = ms;
            win    = t;
        }
    }
    /* then fewer resident blocks per SM for the winning shape */
    for (int bps = 1; bps <= 4 && err == cudaSuccess; ++bps) {
        AcEnsembleTiles t = win;
        t.blocks_per_sm   = bps;
        double ms         = 0;
        err               = time_tiles(t, &ms);
        if (err == cudaSuccess && ms < win_ms * 0.98) {
            win_ms = ms;
            win    = t;
        }
    }
    /* then the two modes on the solve of substep 0 (no halo fill, so the state
     * is left as it was), each replayed from a captured graph */
    auto time_graph = [&](const int mode, double* ms) -> cudaError_t {
        cudaGraph_t graph;
        cudaGraphExec_t exec;
        cudaError_t rec = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
        if (rec != cudaSuccess)
            return rec;
        if (mode == 0)
            rec = launch_solve(e, 0, NULL);
        else
            rec = e->precision == 0 ? record_members<double, false>(e, 0, 1, NULL, false)
                                    : record_members<float, true>(e, 0, 1, NULL, false);
        const cudaError_t end = cudaStreamEndCapture(e->stream, &graph);
        if (rec != cudaSuccess)
            return rec;
        if (end != cudaSuccess)
            return end;
        cudaError_t r = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (r != cudaSuccess)
            return r;
        const int reps = 5;
        r              = cudaGraphLaunch(exec, e->stream);
        cudaEventRecord(t0, e->stream);
        for (int k = 0; k < reps && r == cudaSuccess; ++k)
            r = cudaGraphLaunch(exec, e->stream);
        cudaEventRecord(t1, e->stream);
        if (r == cudaSuccess)
            r = cudaEventSynchronize(t1);
        float f = 0;
        cudaEventElapsedTime(&f, t0, t1);
        *ms = f / reps;
        cudaGraphExecDestroy(exec);
        return r;
    };
    if (err == cudaSuccess)
        err = build_items(e, win);
    double ms0 = 0, ms1 = 1e300;
    if (err == cudaSuccess)
        err = time_graph(0, &ms0);
    if (err == cudaSuccess)
        err = time_graph(1, &ms1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    AC_CUDA_CHECK(err);
    win.mode = ms1 < ms0 ? 1 : 0;
    win_ms   = ms1 < ms0 ? ms1 : ms0;
    AC_CUDA_CHECK(build_items(e, win));
    if (best)
        *best = win;
    if (best_ms)
        *best_ms = win_ms;
    return AC_SUCCESS;
}

extern "C" AcResult
acEnsembleReduceScal(const Ensemble e, const int m, const AcReduction r,
                     const VertexBufferHandle h, AcReal* result)
{
    return reduce_member(e, m, r, 1, &h, result);
}

extern "C" AcResult
acEnsembleReduceVec(const Ensemble e, const int m, const AcReduction r,
                    const VertexBufferHandle a, const VertexBufferHandle b,
                    const VertexBufferHandle c, AcReal* result)
{
    const VertexBufferHandle h[3] = {a, b, c};
    return reduce_member(e, m, r, 3, h, result);
}

extern "C" AcResult
acEnsembleSynchronize(const Ensemble e)
{
    if (!e)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(e->id));
    AC_CUDA_CHECK(cudaStreamSynchronize(e->stream));
    return AC_SUCCESS;
}

extern "C" void*
acEnsembleGetStreamHandle(const Ensemble e)
{
    return e ? (void*)e->stream : NULL;
}

extern "C" unsigned long long
acEnsembleGetLaunchCount(const Ensemble e)
{
    return e ? e->launches : 0ULL;
}

extern "C" long long
acEnsembleCellCount(const Ensemble e)
{
    return e ? e->cells : 0LL;
}
