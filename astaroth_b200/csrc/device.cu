/*
 * The device object and the acDevice* C ABI (include/astaroth_b200.h).
 *
 * Reference: src/core/device.cc (struct device_s :63-74, acDeviceCreate
 * :509-594, acDeviceDestroy :602-630, swaps :635-663, load/store :666-854,
 * acDeviceIntegrateSubstep :941-997, boundconds :999-1017, reductions
 * :1370-1481) and the buffer allocation of acVBACreate
 * (acc-runtime/api/vba.cc:313-488).
 *
 * B200 design: the 8 fields of each buffer are one contiguous allocation
 * (SoA, x fastest, halos included, exactly the host layout so load/store are
 * single copies); every API call returns an AcResult instead of aborting;
 * kernel parameters travel by value (no __constant__ state), so several
 * devices and CUDA graphs coexist without global singletons.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <errno.h>
#include <sys/stat.h>

#include "internal.h"

static const char* kVersion = "astaroth_b200 0.1 (sm_100a)";

/* ------------------------------------------------------------------------- */

Geom
ac_make_geom(const AcMeshInfo& info, const int precision)
{
    Geom g;
    const int3 n = info.int3_params[AC_nlocal];
    g.nx         = n.x;
    g.ny         = n.y;
    g.nz         = n.z;
    g.mx         = n.x + 2 * NGHOST;
    g.my         = n.y + 2 * NGHOST;
    g.mz         = n.z + 2 * NGHOST;
    g.px         = precision == 0 ? g.mx : (g.mx + 3) / 4 * 4;
    g.pxy        = (long long)g.px * g.my;
    g.cells      = g.pxy * g.mz;
    return g;
}

/* ---- buffer access ---- */

static size_t
elem_size(const Device d)
{
    return d->precision == 0 ? sizeof(double) : sizeof(float);
}

static double*
arr64(const Device d, const int b, const int q)
{
    return (double*)d->hi[b] + (size_t)q * d->geom.cells;
}

static float*
arr_hi(const Device d, const int b, const int q)
{
    return (float*)d->hi[b] + (size_t)q * d->geom.cells;
}

static float*
arr_lo(const Device d, const int b, const int q)
{
    return d->lo[b] + (size_t)q * d->geom.cells;
}

static Fields64
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

static Fields32
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
static int
in_block_index(const Device d)
{
    for (int q = 1; q < AC_NF; ++q)
        if (d->in_idx[q] != d->in_idx[0])
            return -1;
    return d->in_idx[0];
}

void
ac_make_stencil(const AcMeshInfo& info, StencilCoef* sc)
{
    const double c[3] = {3.0 / 4.0, -3.0 / 20.0, 1.0 / 60.0};
    const double d[4] = {-49.0 / 18.0, 3.0 / 2.0, -3.0 / 20.0, 1.0 / 90.0};
    const double e[3] = {270.0 / 720.0, -27.0 / 720.0, 2.0 / 720.0};
    const AcReal3 inv = info.real3_params[AC_inv_ds];
    const double iv[3] = {inv.x, inv.y, inv.z};
    /* upwinding: (1/60) (-20 f0 + 15 s1 - 6 s2 + s3) / ds, modelsolver.cc:424-492 */
    const double u[4] = {-20.0 / 60.0, 15.0 / 60.0, -6.0 / 60.0, 1.0 / 60.0};
    for (int a = 0; a < 3; ++a) {
        for (int k = 0; k < 3; ++k)
            sc->d1[a][k] = c[k] * iv[a];
        for (int k = 0; k < 4; ++k) {
            sc->d2[a][k] = d[k] * iv[a] * iv[a];
            sc->up[a][k] = u[k] * iv[a];
        }
    }
    const int pa[3] = {0, 0, 1}, pb[3] = {1, 2, 2};
    for (int m = 0; m < 3; ++m)
        for (int k = 0; k < 3; ++k)
            sc->mix[m][k] = e[k] * iv[pa[m]] * iv[pb[m]];
}

void
ac_make_phys(const AcMeshInfo& info, PhysConst* pc)
{
    const double* r  = info.real_params;
    pc->nu           = r[AC_nu_visc];
    pc->eta          = r[AC_eta];
    pc->zeta         = r[AC_zeta];
    pc->inv_mu0      = 1.0 / r[AC_mu0];
    pc->eta_mu0      = r[AC_eta] * r[AC_mu0];
    pc->cs2_sound    = r[AC_cs_sound] * r[AC_cs_sound];
    pc->gamma        = r[AC_gamma];
    pc->gamma_m1     = r[AC_gamma] - 1.0;
    pc->inv_cp       = 1.0 / r[AC_cp_sound];
    pc->gamma_inv_cp = r[AC_gamma] / r[AC_cp_sound];
    pc->lnrho0       = r[AC_lnrho0];
    pc->inv_exp_lnT0 = exp(-r[AC_lnT0]);
    pc->K            = r[AC_K_heatcond];
    pc->upwind       = info.int_params[AC_upwind] != 0;
    pc->forcing      = 0;
    for (int a = 0; a < 3; ++a)
        pc->f_k[a] = pc->f_re[a] = pc->f_im[a] = 0.0;
    pc->f_cos_phase = 1.0;
    pc->f_sin_phase = 0.0;
    pc->f_scale     = 0.0;
}

/* The forcing of a substep-2 launch (mhdsolver.ac:531-541): active when
 * AC_lforcing is set and AC_current_time > AC_switch_forcing. */
static void
forcing_for_launch(const AcMeshInfo& info, const double dt, PhysConst* pc)
{
    const double* r = info.real_params;
    if (!info.int_params[AC_lforcing] || !(r[AC_current_time] > r[AC_switch_forcing]))
        return;
    const double two_pi = 6.283185307179586476925286766559;
    const int3 ng       = info.int3_params[AC_ngrid];
    const double k[3]   = {r[AC_k_forcex], r[AC_k_forcey], r[AC_k_forcez]};
    const int n[3]      = {ng.x, ng.y, ng.z};
    const double fre[3] = {r[AC_ff_hel_rex], r[AC_ff_hel_rey], r[AC_ff_hel_rez]};
    const double fim[3] = {r[AC_ff_hel_imx], r[AC_ff_hel_imy], r[AC_ff_hel_imz]};
    for (int a = 0; a < 3; ++a) {
        pc->f_k[a]  = k[a] * two_pi / n[a];
        pc->f_re[a] = fre[a];
        pc->f_im[a] = fim[a];
    }
    /* the kernel counts cells from this device's first interior cell; a slab
     * of a larger grid starts at AC_multigpu_offset, which shifts the phase */
    const int3 off    = info.int3_params[AC_multigpu_offset];
    const double ph   = r[AC_forcing_phase] + pc->f_k[0] * off.x + pc->f_k[1] * off.y +
                      pc->f_k[2] * off.z;
    pc->f_cos_phase = cos(ph);
    pc->f_sin_phase = sin(ph);
    /* N = cs magnitude sqrt(kaver cs); the force is sqrt(dt) N f */
    const double cs = sqrt(r[AC_cs_sound] * r[AC_cs_sound]);
    pc->f_scale     = sqrt(dt) * cs * r[AC_forcing_magnitude] * sqrt(r[AC_kaver] * cs);
    pc->forcing     = 1;
}

static bool
stream_ok(const Stream s)
{
    return (int)s >= 0 && (int)s < NUM_STREAMS;
}

/* The B arrays of AC_lbfield, allocated (zeroed) when the flag is first set;
 * never during a stream capture (every caller is outside one). */
static cudaError_t
ensure_bfield(Device d)
{
    if (!d->config.int_params[AC_lbfield] || d->bfield)
        return cudaSuccess;
    const size_t bytes = 3 * (size_t)d->geom.mx * d->geom.my * d->geom.mz * sizeof(double);
    cudaError_t e      = cudaMalloc((void**)&d->bfield, bytes);
    if (e != cudaSuccess)
        return e;
    return cudaMemset(d->bfield, 0, bytes);
}

static void
invalidate_tape_graph(Device d)
{
    for (int b = 0; b < 2; ++b) {
        if (d->tape_valid[b])
            cudaGraphExecDestroy(d->tape_exec[b]);
        d->tape_valid[b] = 0;
    }
}

static void
invalidate_graphs(Device d)
{
    invalidate_tape_graph(d);
    for (int s = 0; s < NUM_STREAMS; ++s)
        for (int p = 0; p < 2; ++p) {
            if (d->graphs[s][p].valid)
                cudaGraphExecDestroy(d->graphs[s][p].exec);
            d->graphs[s][p].valid = 0;
        }
}

static void
release(Device d)
{
    if (!d)
        return;
    cudaSetDevice(d->id);
    cudaDeviceSynchronize();
    invalidate_graphs(d);
    for (int b = 0; b < 2; ++b) {
        cudaFree(d->hi[b]);
        cudaFree(d->lo[b]);
    }
    cudaFree(d->staging);
    cudaFree(d->red.partials);
    cudaFree(d->adj_lf);
    cudaFree(d->adj_lw);
    cudaFree(d->adj_mu);
    cudaFree(d->adj_pgrad);
    cudaFree(d->adj_tape);
    cudaFree(d->bfield);
    cudaFree(d->stage);
    if (d->stage_loaded)
        cudaEventDestroy(d->stage_loaded);
    if (d->stage_read)
        cudaEventDestroy(d->stage_read);
    cudaFreeHost(d->host_result);
    for (int s = 0; s < NUM_STREAMS; ++s)
        if (d->streams[s])
            cudaStreamDestroy(d->streams[s]);
    free(d);
}

/* ------------------------------------------------------------------------- */

extern "C" const char*
acB200Version(void)
{
    return kVersion;
}

extern "C" AcResult
acDeviceCreate(const int id, const AcMeshInfo device_config, Device* device_handle)
{
    if (!device_handle)
        return AC_FAILURE;
    *device_handle = NULL;
    int count      = 0;
    AC_CUDA_CHECK(cudaGetDeviceCount(&count));
    if (id < 0 || id >= count) {
        fprintf(stderr, "astaroth_b200: device id %d out of range (%d devices)\n", id, count);
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(id));

    AcMeshInfo info = device_config;
    if (acHostUpdateParams(&info) != AC_SUCCESS) {
        fprintf(stderr, "astaroth_b200: invalid AcMeshInfo (AC_ngrid and AC_ds must be > 0)\n");
        return AC_FAILURE;
    }
    const int precision = info.int_params[AC_precision];
    if (precision != 0 && precision != 1) {
        fprintf(stderr, "astaroth_b200: AC_precision=%d is not supported (0 FP64, 1 FP32 "
                        "compensated)\n",
                precision);
        return AC_FAILURE;
    }

    /* CUtensorMap members need 64-byte alignment */
    const size_t dbytes = (sizeof(device_s) + 63) / 64 * 64;
    device_s* d         = (device_s*)aligned_alloc(64, dbytes);
    if (!d)
        return AC_FAILURE;
    memset(d, 0, dbytes);
    d->id        = id;
    d->config    = info;
    d->geom      = ac_make_geom(info, precision);
    d->precision = precision;
    d->solve_variant = info.int_params[AC_debug_plain_kernel] ? 0 : 1;

#define CREATE_CHECK(call)                                                                    \
    do {                                                                                      \
        const cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                              \
            fprintf(stderr, "astaroth_b200: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
            release(d);                                                                       \
            return AC_FAILURE;                                                                \
        }                                                                                     \
    } while (0)

    for (int s = 0; s < NUM_STREAMS; ++s)
        CREATE_CHECK(cudaStreamCreateWithFlags(&d->streams[s], cudaStreamNonBlocking));

    const size_t bytes = (size_t)AC_NF * (size_t)d->geom.cells * elem_size(d);
    for (int b = 0; b < 2; ++b) {
        CREATE_CHECK(cudaMalloc(&d->hi[b], bytes));
        /* zero-filled in and out, as acVBAReset (acc-runtime/api/vba.cc:274-307) */
        CREATE_CHECK(cudaMemsetAsync(d->hi[b], 0, bytes, d->streams[0]));
        if (precision == 1) {
            CREATE_CHECK(cudaMalloc((void**)&d->lo[b], bytes));
            CREATE_CHECK(cudaMemsetAsync(d->lo[b], 0, bytes, d->streams[0]));
        }
    }
    if (precision == 1)
        CREATE_CHECK(cudaMalloc((void**)&d->staging, (size_t)d->geom.mx * d->geom.my *
                                                          d->geom.mz * sizeof(double)));
    for (int q = 0; q < AC_NF; ++q)
        d->in_idx[q] = 0;

    /* small scratch block: [partials 2*blocks][result 2][counter, err] */
    const int blocks    = ac_reduce_blocks(d->geom);
    d->red.max_blocks   = blocks;
    const size_t rbytes = (2 * (size_t)blocks + 2) * sizeof(double) + 128;
    CREATE_CHECK(cudaMalloc((void**)&d->red.partials, rbytes));
    CREATE_CHECK(cudaMemsetAsync(d->red.partials, 0, rbytes, d->streams[0]));
    d->red.result  = d->red.partials + 2 * (size_t)blocks;
    d->red.counter = (unsigned int*)(d->red.result + 2);
    d->err_flag    = (int*)(d->red.counter + 4);
    d->cfl         = (unsigned long long*)(d->red.counter + 8);
    d->tmap_ok     = ac_make_tensor_map(&d->tmap[0], d->hi[0], d->geom, precision) &&
                 ac_make_tensor_map(&d->tmap[1], d->hi[1], d->geom, precision);
    if (d->tmap_ok)
        CREATE_CHECK(ac_solve_tiled_init(precision));
    CREATE_CHECK(cudaMallocHost((void**)&d->host_result, sizeof(double)));
    CREATE_CHECK(ensure_bfield(d));
    CREATE_CHECK(cudaStreamSynchronize(d->streams[0]));
#undef CREATE_CHECK

    *device_handle = d;
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceDestroy(Device* device_handle)
{
    if (!device_handle)
        return AC_FAILURE;
    if (!*device_handle)
        return AC_SUCCESS;
    release(*device_handle);
    *device_handle = NULL;
    return AC_SUCCESS;
}

extern "C" AcResult
acDevicePrintInfo(const Device d)
{
    if (!d)
        return AC_FAILURE;
    cudaDeviceProp p;
    AC_CUDA_CHECK(cudaGetDeviceProperties(&p, d->id));
    printf("astaroth_b200 device %d: %s, sm_%d%d, %d SMs, %.1f GiB\n", d->id, p.name, p.major,
           p.minor, p.multiProcessorCount, (double)p.totalGlobalMem / (1 << 30));
    printf("  mesh: n = (%d, %d, %d), m = (%d, %d, %d), precision %s\n", d->geom.nx, d->geom.ny,
           d->geom.nz, d->geom.mx, d->geom.my, d->geom.mz, d->precision ? "fp32-comp" : "fp64");
    return AC_SUCCESS;
}

/* Reads and clears the device error word (set by a kernel whose bounded wait
 * on an mbarrier gave up); nonzero means the last results are invalid. */
static AcResult
check_device_error(const Device d, cudaStream_t st)
{
    int err = 0;
    AC_CUDA_CHECK(cudaMemcpyAsync(&err, d->err_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    AC_CUDA_CHECK(cudaStreamSynchronize(st));
    if (err) {
        fprintf(stderr, "astaroth_b200: a kernel timed out waiting for its TMA loads\n");
        AC_CUDA_CHECK(cudaMemsetAsync(d->err_flag, 0, sizeof(int), st));
        AC_CUDA_CHECK(cudaStreamSynchronize(st));
        return AC_FAILURE;
    }
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceSynchronizeStream(const Device d, const Stream stream)
{
    if (!d)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    if (stream == STREAM_ALL) {
        for (int s = 0; s < NUM_STREAMS; ++s)
            AC_CUDA_CHECK(cudaStreamSynchronize(d->streams[s]));
        return check_device_error(d, d->streams[0]);
    }
    if (!stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaStreamSynchronize(d->streams[stream]));
    return check_device_error(d, d->streams[stream]);
}

extern "C" AcResult
acDeviceSwapBuffer(const Device d, const VertexBufferHandle h)
{
    if (!d || (int)h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    d->in_idx[h] = 1 - d->in_idx[h];
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceSwapBuffers(const Device d)
{
    if (!d)
        return AC_FAILURE;
    for (int q = 0; q < AC_NF; ++q)
        acDeviceSwapBuffer(d, (VertexBufferHandle)q);
    return AC_SUCCESS;
}

/* ---- uniforms / config ---- */

static_assert(sizeof(AcMeshInfo) == sizeof(int) * NUM_INT_PARAMS + sizeof(int3) * NUM_INT3_PARAMS +
                                        sizeof(AcReal) * NUM_REAL_PARAMS +
                                        sizeof(AcReal3) * NUM_REAL3_PARAMS,
              "AcMeshInfo has no padding (refresh_config compares it bytewise)");

static AcResult
refresh_config(Device d, const AcMeshInfo& info)
{
    AcMeshInfo next = info;
    if (acHostUpdateParams(&next) != AC_SUCCESS)
        return AC_FAILURE;
    const Geom g = ac_make_geom(next, d->precision);
    if (g.nx != d->geom.nx || g.ny != d->geom.ny || g.nz != d->geom.nz) {
        fprintf(stderr, "astaroth_b200: mesh dimensions cannot change after acDeviceCreate\n");
        return AC_FAILURE;
    }
    if (next.int_params[AC_precision] != d->precision) {
        fprintf(stderr, "astaroth_b200: AC_precision cannot change after acDeviceCreate\n");
        return AC_FAILURE;
    }
    /* the same parameters again (AcMeshInfo has no padding): the captured
     * graphs stay valid */
    if (memcmp(&next, &d->config, sizeof(AcMeshInfo)) == 0)
        return AC_SUCCESS;
    d->config = next;
    invalidate_graphs(d);
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    AC_CUDA_CHECK(ensure_bfield(d));
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceLoadScalarUniform(const Device d, const Stream stream, const AcRealParam param,
                          const AcReal value)
{
    (void)stream;
    if (!d || (int)param < 0 || param >= NUM_REAL_PARAMS)
        return AC_FAILURE;
    AcMeshInfo info         = d->config;
    info.real_params[param] = value;
    return refresh_config(d, info);
}

extern "C" AcResult
acDeviceLoadVectorUniform(const Device d, const Stream stream, const AcReal3Param param,
                          const AcReal3 value)
{
    (void)stream;
    if (!d || (int)param < 0 || param >= NUM_REAL3_PARAMS)
        return AC_FAILURE;
    AcMeshInfo info          = d->config;
    info.real3_params[param] = value;
    return refresh_config(d, info);
}

/* include/astaroth_device.h device_load_uniform_decl.h: an int3 parameter.
 * The mesh dimensions and offsets cannot change after acDeviceCreate, so
 * this serves the parameters derived from them being loaded unchanged, as
 * the reference's grid layer does. */
extern "C" AcResult
acDeviceLoadInt3Uniform(const Device d, const Stream stream, const AcInt3Param param,
                        const int3 value)
{
    (void)stream;
    if (!d || (int)param < 0 || param >= NUM_INT3_PARAMS)
        return AC_FAILURE;
    AcMeshInfo info          = d->config;
    info.int3_params[param] = value;
    return refresh_config(d, info);
}

extern "C" AcResult
acDeviceLoadIntUniform(const Device d, const Stream stream, const AcIntParam param,
                       const int value)
{
    (void)stream;
    if (!d || (int)param < 0 || param >= NUM_INT_PARAMS)
        return AC_FAILURE;
    AcMeshInfo info        = d->config;
    info.int_params[param] = value;
    const AcResult r       = refresh_config(d, info);
    if (r == AC_SUCCESS)
        d->solve_variant = d->config.int_params[AC_debug_plain_kernel] ? 0 : 1;
    return r;
}

/* include/astaroth_device.h:61 and device_store_uniform_decl.h. */
extern "C" AcResult
acDeviceStoreVectorUniform(const Device d, const Stream stream, const AcReal3Param param,
                           AcReal3* value)
{
    (void)stream;
    if (!d || !value || (int)param < 0 || param >= NUM_REAL3_PARAMS)
        return AC_FAILURE;
    *value = d->config.real3_params[param];
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceStoreIntUniform(const Device d, const Stream stream, const AcIntParam param, int* value)
{
    (void)stream;
    if (!d || !value || (int)param < 0 || param >= NUM_INT_PARAMS)
        return AC_FAILURE;
    *value = d->config.int_params[param];
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceStoreInt3Uniform(const Device d, const Stream stream, const AcInt3Param param,
                         int3* value)
{
    (void)stream;
    if (!d || !value || (int)param < 0 || param >= NUM_INT3_PARAMS)
        return AC_FAILURE;
    *value = d->config.int3_params[param];
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceStoreScalarUniform(const Device d, const Stream stream, const AcRealParam param,
                           AcReal* value)
{
    (void)stream;
    if (!d || !value || (int)param < 0 || param >= NUM_REAL_PARAMS)
        return AC_FAILURE;
    *value = d->config.real_params[param];
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceLoadMeshInfo(const Device d, const AcMeshInfo config)
{
    if (!d)
        return AC_FAILURE;
    return refresh_config(d, config);
}

extern "C" AcMeshInfo
acDeviceGetConfig(const Device d)
{
    AcMeshInfo info;
    if (!d) {
        memset(&info, 0, sizeof(info));
        return info;
    }
    return d->config;
}

/* ---- host <-> device ---- */

static bool
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
static AcResult
worst(const AcResult a, const AcResult b)
{
    if (a == AC_FAILURE || b == AC_FAILURE)
        return AC_FAILURE;
    return a == AC_NOT_ALLOCATED || b == AC_NOT_ALLOCATED ? AC_NOT_ALLOCATED : AC_SUCCESS;
}

extern "C" AcResult
acDeviceLoadVertexBuffer(const Device d, const Stream stream, const AcMesh host_mesh,
                         const VertexBufferHandle h)
{
    if (!d || !stream_ok(stream) || (int)h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    if (!host_mesh.vertex_buffer[h])
        return AC_NOT_ALLOCATED;
    if (!host_matches(d, host_mesh.info)) {
        fprintf(stderr, "astaroth_b200: host mesh dimensions differ from the device's\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const size_t n = (size_t)d->geom.mx * d->geom.my * d->geom.mz;
    const int b    = d->in_idx[h];
    if (d->precision == 0) {
        AC_CUDA_CHECK(cudaMemcpyAsync(arr64(d, b, h), host_mesh.vertex_buffer[h],
                                      n * sizeof(double), cudaMemcpyHostToDevice,
                                      d->streams[stream]));
    }
    else {
        /* through the staging field: double -> (hi, lo) on the device */
        AC_CUDA_CHECK(cudaMemcpyAsync(d->staging, host_mesh.vertex_buffer[h], n * sizeof(double),
                                      cudaMemcpyHostToDevice, d->streams[stream]));
        AC_CUDA_CHECK(ac_launch_split(d->geom, d->staging, arr_hi(d, b, h), arr_lo(d, b, h),
                                      d->streams[stream], &d->launches));
        /* the staging field is shared by all streams: finish before returning */
        AC_CUDA_CHECK(cudaStreamSynchronize(d->streams[stream]));
    }
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceLoadMesh(const Device d, const Stream stream, const AcMesh host_mesh)
{
    AcResult res = AC_SUCCESS;
    for (int q = 0; q < AC_NF; ++q)
        res = worst(res, acDeviceLoadVertexBuffer(d, stream, host_mesh, (VertexBufferHandle)q));
    return res;
}

extern "C" AcResult
acDeviceStoreVertexBuffer(const Device d, const Stream stream, const VertexBufferHandle h,
                          AcMesh* host_mesh)
{
    if (!d || !host_mesh || !stream_ok(stream) || (int)h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    if (!host_mesh->vertex_buffer[h])
        return AC_NOT_ALLOCATED;
    if (!host_matches(d, host_mesh->info)) {
        fprintf(stderr, "astaroth_b200: host mesh dimensions differ from the device's\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const size_t n = (size_t)d->geom.mx * d->geom.my * d->geom.mz;
    const int b    = d->in_idx[h];
    if (d->precision == 0) {
        AC_CUDA_CHECK(cudaMemcpyAsync(host_mesh->vertex_buffer[h], arr64(d, b, h),
                                      n * sizeof(double), cudaMemcpyDeviceToHost,
                                      d->streams[stream]));
    }
    else {
        AC_CUDA_CHECK(ac_launch_join(d->geom, arr_hi(d, b, h), arr_lo(d, b, h), d->staging,
                                     d->streams[stream], &d->launches));
        AC_CUDA_CHECK(cudaMemcpyAsync(host_mesh->vertex_buffer[h], d->staging, n * sizeof(double),
                                      cudaMemcpyDeviceToHost, d->streams[stream]));
    }
    /* The host array is ready when the call returns. */
    AC_CUDA_CHECK(cudaStreamSynchronize(d->streams[stream]));
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceStoreMesh(const Device d, const Stream stream, AcMesh* host_mesh)
{
    AcResult res = AC_SUCCESS;
    for (int q = 0; q < AC_NF; ++q)
        res = worst(res, acDeviceStoreVertexBuffer(d, stream, (VertexBufferHandle)q, host_mesh));
    return res;
}

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

extern "C" AcResult
acDeviceSetVertexBuffer(const Device d, const Stream stream, const VertexBufferHandle h,
                        const AcReal value)
{
    if (!d || !stream_ok(stream) || (int)h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const int b = d->in_idx[h];
    if (d->precision == 0)
        AC_CUDA_CHECK(ac_launch_fill(arr64(d, b, h), d->geom.cells, value, d->streams[stream],
                                     &d->launches));
    else
        AC_CUDA_CHECK(ac_launch_fill_comp(arr_hi(d, b, h), arr_lo(d, b, h), d->geom.cells, value,
                                          d->streams[stream], &d->launches));
    return AC_SUCCESS;
}

/* Zero-fills the in and/or out buffer of every field (value and compensation). */
static AcResult
clear_buffers(const Device d, cudaStream_t st, const bool in, const bool out)
{
    const size_t bytes = (size_t)d->geom.cells * elem_size(d);
    for (int q = 0; q < AC_NF; ++q)
        for (int side = 0; side < 2; ++side) {
            if ((side == 0 && !in) || (side == 1 && !out))
                continue;
            const int b = side == 0 ? d->in_idx[q] : 1 - d->in_idx[q];
            AC_CUDA_CHECK(cudaMemsetAsync((char*)d->hi[b] + q * bytes, 0, bytes, st));
            if (d->precision == 1)
                AC_CUDA_CHECK(cudaMemsetAsync(arr_lo(d, b, q), 0, bytes, st));
        }
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceFlushOutputBuffers(const Device d, const Stream stream)
{
    if (!d || !stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    return clear_buffers(d, d->streams[stream], false, true);
}

extern "C" AcResult
acDeviceResetMesh(const Device d, const Stream stream)
{
    if (!d || !stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    return clear_buffers(d, d->streams[stream], true, true);
}

/* ---- integration ---- */

static bool
is_whole_interior(const Device d, const Volume start, const Volume end)
{
    return start.x == NGHOST && start.y == NGHOST && start.z == NGHOST &&
           end.x == (size_t)(d->geom.nx + NGHOST) && end.y == (size_t)(d->geom.ny + NGHOST) &&
           end.z == (size_t)(d->geom.nz + NGHOST);
}

RkCoef
ac_rk_coef(const int step, const double dt)
{
    /* Williamson 2N RK3, acc-runtime/stdlib/integrators.h:11-13 */
    const double alpha[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
    const double beta[3]  = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
    RkCoef rk;
    rk.step = step;
    rk.dt   = dt;
    rk.beta = beta[step];
    rk.ab   = step == 0 ? 0.0 : alpha[step] / beta[step - 1];
    return rk;
}

static cudaError_t
launch_substep(Device d, cudaStream_t st, const int step, const double dt,
               unsigned long long* launches)
{
    StencilCoef sc;
    PhysConst pc;
    ac_make_stencil(d->config, &sc);
    ac_make_phys(d->config, &pc);
    if (step == 2)
        forcing_for_launch(d->config, dt, &pc);
    const RkCoef rk = ac_rk_coef(step, dt);
    if (step == 2 && d->config.int_params[AC_lbfield] && d->bfield) {
        /* B = curl A of this substep's input (the in-buffer is not written) */
        const void* a[3];
        double* b[3];
        const size_t nm = (size_t)d->geom.mx * d->geom.my * d->geom.mz;
        for (int c = 0; c < 3; ++c) {
            const int q = VTXBUF_AX + c;
            a[c] = d->precision == 0 ? (const void*)arr64(d, d->in_idx[q], q)
                                     : (const void*)arr_hi(d, d->in_idx[q], q);
            b[c] = d->bfield + c * nm;
        }
        const cudaError_t e = ac_launch_bfield(d->geom, a, b, d->precision, sc, st, launches);
        if (e != cudaSuccess)
            return e;
    }
    const int blk   = in_block_index(d);
    const bool tiled = d->solve_variant == 1 && d->tmap_ok && blk >= 0;
    /* substep 2 also produces the CFL maxima of its input state, as the
     * reference's calc_timestep inside the third substep (mhdsolver.ac:611) */
    unsigned long long* cfl = nullptr;
    if (step == 2) {
        const cudaError_t e = cudaMemsetAsync(d->cfl, 0, 3 * sizeof(unsigned long long), st);
        if (e != cudaSuccess)
            return e;
        cfl = d->cfl;
    }
    cudaError_t e;
    if (d->precision == 0) {
        const Fields64 f = fields64(d);
        e = tiled ? ac_launch_solve_tiled64(d->geom, &d->tmap[blk], f, sc, pc, rk, d->err_flag,
                                            cfl, st, launches)
                  : ac_launch_solve_plain64(d->geom, f, sc, pc, rk, cfl, st, launches);
    }
    else {
        const Fields32 f = fields32(d);
        e = tiled ? ac_launch_solve_tiled32(d->geom, &d->tmap[blk], f, sc, pc, rk, d->err_flag,
                                            cfl, st, launches)
                  : ac_launch_solve_plain32(d->geom, f, sc, pc, rk, cfl, st, launches);
    }
    if (e != cudaSuccess || !pc.forcing)
        return e;
    /* helical forcing of the substep's output velocity */
    void* u[3];
    float* lo[3];
    for (int c = 0; c < 3; ++c) {
        const int q = VTXBUF_UUX + c, b = 1 - d->in_idx[q];
        u[c]        = d->precision == 0 ? (void*)arr64(d, b, q) : (void*)arr_hi(d, b, q);
        lo[c]       = d->precision == 0 ? nullptr : arr_lo(d, b, q);
    }
    return ac_launch_forcing(d->geom, u, lo, d->precision, pc, st, launches);
}

/* Periodic halo fill of the in-buffer of fields [q0, q0 + nq). */
static cudaError_t
launch_periodic(Device d, cudaStream_t st, const int q0, const int nq, const Volume start,
                const Volume end, unsigned long long* launches)
{
    if (d->precision == 0) {
        double* a[AC_NF];
        for (int k = 0; k < nq; ++k)
            a[k] = arr64(d, d->in_idx[q0 + k], q0 + k);
        return ac_launch_periodic<double>(d->geom, a, nq, start, end, st, launches);
    }
    float* a[2 * AC_NF];
    for (int k = 0; k < nq; ++k) {
        a[2 * k]     = arr_hi(d, d->in_idx[q0 + k], q0 + k);
        a[2 * k + 1] = arr_lo(d, d->in_idx[q0 + k], q0 + k);
    }
    return ac_launch_periodic<float>(d->geom, a, 2 * nq, start, end, st, launches);
}

extern "C" AcResult
acDeviceIntegrateSubstep(const Device d, const Stream stream, const int step_number,
                         const Volume start, const Volume end, const AcReal dt)
{
    if (!d || !stream_ok(stream) || step_number < 0 || step_number > 2)
        return AC_FAILURE;
    /* As the reference's default (two-pass) build, device.cc:965-970, only the
     * whole interior is accepted. */
    if (!is_whole_interior(d, start, end)) {
        fprintf(stderr, "astaroth_b200: acDeviceIntegrateSubstep needs start = nmin and "
                        "end = nmin + nlocal\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    AC_CUDA_CHECK(launch_substep(d, d->streams[stream], step_number, dt, &d->launches));
    if (step_number == 2)
        d->out_set = 0;
    return AC_SUCCESS;
}

extern "C" AcResult
acDevicePeriodicBoundcondStep(const Device d, const Stream stream, const VertexBufferHandle h,
                              const Volume start, const Volume end)
{
    if (!d || !stream_ok(stream) || (int)h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    AC_CUDA_CHECK(launch_periodic(d, d->streams[stream], h, 1, start, end, &d->launches));
    return AC_SUCCESS;
}

extern "C" AcResult
acDevicePeriodicBoundconds(const Device d, const Stream stream, const Volume start,
                           const Volume end)
{
    if (!d || !stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    AC_CUDA_CHECK(launch_periodic(d, d->streams[stream], 0, AC_NF, start, end, &d->launches));
    return AC_SUCCESS;
}

static cudaError_t
record_step(Device d, cudaStream_t st, const double dt, unsigned long long* launches)
{
    const Volume m0 = {0, 0, 0};
    const Volume m1 = {(size_t)d->geom.mx, (size_t)d->geom.my, (size_t)d->geom.mz};
    for (int s = 0; s < 3; ++s) {
        cudaError_t e = launch_periodic(d, st, 0, AC_NF, m0, m1, launches);
        if (e != cudaSuccess)
            return e;
        e = launch_substep(d, st, s, dt, launches);
        if (e != cudaSuccess)
            return e;
        acDeviceSwapBuffers(d);
    }
    return cudaSuccess;
}

extern "C" AcResult
acDeviceIntegrateStep(const Device d, const Stream stream, const AcReal dt)
{
    if (!d || !stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    cudaStream_t st = d->streams[stream];
    /* All fields must be in the same buffer for the graph (true unless the
     * caller swapped single fields); otherwise run the launches directly. */
    const int parity = in_block_index(d);
    if (parity < 0) {
        AC_CUDA_CHECK(record_step(d, st, dt, &d->launches));
        d->out_set = 0;
        return AC_SUCCESS;
    }
    StepGraph& sg = d->graphs[stream][parity];
    if (!sg.valid || sg.dt != dt) {
        if (sg.valid)
            cudaGraphExecDestroy(sg.exec);
        sg.valid = 0;
        cudaGraph_t graph;
        AC_CUDA_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const cudaError_t rec = record_step(d, st, dt, NULL);
        const cudaError_t end = cudaStreamEndCapture(st, &graph);
        acDeviceSwapBuffers(d); /* undo the capture's swaps (three swaps = one) */
        AC_CUDA_CHECK(rec);
        AC_CUDA_CHECK(end);
        const cudaError_t inst = cudaGraphInstantiate(&sg.exec, graph, 0);
        cudaGraphDestroy(graph);
        AC_CUDA_CHECK(inst);
        sg.valid = 1;
        sg.dt    = dt;
    }
    AC_CUDA_CHECK(cudaGraphLaunch(sg.exec, st));
    d->launches += 6;
    d->out_set = 0;
    acDeviceSwapBuffers(d);
    return AC_SUCCESS;
}

/* ---- reductions ---- */

static AcResult
reduce_common(const Device d, const Stream stream, const AcReduction r, const int kind,
              const VertexBufferHandle* h, AcReal* result)
{
    if (!d || !result || !stream_ok(stream))
        return AC_FAILURE;
    for (int q = 0; q < kind; ++q)
        if ((int)h[q] < 0 || h[q] >= NUM_VTXBUF_HANDLES)
            return AC_NOT_ALLOCATED;
    const int map = kind == 1 ? r.map_vtxbuf_single
                              : kind == 3 ? r.map_vtxbuf_vec : r.map_vtxbuf_vec_scal;
    const bool map_ok = kind == 1 ? (map >= AC_MAP_VTXBUF && map <= AC_MAP_VTXBUF_EXP_SQUARE)
                        : kind == 3 ? (map >= AC_MAP_VTXBUF3_NORM &&
                                       map <= AC_MAP_VTXBUF3_EXP_SQUARE)
                                    : (map >= AC_MAP_VTXBUF4_ALFVEN_NORM &&
                                       map <= AC_MAP_VTXBUF4_ALFVEN_SQUARE);
    if (!map_ok) {
        fprintf(stderr, "astaroth_b200: invalid reduction type for this call\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    /* Reductions observe all previously issued work of this device
     * (the reference synchronizes the device first, reductions.cu:103). */
    for (int s = 0; s < NUM_STREAMS; ++s)
        if (s != (int)stream)
            AC_CUDA_CHECK(cudaStreamSynchronize(d->streams[s]));
    const void* fp[4];
    const float* lo[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int q = 0; q < kind; ++q) {
        const int b = d->in_idx[h[q]];
        if (d->precision == 0) {
            fp[q] = arr64(d, b, h[q]);
        }
        else {
            fp[q] = arr_hi(d, b, h[q]);
            lo[q] = arr_lo(d, b, h[q]);
        }
    }
    cudaStream_t st = d->streams[stream];
    AC_CUDA_CHECK(ac_launch_reduce(d->geom, fp, lo, kind, d->precision, map, r.reduce_op, d->red,
                                   st, &d->launches));
    AC_CUDA_CHECK(cudaMemcpyAsync(d->host_result, d->red.result, sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
    AC_CUDA_CHECK(cudaStreamSynchronize(st));
    *result = *d->host_result;
    return AC_SUCCESS;
}

/* device.cc:1384-1401 */
static AcReal
post_process(const Device d, const AcReductionPostProcessingOp op, const AcReal v)
{
    if (op == AC_RMS) {
        const AcReal inv_n =
            AcReal(1.) / ((double)d->geom.nx * (double)d->geom.ny * (double)d->geom.nz);
        return sqrt(inv_n * v);
    }
    return v;
}

extern "C" AcResult
acDeviceReduceScalNoPostProcessing(const Device d, const Stream stream, const AcReduction r,
                                   const VertexBufferHandle h, AcReal* result)
{
    return reduce_common(d, stream, r, 1, &h, result);
}

extern "C" AcResult
acDeviceReduceScal(const Device d, const Stream stream, const AcReduction r,
                   const VertexBufferHandle h, AcReal* result)
{
    const AcResult res = reduce_common(d, stream, r, 1, &h, result);
    if (res == AC_SUCCESS)
        *result = post_process(d, r.post_processing_op, *result);
    return res;
}

extern "C" AcResult
acDeviceReduceVecNoPostProcessing(const Device d, const Stream stream, const AcReduction r,
                                  const VertexBufferHandle a, const VertexBufferHandle b,
                                  const VertexBufferHandle c, AcReal* result)
{
    const VertexBufferHandle h[3] = {a, b, c};
    return reduce_common(d, stream, r, 3, h, result);
}

extern "C" AcResult
acDeviceReduceVec(const Device d, const Stream stream, const AcReduction r,
                  const VertexBufferHandle a, const VertexBufferHandle b,
                  const VertexBufferHandle c, AcReal* result)
{
    const VertexBufferHandle h[3] = {a, b, c};
    const AcResult res            = reduce_common(d, stream, r, 3, h, result);
    if (res == AC_SUCCESS)
        *result = post_process(d, r.post_processing_op, *result);
    return res;
}

extern "C" AcResult
acDeviceReduceVecScalNoPostProcessing(const Device d, const Stream stream, const AcReduction r,
                                      const VertexBufferHandle a, const VertexBufferHandle b,
                                      const VertexBufferHandle c, const VertexBufferHandle e,
                                      AcReal* result)
{
    const VertexBufferHandle h[4] = {a, b, c, e};
    return reduce_common(d, stream, r, 4, h, result);
}

extern "C" AcResult
acDeviceReduceVecScal(const Device d, const Stream stream, const AcReduction r,
                      const VertexBufferHandle a, const VertexBufferHandle b,
                      const VertexBufferHandle c, const VertexBufferHandle e, AcReal* result)
{
    const VertexBufferHandle h[4] = {a, b, c, e};
    const AcResult res            = reduce_common(d, stream, r, 4, h, result);
    if (res == AC_SUCCESS)
        *result = post_process(d, r.post_processing_op, *result);
    return res;
}

/* ---- misc ---- */

extern "C" AcResult
acDeviceGetVertexBufferPtrs(Device d, const VertexBufferHandle h, AcReal** in, AcReal** out)
{
    if (!d || !in || !out || (int)h < 0 || h >= NUM_VTXBUF_HANDLES)
        return AC_FAILURE;
    if (d->precision != 0) {
        fprintf(stderr, "astaroth_b200: acDeviceGetVertexBufferPtrs needs an FP64 device\n");
        return AC_FAILURE;
    }
    *in  = arr64(d, d->in_idx[h], h);
    *out = arr64(d, 1 - d->in_idx[h], h);
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceMemGetInfo(const Device d, size_t* free_mem, size_t* total_mem)
{
    if (!d || !free_mem || !total_mem)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    AC_CUDA_CHECK(cudaMemGetInfo(free_mem, total_mem));
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceCalcTimestep(const Device d, const Stream stream)
{
    if (!d || !stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    StencilCoef sc;
    ac_make_stencil(d->config, &sc);
    const double cs2 = d->config.real_params[AC_cs_sound] * d->config.real_params[AC_cs_sound];
    if (d->precision == 0)
        AC_CUDA_CHECK(ac_launch_cfl<double>(d->geom, fields64(d), sc, cs2, d->cfl,
                                            d->streams[stream], &d->launches));
    else
        AC_CUDA_CHECK(ac_launch_cfl<float>(d->geom, fields32(d), sc, cs2, d->cfl,
                                           d->streams[stream], &d->launches));
    d->out_set = 0;
    return AC_SUCCESS;
}

/* dt of the additive form, mhdsolver.ac:558-569: the minimum over cells of
 * min(visc_dt, advec_dt); visc_dt is uniform, so the minimum of advec_dt comes
 * from the maximum of |u| + sqrt(cs^2 + vA^2) */
static double
additive_dt(const AcMeshInfo& c, const double advec_sum_max)
{
    const double dsmin   = c.real_params[AC_dsmin];
    double visc          = c.real_params[AC_nu_visc] > c.real_params[AC_eta]
                               ? c.real_params[AC_nu_visc]
                               : c.real_params[AC_eta];
    const double gchi    = c.real_params[AC_gamma] * c.real_params[AC_chi];
    visc                 = visc > gchi ? visc : gchi;
    const double visc_dt = visc > 0 ? c.real_params[AC_cdtv] * dsmin * dsmin / visc : INFINITY;
    const double advec_dt = c.real_params[AC_cdt] * dsmin / advec_sum_max;
    return visc_dt < advec_dt ? visc_dt : advec_dt;
}

/* The outputs as the device reduced them, after waiting for `st` (all of the
 * device's streams when st is NULL). */
static cudaError_t
device_outputs(Device d, const cudaStream_t* st, double v[NUM_REAL_OUTPUTS])
{
    cudaError_t e = cudaSetDevice(d->id);
    if (e != cudaSuccess)
        return e;
    if (st) {
        e = cudaStreamSynchronize(*st);
        if (e != cudaSuccess)
            return e;
    }
    else {
        for (int s = 0; s < NUM_STREAMS; ++s)
            if ((e = cudaStreamSynchronize(d->streams[s])) != cudaSuccess)
                return e;
    }
    unsigned long long w[3];
    if ((e = cudaMemcpy(w, d->cfl, sizeof(w), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return e;
    double m[3];
    memcpy(m, w, sizeof(m));
    v[UU_MAX_ADVEC]     = m[0];
    v[ALFVEN_SPEED_MAX] = m[1];
    v[AC_dt_min]        = additive_dt(d->config, m[2]);
    return cudaSuccess;
}

/* The device's outputs with the acDeviceSetOutput values in their place. */
static cudaError_t
current_outputs(Device d, double v[NUM_REAL_OUTPUTS])
{
    const unsigned all = (1u << NUM_REAL_OUTPUTS) - 1;
    if ((d->out_set & all) != all) {
        const cudaError_t e = device_outputs(d, NULL, v);
        if (e != cudaSuccess)
            return e;
    }
    for (int p = 0; p < NUM_REAL_OUTPUTS; ++p)
        if (d->out_set >> p & 1)
            v[p] = d->outputs[p];
    return cudaSuccess;
}

extern "C" AcResult
acDeviceGetTimestepMaxima(const Device d, AcReal* uu_max, AcReal* alfven_max)
{
    if (!d || !uu_max || !alfven_max)
        return AC_FAILURE;
    double v[NUM_REAL_OUTPUTS];
    AC_CUDA_CHECK(current_outputs(d, v));
    *uu_max     = v[UU_MAX_ADVEC];
    *alfven_max = v[ALFVEN_SPEED_MAX];
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceGetTimestep(const Device d, AcReal* dt)
{
    if (!d || !dt)
        return AC_FAILURE;
    double v[NUM_REAL_OUTPUTS];
    AC_CUDA_CHECK(current_outputs(d, v));
    *dt = d->config.int_params[AC_additive_timestep]
              ? v[AC_dt_min]
              : acHostTimestepFromMaxima(d->config, v[UU_MAX_ADVEC], v[ALFVEN_SPEED_MAX]);
    return AC_SUCCESS;
}

static AcResult
finish_reduce(Device d, const cudaStream_t st, AcReal* result, const AcKernel kernel,
              const AcReduceOp op, const AcRealOutputParam output)
{
    if (!d || !result || (int)output < 0 || output >= NUM_REAL_OUTPUTS ||
        (kernel != AC_KERNEL_SOLVE && kernel != AC_KERNEL_CALC_TIMESTEP))
        return AC_FAILURE;
    const AcReduceOp own = output == AC_dt_min ? AC_REDUCE_OP_MIN : AC_REDUCE_OP_MAX;
    if (op != own)
        return AC_FAILURE;
    double v[NUM_REAL_OUTPUTS];
    AC_CUDA_CHECK(device_outputs(d, &st, v));
    d->out_set &= ~(1u << output);
    *result = v[output];
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceFinishReduceReal(Device d, const Stream stream, AcReal* result, const AcKernel kernel,
                         const AcReduceOp reduce_op, const AcRealOutputParam output)
{
    if (!d || !stream_ok(stream))
        return AC_FAILURE;
    return finish_reduce(d, d->streams[stream], result, kernel, reduce_op, output);
}

extern "C" AcResult
acDeviceFinishReduceRealStream(Device d, struct CUstream_st* stream, AcReal* result,
                               const AcKernel kernel, const AcReduceOp reduce_op,
                               const AcRealOutputParam output)
{
    return finish_reduce(d, (cudaStream_t)stream, result, kernel, reduce_op, output);
}

extern "C" AcReal
acDeviceGetOutput(const Device d, const AcRealOutputParam param)
{
    if (!d || (int)param < 0 || param >= NUM_REAL_OUTPUTS)
        return NAN;
    if (d->out_set >> param & 1)
        return d->outputs[param];
    double v[NUM_REAL_OUTPUTS];
    if (device_outputs(d, NULL, v) != cudaSuccess)
        return NAN;
    return v[param];
}

extern "C" AcResult
acDeviceSetOutput(const Device d, const AcRealOutputParam param, const AcReal value)
{
    if (!d || (int)param < 0 || param >= NUM_REAL_OUTPUTS)
        return AC_FAILURE;
    d->outputs[param] = value;
    d->out_set |= 1u << param;
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

/* ---- discrete adjoint ---- */

static AcResult
ensure_adjoint(const Device d)
{
    if (d->precision != 0) {
        fprintf(stderr, "astaroth_b200: the adjoint needs an FP64 device (AC_precision = 0)\n");
        return AC_FAILURE;
    }
    if (d->config.int_params[AC_upwind]) {
        /* |u| in the upwinding terms has no derivative at u = 0; the reverse
         * pass covers the equations without them */
        fprintf(stderr, "astaroth_b200: the adjoint does not cover AC_upwind\n");
        return AC_FAILURE;
    }
    if (d->adj_lf)
        return AC_SUCCESS;
    const size_t fb = (size_t)d->geom.cells * sizeof(double);
    AC_CUDA_CHECK(cudaMalloc((void**)&d->adj_lf, AC_NF * fb));
    AC_CUDA_CHECK(cudaMalloc((void**)&d->adj_lw, AC_NF * fb));
    AC_CUDA_CHECK(cudaMalloc((void**)&d->adj_mu, AC_MU_COUNT * fb));
    AC_CUDA_CHECK(cudaMalloc((void**)&d->adj_pgrad, 2 * sizeof(double)));
    AC_CUDA_CHECK(cudaMemset(d->adj_mu, 0, AC_MU_COUNT * fb));
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceLoadAdjoint(const Device d, const Stream stream, const AcReal* const* lam_f)
{
    if (!d || !stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    if (ensure_adjoint(d) != AC_SUCCESS)
        return AC_FAILURE;
    cudaStream_t st = d->streams[stream];
    const size_t fb = (size_t)d->geom.cells * sizeof(double);
    for (int q = 0; q < AC_NF; ++q) {
        if (lam_f && lam_f[q])
            AC_CUDA_CHECK(cudaMemcpyAsync(d->adj_lf + (size_t)q * d->geom.cells, lam_f[q], fb,
                                          cudaMemcpyDeviceToDevice, st));
        else
            AC_CUDA_CHECK(cudaMemsetAsync(d->adj_lf + (size_t)q * d->geom.cells, 0, fb, st));
    }
    AC_CUDA_CHECK(cudaMemsetAsync(d->adj_lw, 0, AC_NF * fb, st));
    AC_CUDA_CHECK(cudaMemsetAsync(d->adj_pgrad, 0, 2 * sizeof(double), st));
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceStoreAdjoint(const Device d, const Stream stream, AcReal* const* lam_f)
{
    if (!d || !lam_f || !stream_ok(stream) || !d->adj_lf)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const size_t fb = (size_t)d->geom.cells * sizeof(double);
    for (int q = 0; q < AC_NF; ++q)
        if (lam_f[q])
            AC_CUDA_CHECK(cudaMemcpyAsync(lam_f[q], d->adj_lf + (size_t)q * d->geom.cells, fb,
                                          cudaMemcpyDeviceToDevice, d->streams[stream]));
    return AC_SUCCESS;
}

/* One adjoint substep about the state `state` (8 fields at q * cells, halos
 * filled), or about the in-buffers when state is NULL. */
static cudaError_t
launch_adjoint(const Device d, cudaStream_t st, const int step, const double dt,
               const double* state)
{
    StencilCoef sc;
    PhysConst pc;
    ac_make_stencil(d->config, &sc);
    ac_make_phys(d->config, &pc);
    AdjointFields a;
    for (int q = 0; q < AC_NF; ++q) {
        a.f[q]  = state ? state + (size_t)q * d->geom.cells : arr64(d, d->in_idx[q], q);
        a.lf[q] = d->adj_lf + (size_t)q * d->geom.cells;
        a.lw[q] = d->adj_lw + (size_t)q * d->geom.cells;
    }
    for (int m = 0; m < AC_MU_COUNT; ++m)
        a.mu[m] = d->adj_mu + (size_t)m * d->geom.cells;
    const double alpha[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
    const double beta[3]  = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
    return ac_launch_adjoint_substep(d->geom, a, sc, pc, alpha[step], beta[step], dt,
                                     d->adj_pgrad, st, &d->launches);
}

extern "C" AcResult
acDeviceIntegrateSubstepAdjoint(const Device d, const Stream stream, const int step_number,
                                const Volume start, const Volume end, const AcReal dt)
{
    if (!d || !stream_ok(stream) || step_number < 0 || step_number > 2 || !d->adj_lf)
        return AC_FAILURE;
    if (ensure_adjoint(d) != AC_SUCCESS)
        return AC_FAILURE;
    if (!is_whole_interior(d, start, end)) {
        fprintf(stderr, "astaroth_b200: acDeviceIntegrateSubstepAdjoint needs the whole interior\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    AC_CUDA_CHECK(launch_adjoint(d, d->streams[stream], step_number, dt, NULL));
    return AC_SUCCESS;
}

/* The launches of a tape recompute: per substep, halo fill, copy of the
 * in-block to the tape, substep, swap. */
static cudaError_t
record_tape(Device d, cudaStream_t st, const int steps, const double dt)
{
    const size_t state_elems = (size_t)AC_NF * d->geom.cells;
    const Volume m0          = {0, 0, 0};
    const Volume m1          = {(size_t)d->geom.mx, (size_t)d->geom.my, (size_t)d->geom.mz};
    for (int n = 0; n < steps; ++n)
        for (int s = 0; s < 3; ++s) {
            cudaError_t e = launch_periodic(d, st, 0, AC_NF, m0, m1, NULL);
            if (e != cudaSuccess)
                return e;
            /* the 8 in-buffers are one contiguous block: one copy per state */
            e = ac_launch_copy(arr64(d, d->in_idx[0], 0),
                               d->adj_tape + (size_t)(3 * n + s) * state_elems,
                               (long long)state_elems, st, NULL);
            if (e != cudaSuccess)
                return e;
            e = launch_substep(d, st, s, dt, NULL);
            if (e != cudaSuccess)
                return e;
            acDeviceSwapBuffers(d);
        }
    return cudaSuccess;
}

extern "C" AcResult
acDeviceAdjointTapeForward(const Device d, const Stream stream, const int steps, const AcReal dt)
{
    if (!d || !stream_ok(stream) || steps < 1)
        return AC_FAILURE;
    const int blk = in_block_index(d);
    if (blk < 0) {
        fprintf(stderr, "astaroth_b200: the tape needs every field's in-buffer in one block\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    if (ensure_adjoint(d) != AC_SUCCESS)
        return AC_FAILURE;
    const size_t state_elems = (size_t)AC_NF * d->geom.cells;
    if (d->adj_tape_states < 3 * steps) {
        AC_CUDA_CHECK(cudaDeviceSynchronize());
        invalidate_tape_graph(d);
        cudaFree(d->adj_tape);
        d->adj_tape        = NULL;
        d->adj_tape_states = 0;
        AC_CUDA_CHECK(cudaMalloc((void**)&d->adj_tape, 3 * (size_t)steps * state_elems *
                                                           sizeof(double)));
        d->adj_tape_states = 3 * steps;
    }
    cudaStream_t st = d->streams[stream];
    /* the recompute is one CUDA graph per in-block, kept for the next call
     * with the same steps, dt and stream (one capture per checkpoint length) */
    if (!(d->tape_valid[blk] && d->tape_steps[blk] == steps && d->tape_dt[blk] == dt &&
          d->tape_stream[blk] == (int)stream)) {
        if (d->tape_valid[blk])
            cudaGraphExecDestroy(d->tape_exec[blk]);
        d->tape_valid[blk] = 0;
        cudaGraph_t graph;
        AC_CUDA_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const cudaError_t rec = record_tape(d, st, steps, dt);
        const cudaError_t end = cudaStreamEndCapture(st, &graph);
        for (int q = 0; q < AC_NF; ++q) /* undo the capture's swaps */
            d->in_idx[q] = blk;
        AC_CUDA_CHECK(rec);
        AC_CUDA_CHECK(end);
        const cudaError_t inst = cudaGraphInstantiate(&d->tape_exec[blk], graph, 0);
        cudaGraphDestroy(graph);
        AC_CUDA_CHECK(inst);
        d->tape_valid[blk]  = 1;
        d->tape_steps[blk]  = steps;
        d->tape_dt[blk]     = dt;
        d->tape_stream[blk] = (int)stream;
    }
    AC_CUDA_CHECK(cudaGraphLaunch(d->tape_exec[blk], st));
    d->launches += 9ull * steps;
    d->out_set = 0;
    if ((3 * steps) & 1) /* three swaps per step */
        acDeviceSwapBuffers(d);
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceAdjointTapeBackward(const Device d, const Stream stream, const int steps,
                            const AcReal dt)
{
    if (!d || !stream_ok(stream) || steps < 1)
        return AC_FAILURE;
    if (!d->adj_lf || d->adj_tape_states < 3 * steps) {
        fprintf(stderr,
                "astaroth_b200: acDeviceAdjointTapeBackward(%d steps) needs acDeviceLoadAdjoint "
                "and a tape of %d states (has %d)\n",
                steps, 3 * steps, d->adj_tape_states);
        return AC_FAILURE;
    }
    if (ensure_adjoint(d) != AC_SUCCESS)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    cudaStream_t st             = d->streams[stream];
    const size_t state_elems    = (size_t)AC_NF * d->geom.cells;
    for (int n = steps - 1; n >= 0; --n)
        for (int s = 2; s >= 0; --s)
            AC_CUDA_CHECK(launch_adjoint(d, st, s, dt,
                                         d->adj_tape + (size_t)(3 * n + s) * state_elems));
    return AC_SUCCESS;
}

extern "C" AcResult
acDeviceGetParamAdjoints(const Device d, AcReal* nu_bar, AcReal* eta_bar)
{
    if (!d || !nu_bar || !eta_bar || !d->adj_pgrad)
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    for (int s = 0; s < NUM_STREAMS; ++s)
        AC_CUDA_CHECK(cudaStreamSynchronize(d->streams[s]));
    double v[2];
    AC_CUDA_CHECK(cudaMemcpy(v, d->adj_pgrad, sizeof(v), cudaMemcpyDeviceToHost));
    *nu_bar  = v[0];
    *eta_bar = v[1];
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

static AcResult
copy_planes(const Device d, const Stream stream, const int z0, const int nplanes, char* buffer,
            const bool pack)
{
    if (!planes_ok(d, z0, nplanes) || !buffer || !stream_ok(stream))
        return AC_FAILURE;
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    const size_t es = elem_size(d);
    void* arrays[2 * AC_NF];
    for (int a = 0; a < plane_arrays(d); ++a) {
        const int q = a % AC_NF;
        arrays[a]   = a < AC_NF ? (void*)((char*)d->hi[d->in_idx[q]] + (size_t)q * d->geom.cells * es)
                                : (void*)arr_lo(d, d->in_idx[q], q);
    }
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

extern "C" void*
acDeviceGetStreamHandle(const Device d, const Stream stream)
{
    if (!d || !stream_ok(stream))
        return NULL;
    return (void*)d->streams[stream];
}

extern "C" unsigned long long
acDeviceGetLaunchCount(const Device d)
{
    return d ? d->launches : 0ull;
}
