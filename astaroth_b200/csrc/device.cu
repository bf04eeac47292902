/*
 * The device object and the acDevice* C ABI (include/astaroth_b200.h):
 * creation, configuration, whole-mesh host transfers, the substep and step,
 * boundary conditions, reductions and the CFL outputs.  Ranges, transfers
 * between devices, staged loads, plane packing and snapshots are in
 * device_data.cu; the discrete adjoint is in device_adjoint.cu.
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

#include "internal.h"
#include "device_impl.h"

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
    pc->debug_skip_load = 0;
    pc->cfl_sum         = info.int_params[AC_additive_timestep] != 0;
    pc->zlo             = 0;
    pc->zhi             = info.int3_params[AC_nlocal].z;
    pc->forcing      = 0;
    for (int a = 0; a < 3; ++a)
        pc->f_k[a] = pc->f_re[a] = pc->f_im[a] = 0.0;
    pc->f_cos_phase = 1.0;
    pc->f_sin_phase = 0.0;
    pc->f_scale     = 0.0;
}

/* The forcing of a substep-2 launch (mhdsolver.ac:531-541): active when
 * AC_lforcing is set and AC_current_time > AC_switch_forcing. */
/* AC_debug_plain_kernel: 0 = the automatic tiled choice (default), 1 = the plain
 * kernel, 2 = the per-plane tap tiled kernel, 3 = the leading-plane kernel,
 * 4 = the leading-plane kernel with the other group exchange */
static int
solve_variant_of(const AcMeshInfo& info)
{
    switch (info.int_params[AC_debug_plain_kernel]) {
    case 1: return 0;
    case 2: return AC_SOLVE_TILED_TAPS;
    case 3: return AC_SOLVE_TILED_LEAD;
    case 4: return AC_SOLVE_TILED_LEAD_ALT;
    default: return AC_SOLVE_TILED_AUTO;
    }
}

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

void
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
    cudaFree(d->adj_state);
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

/* Host-side fault injection for the failure-path tests.  With the environment
 * variable AC_FAULT_INJECT set to
 *   "create": acDeviceCreate fails before it allocates anything;
 *   "alloc":  acDeviceCreate's second state allocation fails, after the first
 *             succeeded, so its release path runs;
 *   "launch": every substep launch fails,
 * each as the CUDA call at that point would fail.  Unset, it costs one getenv
 * per create and per substep launch. */
static bool
fault_at(const char* site)
{
    const char* v = getenv("AC_FAULT_INJECT");
    return v && strcmp(v, site) == 0;
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
    if (fault_at("create")) {
        fprintf(stderr, "astaroth_b200: acDeviceCreate failed (AC_FAULT_INJECT=create)\n");
        return AC_FAILURE;
    }

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
    d->solve_variant = solve_variant_of(info);

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
        CREATE_CHECK(b == 1 && fault_at("alloc") ? cudaErrorMemoryAllocation
                                                 : cudaMalloc(&d->hi[b], bytes));
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
    d->red.nonfinite = (unsigned int*)(d->red.result + 1);
    d->red.counter = (unsigned int*)(d->red.result + 2);
    d->err_flag    = (int*)(d->red.counter + 4);
    d->cfl         = (unsigned long long*)(d->red.counter + 8);
    d->tmap_ok     = ac_make_tensor_map(&d->tmap[0], d->hi[0], d->geom, precision) &&
                 ac_make_tensor_map(&d->tmap[1], d->hi[1], d->geom, precision);
    if (d->tmap_ok)
        CREATE_CHECK(ac_solve_tiled_init(precision));
    CREATE_CHECK(cudaMallocHost((void**)&d->host_result, 2 * sizeof(double)));
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
acDeviceDebugSkipPlaneLoad(const Device d, const int enable)
{
    if (!d)
        return AC_FAILURE;
    if ((enable != 0) != (d->debug_skip_load != 0)) {
        d->debug_skip_load = enable != 0;
        invalidate_graphs(d); /* captured launches carry the switch */
    }
    return AC_SUCCESS;
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
        d->solve_variant = solve_variant_of(d->config);
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

cudaError_t
launch_substep(Device d, cudaStream_t st, const int step, const double dt,
               unsigned long long* launches, const int zlo, const int zhi)
{
    if (fault_at("launch"))
        return cudaErrorLaunchFailure;
    StencilCoef sc;
    PhysConst pc;
    ac_make_stencil(d->config, &sc);
    ac_make_phys(d->config, &pc);
    pc.debug_skip_load = d->debug_skip_load;
    if (zhi >= 0) {
        pc.zlo = zlo;
        pc.zhi = zhi;
    }
    /* substep 2 in z boxes: the CFL maxima (and B) are set up at the first box,
     * when the planes solved since the last clear cover the interior */
    bool first_box = true;
    if (step == 2) {
        const bool whole = pc.zlo == 0 && pc.zhi == d->geom.nz;
        first_box        = whole || d->cfl_cover <= 0 || d->cfl_cover >= d->geom.nz;
        d->cfl_cover     = (first_box ? 0 : d->cfl_cover) + (pc.zhi - pc.zlo);
    }
    if (step == 2)
        forcing_for_launch(d->config, dt, &pc);
    const RkCoef rk = ac_rk_coef(step, dt);
    if (step == 2 && first_box && d->config.int_params[AC_lbfield] && d->bfield) {
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
    const bool tiled = d->solve_variant != 0 && d->tmap_ok && blk >= 0;
    /* substep 2 also produces the CFL maxima of its input state, as the
     * reference's calc_timestep inside the third substep (mhdsolver.ac:611) */
    unsigned long long* cfl = nullptr;
    if (step == 2) {
        if (first_box) {
            const cudaError_t e = cudaMemsetAsync(d->cfl, 0, 3 * sizeof(unsigned long long), st);
            if (e != cudaSuccess)
                return e;
        }
        cfl = d->cfl;
    }
    cudaError_t e;
    if (d->precision == 0) {
        const Fields64 f = fields64(d);
        e = tiled ? ac_launch_solve_tiled64(d->geom, &d->tmap[blk], f, sc, pc, rk, d->err_flag,
                                            cfl, st, launches, d->solve_variant)
                  : ac_launch_solve_plain64(d->geom, f, sc, pc, rk, cfl, st, launches);
    }
    else {
        const Fields32 f = fields32(d);
        e = tiled ? ac_launch_solve_tiled32(d->geom, &d->tmap[blk], f, sc, pc, rk, d->err_flag,
                                            cfl, st, launches, d->solve_variant)
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
cudaError_t
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
    /* The whole interior, as the reference's default (two-pass) build,
     * device.cc:965-970, or a box of whole interior x-y planes: the singlepass
     * build solves any box (device.cc:941-964) and its task graph solves the
     * inner planes while the halos travel (task.cc:1933-1993); z boxes are that
     * split for the z-slab grid.  The boxes of one substep cover the interior
     * once; in substep 2 their CFL maxima accumulate from the first box on. */
    if (!is_z_box(d, start, end)) {
        fprintf(stderr, "astaroth_b200: acDeviceIntegrateSubstep needs start.xy = nmin.xy, "
                        "end.xy = nmin.xy + nlocal.xy and nmin.z <= start.z < end.z <= "
                        "nmin.z + nlocal.z\n");
        return AC_FAILURE;
    }
    AC_CUDA_CHECK(cudaSetDevice(d->id));
    AC_CUDA_CHECK(launch_substep(d, d->streams[stream], step_number, dt, &d->launches,
                                 (int)start.z - NGHOST, (int)end.z - NGHOST));
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
        cudaGraph_t graph = nullptr;
        int in_idx[AC_NF];
        memcpy(in_idx, d->in_idx, sizeof(in_idx));
        AC_CUDA_CHECK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const cudaError_t rec = record_step(d, st, dt, NULL);
        const cudaError_t end = cudaStreamEndCapture(st, &graph);
        /* the capture's swaps (three on success, fewer when a launch failed) undone */
        memcpy(d->in_idx, in_idx, sizeof(in_idx));
        if (rec != cudaSuccess || end != cudaSuccess) {
            if (graph)
                cudaGraphDestroy(graph);
            AC_CUDA_CHECK(rec);
            AC_CUDA_CHECK(end);
        }
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
    AC_CUDA_CHECK(cudaMemsetAsync(d->red.nonfinite, 0, sizeof(unsigned int), st));
    AC_CUDA_CHECK(ac_launch_reduce(d->geom, fp, lo, kind, d->precision, map, r.reduce_op, d->red,
                                   st, &d->launches));
    /* the result and the non-finite flag behind it */
    AC_CUDA_CHECK(cudaMemcpyAsync(d->host_result, d->red.result, 2 * sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
    AC_CUDA_CHECK(cudaStreamSynchronize(st));
    *result           = d->host_result[0];
    unsigned int flag = 0;
    memcpy(&flag, &d->host_result[1], sizeof(flag));
    d->last_nonfinite = flag != 0;
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

/* Whether the last acDeviceReduce* call on this device met a mapped value that
 * was NaN or infinite (a maximum or minimum drops NaN, so the value alone does
 * not show it). */
extern "C" AcResult
acDeviceGetReduceNonFinite(const Device d, int* nonfinite)
{
    if (!d || !nonfinite)
        return AC_FAILURE;
    *nonfinite = d->last_nonfinite;
    return AC_SUCCESS;
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
