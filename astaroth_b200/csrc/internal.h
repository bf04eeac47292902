/*
 * Internal declarations shared by the translation units of libastaroth_b200:
 * the device object, kernel parameter blocks and the launchers each .cu file
 * provides.  Not part of the public C ABI (include/astaroth_b200.h).
 */
#pragma once

#include <cuda.h> /* CUtensorMap (encoded through cudaGetDriverEntryPoint) */
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "astaroth_b200.h"

#define AC_NF 8 /* number of fields of the MHD module */

/* Report a CUDA error and return AC_FAILURE from the calling API function. */
#define AC_CUDA_CHECK(call)                                                                   \
    do {                                                                                      \
        const cudaError_t ac_err_ = (call);                                                   \
        if (ac_err_ != cudaSuccess) {                                                         \
            fprintf(stderr, "astaroth_b200: %s failed: %s (%s:%d)\n", #call,                  \
                    cudaGetErrorString(ac_err_), __FILE__, __LINE__);                         \
            return AC_FAILURE;                                                                \
        }                                                                                     \
    } while (0)

/* Geometry of one mesh: interior n, allocated m = n + 2*NGHOST, x fastest. */
struct Geom {
    int nx, ny, nz;
    int mx, my, mz;
    long long mxy;   /* mx*my */
    long long cells; /* mx*my*mz */
};

/* Physics constants of the RHS, precomputed on the host in double.  The
 * names follow the reference's run_const params
 * (acc-runtime/samples/mhd_modular/mhdsolver.ac:230-251). */
struct PhysConst {
    double nu, eta, zeta;
    double inv_mu0;       /* 1/mu0 */
    double eta_mu0;       /* eta*mu0 */
    double cs2_sound;     /* cs^2 */
    double gamma, gamma_m1, inv_cp, gamma_inv_cp;
    double lnrho0;
    double inv_exp_lnT0;  /* exp(-lnT0) */
    double K;             /* K_heatcond */
};

/* Stencil coefficients with the grid spacing folded in (6th order). */
struct StencilCoef {
    double d1[3][3];  /* [axis][k-1] = c_k / ds_axis, c = (3/4, -3/20, 1/60) */
    double d2[3][4];  /* [axis][k]   = d_k / ds_axis^2, d = (-49/18, 3/2, -3/20, 1/90) */
    double mix[3][3]; /* [xy,xz,yz][k-1] = e_k / (ds_a ds_b), e = (270,-27,2)/720 */
};

/* Coefficients of one substep of the 2N RK3 scheme in single-pass form
 * (acc-runtime/stdlib/integrators.h:11-29):
 *   f_new = f + beta_s * (ab * (f - f_prev) + dt * rate),  ab = alpha_s / beta_{s-1}
 * with ab = 0 at s = 0 (f_prev is then not read). */
struct RkCoef {
    double beta;
    double ab;
    double dt;
    int step;
};

struct Fields64 {
    double* in[AC_NF];
    double* out[AC_NF];
};

/* Scratch of the reductions: per-block partials, a completion counter and
 * the device-side result. */
struct ReduceScratch {
    double* partials;      /* 2 doubles per block */
    unsigned int* counter; /* zero between calls */
    double* result;        /* 1 double */
    int max_blocks;
};

struct StepGraph {
    cudaGraphExec_t exec;
    double dt;
    const void* in0; /* in-buffer pointer of field 0 the graph was captured with */
    int valid;
};

struct device_s {
    CUtensorMap tmap[2]; /* 4-D (x, y, z, field) maps of in_block / out_block */
    int tmap_ok;
    int* err_flag;       /* device word set by kernels whose bounded waits gave up */
    int id;
    AcMeshInfo config;
    Geom geom;
    int precision;
    cudaStream_t streams[NUM_STREAMS];
    double* in_block;
    double* out_block;
    Fields64 f;
    ReduceScratch red;
    double* host_result; /* pinned */
    StepGraph graphs[NUM_STREAMS][2];
    int solve_variant; /* 0 = plain, 1 = tiled */
    unsigned long long launches;
};

/* ---- launchers (each returns the launch error, cudaSuccess on success) ---- */

cudaError_t ac_launch_periodic(const Geom& g, double* const* fields, const int nfields,
                               const Volume start, const Volume end, cudaStream_t stream,
                               unsigned long long* launches);

cudaError_t ac_launch_fill(double* ptr, const long long count, const double value,
                           cudaStream_t stream, unsigned long long* launches);

cudaError_t ac_launch_solve64(const Geom& g, const Fields64& f, const StencilCoef& sc,
                              const PhysConst& pc, const RkCoef& rk, const int variant,
                              cudaStream_t stream, unsigned long long* launches);

/* map: AcKernel of the reduction's map; op: AcReduceOp; fields: up to 4. */
cudaError_t ac_launch_reduce(const Geom& g, const double* const* fields, const int nfields,
                             const int map, const int op, const ReduceScratch& scratch,
                             cudaStream_t stream, unsigned long long* launches);

int ac_reduce_blocks(const Geom& g);

bool ac_tiled_supported(const Geom& g);
cudaError_t ac_solve_tiled_init();
bool ac_make_tensor_map64(void* map_out, double* base, const Geom& g);
cudaError_t ac_launch_solve64_tiled(const Geom& g, const void* tmap_in, const Fields64& f,
                                    const StencilCoef& sc, const PhysConst& pc, const RkCoef& rk,
                                    int* err, cudaStream_t stream, unsigned long long* launches);

/* Host-side setup helpers (device.cu). */
void ac_make_stencil(const AcMeshInfo& info, StencilCoef* sc);
void ac_make_phys(const AcMeshInfo& info, PhysConst* pc);
Geom ac_make_geom(const AcMeshInfo& info);
