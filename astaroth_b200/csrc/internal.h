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

/* Geometry of one mesh: interior n, allocated m = n + 2*NGHOST per axis, x
 * fastest.  Rows are `px` elements apart (px >= mx); FP64 meshes use the host
 * layout (px = mx), FP32 meshes round px up to a multiple of 4 so every row
 * starts on a 16-byte boundary (a TMA requirement). */
struct Geom {
    int nx, ny, nz;
    int mx, my, mz;
    int px;          /* row pitch in elements */
    long long pxy;   /* px*my: plane pitch in elements */
    long long cells; /* px*my*mz: elements per field */
};

__host__ __device__ inline long long
geom_idx(const Geom& g, const int i, const int j, const int k)
{
    return (long long)i + (long long)j * g.px + (long long)k * g.pxy;
}

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
    int upwind;           /* AC_upwind: the LUPWD terms (selects the kernel variant) */
    int debug_skip_load;  /* acDeviceDebugSkipPlaneLoad: the fault-path test of the tiled kernels */
    int cfl_sum;          /* AC_additive_timestep: substep 2 also forms the additive CFL sum */
    int zlo, zhi;         /* the interior z planes [zlo, zhi) this launch solves */
    /* helical forcing of this launch (substep 2 only; forcing = 0 otherwise):
     * u += scale (re cos(a + phase) - im sin(a + phase)), a = sum_d f_k[d] idx_d
     * with idx the interior cell index (mhdsolver.ac:286-331) */
    int forcing;
    double f_k[3];        /* k_force[d] 2 pi / ngrid[d] */
    double f_re[3], f_im[3];
    double f_cos_phase, f_sin_phase;
    double f_scale;       /* sqrt(dt) cs magnitude sqrt(kaver cs) */
};

/* Stencil coefficients with the grid spacing folded in (6th order). */
template <typename T>
struct StencilT {
    T d1[3][3];  /* [axis][k-1] = c_k / ds_axis, c = (3/4, -3/20, 1/60) */
    T d2[3][4];  /* [axis][k]   = d_k / ds_axis^2, d = (-49/18, 3/2, -3/20, 1/90) */
    T mix[3][3]; /* [xy,xz,yz][k-1] = e_k / (ds_a ds_b), e = (270,-27,2)/720 */
    T up[3][4];  /* [axis][k] = u_k / ds_axis, u = (-20, 15, -6, 1)/60: upwinding */
};
typedef StencilT<double> StencilCoef;

template <typename T>
inline StencilT<T>
stencil_cast(const StencilCoef& s)
{
    StencilT<T> o;
    for (int a = 0; a < 3; ++a) {
        for (int k = 0; k < 3; ++k) {
            o.d1[a][k]  = (T)s.d1[a][k];
            o.mix[a][k] = (T)s.mix[a][k];
        }
        for (int k = 0; k < 4; ++k) {
            o.d2[a][k] = (T)s.d2[a][k];
            o.up[a][k] = (T)s.up[a][k];
        }
    }
    return o;
}

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

/* Field arrays of one substep.  FP64: `in`/`out` hold the values (lo unused).
 * FP32 compensated: the value is hi + lo with |lo| <= ulp(hi)/2; stencils read
 * hi, the RK3 update is carried out on the (hi, lo) pair. */
template <typename T>
struct FieldsT {
    const T* in[AC_NF];
    const T* in_lo[AC_NF];
    T* out[AC_NF];
    T* out_lo[AC_NF];
};
typedef FieldsT<double> Fields64;
typedef FieldsT<float> Fields32;

/* Scratch of the reductions: per-block partials, a completion counter and
 * the device-side result. */
struct ReduceScratch {
    double* partials;        /* 2 doubles per block */
    unsigned int* counter;   /* zero between calls */
    double* result;          /* 1 double, then the non-finite flag (result + 1) */
    unsigned int* nonfinite; /* the low word of result[1]: 1 when a mapped value was NaN or
                              * infinite; cleared before each call (may be null) */
    int max_blocks;
};

/* Adjoint state of one device (FP64 only): adjoints of f and w per field, the
 * 46 derivative-slot adjoints mu, and the parameter adjoints (nu, eta). */
#define AC_MU_COUNT 46
struct AdjointFields {
    const double* f[AC_NF];
    double* lf[AC_NF];
    double* lw[AC_NF];
    double* mu[AC_MU_COUNT];
};

struct StepGraph {
    cudaGraphExec_t exec;
    double dt;
    int valid;
};

/* The two buffers of every field: block b holds all 8 fields of buffer b
 * (field q at offset q*cells).  in_idx[q] says which block is field q's
 * in-buffer; swaps flip it. */
struct device_s {
    CUtensorMap tmap[2]; /* 4-D (x, y, z, field) maps of the value (hi) array of each block */
    int tmap_ok;
    int* err_flag;       /* device word set by kernels whose bounded waits gave up */
    /* CFL maxima of the last substep 2 (bit patterns of non-negative doubles):
     * [0] max |u|, [1] max Alfven speed |B|/sqrt(rho), [2] max |u| + sqrt(cs^2 + vA^2) */
    unsigned long long* cfl;
    int id;
    AcMeshInfo config;
    Geom geom;
    int precision;       /* 0 FP64, 1 FP32 compensated */
    cudaStream_t streams[NUM_STREAMS];
    void* hi[2];         /* double* (FP64) or float* (FP32) value arrays per block */
    float* lo[2];        /* FP32 compensation arrays per block (NULL for FP64) */
    double* staging;     /* FP32: one field of doubles for host transfers */
    int in_idx[AC_NF];
    ReduceScratch red;
    double* host_result; /* pinned */
    StepGraph graphs[NUM_STREAMS][2];
    int solve_variant;   /* 0 = plain, else the tiled kernel AC_SOLVE_TILED_* */
    int debug_skip_load; /* acDeviceDebugSkipPlaneLoad */
    int last_nonfinite;  /* the last reduction met a NaN or infinite mapped value */
    /* planes of substep 2 solved since the CFL maxima were last cleared (a
     * substep solved in z boxes clears them once, at its first box) */
    int cfl_cover;
    /* adjoint buffers, allocated by the first acDeviceLoadAdjoint */
    double* adj_lf;      /* 8 fields */
    double* adj_lw;      /* 8 fields */
    double* adj_mu;      /* AC_MU_COUNT fields */
    double* adj_pgrad;   /* 2 values: d/d nu, d/d eta */
    double* bfield;      /* AC_lbfield: B = curl A, 3 arrays of mx*my*mz doubles */
    double* adj_tape;    /* substep input states of a recomputed segment, 8 fields each */
    double* adj_state;   /* FP32 compensated: the joined in-buffers of a per-substep adjoint */
    int adj_tape_states; /* states the tape holds */
    /* graphs of acDeviceAdjointTapeForward, one per in-block, each kept for
     * the next call with the same steps, dt and stream */
    cudaGraphExec_t tape_exec[2];
    int tape_valid[2], tape_steps[2], tape_stream[2];
    double tape_dt[2];
    /* acDeviceSetOutput values; bit p of out_set says output p holds one, until
     * the next launch that recomputes the CFL words */
    double outputs[NUM_REAL_OUTPUTS];
    unsigned out_set;
    /* acDeviceLoadMeshStaged: a device copy of a whole host mesh (8 fields of
     * mx*my*mz doubles, host layout), allocated on first use; stage_loaded is
     * recorded after its copy from the host, stage_read after the commit has
     * read it */
    double* stage;
    cudaEvent_t stage_loaded, stage_read;
    unsigned long long launches;
};

/* ---- launchers (each returns the launch error, cudaSuccess on success) ---- */

/* Periodic halo fill of n arrays of element type T (double or float). */
template <typename T>
cudaError_t ac_launch_periodic(const Geom& g, T* const* arrays, const int n, const Volume start,
                               const Volume end, cudaStream_t stream,
                               unsigned long long* launches);

cudaError_t ac_launch_fill(double* ptr, const long long count, const double value,
                           cudaStream_t stream, unsigned long long* launches);
/* dst = src for `count` doubles on the device (a vectorised copy kernel when
 * both are 16-byte aligned and count is even, else cudaMemcpyAsync) */
/* Pack (or unpack) bytes starting at offset_bytes of each of narrays (<= 16)
 * arrays into (from) buffer + a * bytes, one launch; everything 8-byte aligned. */
cudaError_t ac_launch_planes(void* const* arrays, const int narrays, const long long offset_bytes,
                             const long long bytes, void* buffer, const bool pack,
                             cudaStream_t stream, unsigned long long* launches);
/* Pack (or unpack) the box [start, start + dims) of each of narrays (<= 16)
 * arrays of geometry g, elements of `elem` bytes (4 or 8), into (from) buffer,
 * array-major then z, y, x; one launch.  Boxes outside the padded mesh are
 * refused (cudaErrorInvalidValue). */
cudaError_t ac_launch_box(void* const* arrays, const int narrays, const size_t elem, const Geom& g,
                          const int3 start, const int3 dims, void* buffer, const bool pack,
                          cudaStream_t stream, unsigned long long* launches);
/* Host-layout linear range [first, first + count) of one field: doubles at
 * those indices of src/dst <-> (hi, lo) in the FP32 device layout. */
cudaError_t ac_launch_split_range(const Geom& g, const double* src, float* hi, float* lo,
                                  const long long first, const long long count,
                                  cudaStream_t stream, unsigned long long* launches);
cudaError_t ac_launch_join_range(const Geom& g, const float* hi, const float* lo, double* dst,
                                 const long long first, const long long count,
                                 cudaStream_t stream, unsigned long long* launches);
/* The box nn from in (offset in_offset in an in_volume array) to out. */
cudaError_t ac_launch_volume_copy(const double* in, const Volume in_offset,
                                  const Volume in_volume, double* out, const Volume out_offset,
                                  const Volume out_volume, const Volume nn, cudaStream_t stream,
                                  unsigned long long* launches);
cudaError_t ac_launch_copy(const double* src, double* dst, const long long count,
                           cudaStream_t stream, unsigned long long* launches);
/* FP32 compensated: hi/lo of `count` elements from a double value */
cudaError_t ac_launch_fill_comp(float* hi, float* lo, const long long count, const double value,
                                cudaStream_t stream, unsigned long long* launches);
/* FP32 compensated <-> double (host layout, row pitch mx) conversions of one field */
cudaError_t ac_launch_split(const Geom& g, const double* src, float* hi, float* lo,
                            cudaStream_t stream, unsigned long long* launches);
cudaError_t ac_launch_join(const Geom& g, const float* hi, const float* lo, double* dst,
                           cudaStream_t stream, unsigned long long* launches);

cudaError_t ac_launch_solve_plain64(const Geom& g, const Fields64& f, const StencilCoef& sc,
                                    const PhysConst& pc, const RkCoef& rk,
                                    unsigned long long* cfl, cudaStream_t stream,
                                    unsigned long long* launches);
cudaError_t ac_launch_solve_plain32(const Geom& g, const Fields32& f, const StencilCoef& sc,
                                    const PhysConst& pc, const RkCoef& rk,
                                    unsigned long long* cfl, cudaStream_t stream,
                                    unsigned long long* launches);

/* map: AcKernel of the reduction's map; op: AcReduceOp; up to 4 fields; lo
 * arrays are NULL for FP64 meshes. */
cudaError_t ac_launch_reduce(const Geom& g, const void* const* fields, const float* const* lo,
                             const int nfields, const int precision, const int map,
                             const int op, const ReduceScratch& scratch, cudaStream_t stream,
                             unsigned long long* launches);

int ac_reduce_blocks(const Geom& g);

/* Tiled substep kernels (solve_tiled.cu): the leading-plane kernel (in-plane
 * derivatives of plane z+3 kept in tensor memory until plane z is solved) and
 * the per-plane tap kernel.  AUTO takes the leading-plane kernel for z chunks
 * of 32 planes and more; _ALT is the leading-plane kernel with the group
 * exchange through shared memory instead of tensor memory.  Meshes with the
 * upwinding terms always take the per-plane tap kernel. */
enum {
    AC_SOLVE_TILED_AUTO     = 1,
    AC_SOLVE_TILED_TAPS     = 2,
    AC_SOLVE_TILED_LEAD     = 3,
    AC_SOLVE_TILED_LEAD_ALT = 4
};
bool ac_tiled_supported(const Geom& g, const int precision);
bool ac_make_tensor_map(void* map_out, void* base, const Geom& g, const int precision);
cudaError_t ac_solve_tiled_init(const int precision);
cudaError_t ac_launch_solve_tiled64(const Geom& g, const void* tmap_in, const Fields64& f,
                                    const StencilCoef& sc, const PhysConst& pc, const RkCoef& rk,
                                    int* err, unsigned long long* cfl, cudaStream_t stream,
                                    unsigned long long* launches, const int kernel);
cudaError_t ac_launch_solve_tiled32(const Geom& g, const void* tmap_in, const Fields32& f,
                                    const StencilCoef& sc, const PhysConst& pc, const RkCoef& rk,
                                    int* err, unsigned long long* cfl, cudaStream_t stream,
                                    unsigned long long* launches, const int kernel);

/* Helical forcing added to the three velocity arrays u (and their
 * compensation arrays lo in FP32) after substep 2 (forcing.cu). */
cudaError_t ac_launch_forcing(const Geom& g, void* const* u, float* const* lo, const int precision,
                              const PhysConst& pc, cudaStream_t stream,
                              unsigned long long* launches);

/* B = curl A of the A arrays a[3] (in-buffer, element type of the precision)
 * into the double arrays b[3] in the host layout (bfield.cu). */
cudaError_t ac_launch_bfield(const Geom& g, const void* const* a, double* const* b,
                             const int precision, const StencilCoef& sc, cudaStream_t stream,
                             unsigned long long* launches);

/* CFL maxima of the in-buffer (cfl.cu); zeroes the three words first. */
template <typename T>
cudaError_t ac_launch_cfl(const Geom& g, const FieldsT<T>& f, const StencilCoef& sc,
                          const double cs2_sound, unsigned long long* cfl, cudaStream_t stream,
                          unsigned long long* launches);

/* One adjoint substep (adjoint.cu): local reverse + halo fill of mu + gather. */
cudaError_t ac_launch_adjoint_substep(const Geom& g, const AdjointFields& a,
                                      const StencilCoef& sc, const PhysConst& pc,
                                      const double alpha, const double beta, const double dt,
                                      double* pgrad, cudaStream_t stream,
                                      unsigned long long* launches);

/* Host-side setup helpers (device.cu). */
void ac_make_stencil(const AcMeshInfo& info, StencilCoef* sc);
void ac_make_phys(const AcMeshInfo& info, PhysConst* pc);
Geom ac_make_geom(const AcMeshInfo& info, const int precision);
/* Coefficients of RK3 substep `step` (0, 1, 2) with timestep dt. */
RkCoef ac_rk_coef(const int step, const double dt);
