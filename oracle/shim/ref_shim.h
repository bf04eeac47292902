/*
 * Test infrastructure only: a hand-written stand-in for the DSL-generated headers
 * (user_defines.h, builtin_enums.h, the generated AcMeshInfo body, ...) that
 * Astaroth's host model files include.  It lets g++ compile the reference's own
 * src/utils/{modelsolver,memory,modelreduce,verification}.cc unchanged, for the
 * single configuration this project implements:
 *
 *   8 fields (lnrho, uux, uuy, uuz, ax, ay, az, entropy), declaration order of
 *   acc-runtime/samples/mhd_modular/mhdsolver.ac:125,136,140;
 *   LENTROPY=1, LMAGNETIC=1, LUPWD=0, LBFIELD=0, LFORCING=0, STENCIL_ORDER=6.
 *
 * Nothing here is a copy of a reference header: only the names and the meaning
 * of the symbols the four model files use are kept, so that they compile.
 * The product library never includes this file.
 */
#pragma once

#include <float.h>
#include <math.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>

#ifdef __cplusplus
#include <cmath>
using std::isinf;
using std::isnan;
#endif

/* ---- build switches (hostdefines of the MHD module) ---- */
#define AC_DOUBLE_PRECISION (1)
#define STENCIL_ORDER (6)
#define NGHOST (3)
#define LDENSITY (1)
#define LHYDRO (1)
#define LMAGNETIC (1)
#define LENTROPY (1)
#define LTEMPERATURE (0)
#ifndef LUPWD /* the upwinding variant of the model is built with -DLUPWD=1 */
#define LUPWD (0)
#endif
#define LBFIELD (0)
#ifndef LFORCING /* the forcing variant of the model is built with -DLFORCING=1 */
#define LFORCING (0)
#endif
#define LSHOCK (0)
#define AC_LAGRANGIAN_GRID (0)
#define AC_VERBOSE (0)
#define AC_INTEGRATION_ENABLED (1)
#define AC_MAPPING_FUNCTIONS_INCLUDED (1)

#ifndef __device__
#define __device__
#endif
#define UNUSED __attribute__((unused))

#define AC_GRN ""
#define AC_RED ""
#define AC_COL_RESET ""

typedef double AcReal;
#define AC_REAL_EPSILON (DBL_EPSILON)

typedef struct { AcReal x, y, z; } AcReal3;
#ifndef INT3_DEFINED
typedef struct { int x, y, z; } int3;
#define INT3_DEFINED
#endif
typedef struct { size_t x, y, z; } Volume;

typedef enum { AC_SUCCESS = 0, AC_FAILURE = 1, AC_NOT_ALLOCATED = 2 } AcResult;

/* ---- fields ---- */
typedef enum {
    VTXBUF_LNRHO = 0,
    VTXBUF_UUX,
    VTXBUF_UUY,
    VTXBUF_UUZ,
    VTXBUF_AX,
    VTXBUF_AY,
    VTXBUF_AZ,
    VTXBUF_ENTROPY,
    NUM_VTXBUF_HANDLES
} VertexBufferHandle;
#define NUM_FIELDS (NUM_VTXBUF_HANDLES)
#define NUM_ALL_FIELDS (NUM_VTXBUF_HANDLES)
typedef VertexBufferHandle Field;
typedef struct { Field x, y; } Field2;
typedef struct { Field x, y, z; } Field3;

static const bool vtxbuf_is_communicated[NUM_VTXBUF_HANDLES] UNUSED = {1, 1, 1, 1, 1, 1, 1, 1};
static const char* vtxbuf_names[NUM_VTXBUF_HANDLES] UNUSED = {
    "VTXBUF_LNRHO", "VTXBUF_UUX", "VTXBUF_UUY", "VTXBUF_UUZ",
    "VTXBUF_AX",    "VTXBUF_AY",  "VTXBUF_AZ",  "VTXBUF_ENTROPY"};
static const char* field_names[NUM_VTXBUF_HANDLES] UNUSED = {
    "VTXBUF_LNRHO", "VTXBUF_UUX", "VTXBUF_UUY", "VTXBUF_UUZ",
    "VTXBUF_AX",    "VTXBUF_AY",  "VTXBUF_AZ",  "VTXBUF_ENTROPY"};

/* ---- parameters used by the model files ---- */
typedef enum {
    AC_nu_visc = 0,
    AC_eta,
    AC_cs_sound,
    AC_gamma,
    AC_cp_sound,
    AC_lnrho0,
    AC_lnT0,
    AC_mu0,
    AC_zeta,
    AC_K_heatcond,
    /* used by the forcing of the LFORCING=1 build (modelsolver.cc:1031-1076) */
    AC_cs2_sound,
    AC_forcing_magnitude,
    AC_forcing_phase,
    AC_k_forcex,
    AC_k_forcey,
    AC_k_forcez,
    AC_ff_hel_rex,
    AC_ff_hel_rey,
    AC_ff_hel_rez,
    AC_ff_hel_imx,
    AC_ff_hel_imy,
    AC_ff_hel_imz,
    AC_kaver,
    NUM_REAL_PARAMS
} AcRealParam;
typedef enum { AC_ds = 0, NUM_REAL3_PARAMS } AcReal3Param;
typedef enum {
    AC_nmin = 0,
    AC_ngrid,
    AC_ngrid_max,
    AC_nlocal,
    AC_nlocal_max,
    AC_mlocal,
    AC_mgrid,
    AC_reduction_tile_dimensions,
    NUM_INT3_PARAMS
} AcInt3Param;
typedef enum { AC_dummy_int = 0, NUM_INT_PARAMS } AcIntParam;
typedef struct { int xy, xz, yz, xyz; } AcProducts;
typedef enum { AC_ngrid_products = 0 } AcProductsParam;

typedef struct AcMeshInfo {
    int int_params[NUM_INT_PARAMS];
    int3 int3_params[NUM_INT3_PARAMS];
    AcReal real_params[NUM_REAL_PARAMS];
    AcReal3 real3_params[NUM_REAL3_PARAMS];
    AcProducts ngrid_products;
#ifdef __cplusplus
    int& operator[](AcIntParam p) { return int_params[p]; }
    int operator[](AcIntParam p) const { return int_params[p]; }
    int3& operator[](AcInt3Param p) { return int3_params[p]; }
    int3 operator[](AcInt3Param p) const { return int3_params[p]; }
    AcReal& operator[](AcRealParam p) { return real_params[p]; }
    AcReal operator[](AcRealParam p) const { return real_params[p]; }
    AcReal3& operator[](AcReal3Param p) { return real3_params[p]; }
    AcReal3 operator[](AcReal3Param p) const { return real3_params[p]; }
    AcProducts operator[](AcProductsParam) const { return ngrid_products; }
#endif
} AcMeshInfo;

typedef struct {
    AcReal* vertex_buffer[NUM_VTXBUF_HANDLES];
    AcMeshInfo info;
} AcMesh;

/* ---- reductions ---- */
typedef enum AcReduceOp {
    AC_REDUCE_OP_NO_REDUCE,
    AC_REDUCE_OP_MIN,
    AC_REDUCE_OP_MAX,
    AC_REDUCE_OP_SUM,
} AcReduceOp;
typedef enum { AC_NO_REDUCE_POST_PROCESSING = 0, AC_RMS = 1 } AcReductionPostProcessingOp;
typedef enum {
    AC_NULL_KERNEL = 0,
    AC_MAP_VTXBUF,
    AC_MAP_VTXBUF_SQUARE,
    AC_MAP_VTXBUF_EXP_SQUARE,
    AC_MAP_VTXBUF3_NORM,
    AC_MAP_VTXBUF3_SQUARE,
    AC_MAP_VTXBUF3_EXP_SQUARE,
    AC_MAP_VTXBUF4_ALFVEN_NORM,
    AC_MAP_VTXBUF4_ALFVEN_SQUARE,
} AcKernel;
typedef struct {
    AcReduceOp reduce_op;
    AcReductionPostProcessingOp post_processing_op;
    AcKernel map_vtxbuf_single;
    AcKernel map_vtxbuf_vec;
    AcKernel map_vtxbuf_vec_scal;
    const char* name;
} AcReduction;

/* ---- verification record ---- */
typedef struct {
    AcReal model;
    AcReal candidate;
    long double abs_error;
    long double ulp_error;
    long double rel_error;
    AcReal maximum_magnitude;
    AcReal minimum_magnitude;
    int x;
    int y;
    int z;
} Error;

typedef Volume size3_t;
typedef struct {
    size3_t n0, n1;
    size3_t m0, m1;
    size3_t nn;
    size3_t reduction_tile;
} AcMeshDims;

/* ---- error macros (abort on failure, as the reference's ERRCHK_ALWAYS) ---- */
#define ERRCHK_ALWAYS(expr)                                                           \
    do {                                                                              \
        if (!(expr)) {                                                                \
            fprintf(stderr, "ref_shim: check failed: %s (%s:%d)\n", #expr, __FILE__, \
                    __LINE__);                                                        \
            abort();                                                                  \
        }                                                                             \
    } while (0)
#define ERRCHK(expr) ERRCHK_ALWAYS(expr)
#define ERROR(str)                                                                    \
    do {                                                                              \
        fprintf(stderr, "ref_shim: error: %s (%s:%d)\n", str, __FILE__, __LINE__);   \
        abort();                                                                      \
    } while (0)
#define WARNING(str) fprintf(stderr, "ref_shim: warning: %s\n", str)

/* ---- index helpers ---- */
static inline size_t UNUSED as_size_t(const long long v) { return (size_t)v; }

static inline Volume UNUSED
shim_vol(const int3 v)
{
    Volume r;
    r.x = (size_t)v.x;
    r.y = (size_t)v.y;
    r.z = (size_t)v.z;
    return r;
}
static inline Volume UNUSED acGetLocalNN(const AcMeshInfo info) { return shim_vol(info.int3_params[AC_nlocal]); }
static inline Volume UNUSED acGetLocalMM(const AcMeshInfo info) { return shim_vol(info.int3_params[AC_mlocal]); }
static inline Volume UNUSED acGetGridNN(const AcMeshInfo info) { return shim_vol(info.int3_params[AC_ngrid]); }
static inline Volume UNUSED acGetGridMM(const AcMeshInfo info) { return shim_vol(info.int3_params[AC_mgrid]); }
static inline Volume UNUSED acGetMinNN(const AcMeshInfo info) { return shim_vol(info.int3_params[AC_nmin]); }
static inline Volume UNUSED acGetMaxNN(const AcMeshInfo info) { return shim_vol(info.int3_params[AC_nlocal_max]); }
static inline Volume UNUSED acGetGridMaxNN(const AcMeshInfo info) { return shim_vol(info.int3_params[AC_ngrid_max]); }

static inline size_t UNUSED
acVertexBufferSize(const AcMeshInfo info)
{
    const Volume mm = acGetLocalMM(info);
    return mm.x * mm.y * mm.z;
}
static inline size_t UNUSED
acGridVertexBufferSize(const AcMeshInfo info)
{
    const Volume mm = acGetGridMM(info);
    return mm.x * mm.y * mm.z;
}
static inline size_t UNUSED
acGridVertexBufferIdx(const int i, const int j, const int k, const AcMeshInfo info)
{
    const int3 mm = info.int3_params[AC_mgrid];
    return (size_t)i + (size_t)mm.x * (size_t)j + (size_t)mm.x * (size_t)mm.y * (size_t)k;
}
static inline size_t UNUSED
acVertexBufferIdx(const int i, const int j, const int k, const AcMeshInfo info)
{
    const int3 mm = info.int3_params[AC_mlocal];
    return (size_t)i + (size_t)mm.x * (size_t)j + (size_t)mm.x * (size_t)mm.y * (size_t)k;
}
static inline AcMeshDims UNUSED
acGetMeshDims(const AcMeshInfo info)
{
    AcMeshDims d;
    d.n0 = acGetMinNN(info);
    d.n1 = acGetMaxNN(info);
    d.m0.x = d.m0.y = d.m0.z = 0;
    d.m1 = acGetLocalMM(info);
    d.nn = acGetLocalNN(info);
    d.reduction_tile = d.nn;
    return d;
}
static inline AcMeshDims UNUSED
acGetGridMeshDims(const AcMeshInfo info)
{
    AcMeshDims d;
    d.n0 = acGetMinNN(info);
    d.n1 = acGetGridMaxNN(info);
    d.m0.x = d.m0.y = d.m0.z = 0;
    d.m1 = acGetGridMM(info);
    d.nn = acGetGridNN(info);
    d.reduction_tile = d.nn;
    return d;
}

#ifdef __cplusplus
extern "C" {
#endif
/* Implemented by oracle/ref_driver.cc (project code, not the reference). */
AcResult acHostGridMeshCreate(const AcMeshInfo info, AcMesh* mesh);
AcResult acHostMeshDestroy(AcMesh* mesh);
#ifdef __cplusplus
}
#endif

/* Declarations of the reference functions compiled from the model files. */
AcResult acHostMeshApplyPeriodicBounds(AcMesh* mesh);
AcResult acHostIntegrateStep(AcMesh mesh, const AcReal dt);
AcResult acHostMeshWriteToFile(const AcMesh mesh, const size_t id);
AcResult acHostMeshReadFromFile(const size_t id, AcMesh* mesh);
AcReal acHostReduceScal(const AcMesh mesh, const AcReduction reduction, const VertexBufferHandle a);
AcReal acHostReduceVec(const AcMesh mesh, const AcReduction reduction, const VertexBufferHandle a,
                       const VertexBufferHandle b, const VertexBufferHandle c);
AcReal acHostReduceVecScal(const AcMesh mesh, const AcReduction reduction,
                           const VertexBufferHandle a, const VertexBufferHandle b,
                           const VertexBufferHandle c, const VertexBufferHandle d);
Error acGetError(const AcReal model, const AcReal candidate);
AcResult acVerifyMeshWithMaximumError(const char* label, const AcMesh model,
                                      const AcMesh candidate, const long double max_ulp_error);
