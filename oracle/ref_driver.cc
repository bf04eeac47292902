/*
 * Test infrastructure only (the oracle): a C entry layer over the reference's own
 * host model files, compiled unchanged from the reference tree against
 * oracle/shim/.  Built into oracle/_ref/libastaroth_ref.so by oracle/Makefile;
 * the tests call it through ctypes to pin the project's C restatement
 * (oracle/astaroth_oracle.c) and to produce golden vectors.
 *
 * Reference functions reached from here:
 *   acHostIntegrateStep            src/utils/modelsolver.cc:1214-1272
 *   acHostMeshApplyPeriodicBounds  src/utils/memory.cc:76-149
 *   acHostReduceScal/Vec/VecScal   src/utils/modelreduce.cc:108-340
 *   acGetError                     src/utils/verification.cc:45-83
 *   acHostMeshWriteToFile/ReadFromFile  src/utils/memory.cc:182-247 (snapshot format)
 *   helical_forcing_special_vector src/utils/astaroth_forcing.cc:158-216 (LFORCING build)
 * The two mesh helpers below stand in for src/core/astaroth.cc:324-335,425-431.
 */
#include <stdlib.h>
#include <string.h>

#include "ref_shim.h"
#include "oracle_params.h"

extern "C" AcResult
acHostGridMeshCreate(const AcMeshInfo info, AcMesh* mesh)
{
    mesh->info = info;
    const size_t n = acGridVertexBufferSize(info);
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w) {
        mesh->vertex_buffer[w] = (AcReal*)calloc(n, sizeof(AcReal));
        ERRCHK_ALWAYS(mesh->vertex_buffer[w]);
    }
    return AC_SUCCESS;
}

extern "C" AcResult
acHostMeshDestroy(AcMesh* mesh)
{
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w) {
        free(mesh->vertex_buffer[w]);
        mesh->vertex_buffer[w] = NULL;
    }
    return AC_SUCCESS;
}

/* The reduction types of stdlib/reduction.h:1-8, restated as a table. */
static const AcReduction ref_rtypes[] = {
    {AC_REDUCE_OP_MAX, AC_NO_REDUCE_POST_PROCESSING, AC_MAP_VTXBUF, AC_MAP_VTXBUF3_NORM,
     AC_NULL_KERNEL, "RTYPE_MAX"},
    {AC_REDUCE_OP_MIN, AC_NO_REDUCE_POST_PROCESSING, AC_MAP_VTXBUF, AC_MAP_VTXBUF3_NORM,
     AC_NULL_KERNEL, "RTYPE_MIN"},
    {AC_REDUCE_OP_SUM, AC_NO_REDUCE_POST_PROCESSING, AC_MAP_VTXBUF, AC_MAP_VTXBUF3_NORM,
     AC_NULL_KERNEL, "RTYPE_SUM"},
    {AC_REDUCE_OP_SUM, AC_RMS, AC_MAP_VTXBUF_SQUARE, AC_MAP_VTXBUF3_SQUARE, AC_NULL_KERNEL,
     "RTYPE_RMS"},
    {AC_REDUCE_OP_SUM, AC_RMS, AC_MAP_VTXBUF_EXP_SQUARE, AC_MAP_VTXBUF3_EXP_SQUARE,
     AC_NULL_KERNEL, "RTYPE_RMS_EXP"},
    {AC_REDUCE_OP_MAX, AC_NO_REDUCE_POST_PROCESSING, AC_NULL_KERNEL, AC_NULL_KERNEL,
     AC_MAP_VTXBUF4_ALFVEN_NORM, "RTYPE_ALFVEN_MAX"},
    {AC_REDUCE_OP_MIN, AC_NO_REDUCE_POST_PROCESSING, AC_NULL_KERNEL, AC_NULL_KERNEL,
     AC_MAP_VTXBUF4_ALFVEN_NORM, "RTYPE_ALFVEN_MIN"},
    {AC_REDUCE_OP_SUM, AC_RMS, AC_NULL_KERNEL, AC_NULL_KERNEL, AC_MAP_VTXBUF4_ALFVEN_SQUARE,
     "RTYPE_ALFVEN_RMS"},
};

static AcMesh
make_mesh(double* const* fields, const int nx, const int ny, const int nz, const OracleParams* p)
{
    AcMesh mesh;
    memset(&mesh, 0, sizeof(mesh));
    AcMeshInfo& info = mesh.info;
    const int3 n     = {nx, ny, nz};
    const int3 nmin  = {NGHOST, NGHOST, NGHOST};
    const int3 nmax  = {nx + NGHOST, ny + NGHOST, nz + NGHOST};
    const int3 mm    = {nx + 2 * NGHOST, ny + 2 * NGHOST, nz + 2 * NGHOST};
    info[AC_nmin]    = nmin;
    info[AC_ngrid]   = n;
    info[AC_nlocal]  = n;
    info[AC_ngrid_max]  = nmax;
    info[AC_nlocal_max] = nmax;
    info[AC_mlocal]     = mm;
    info[AC_mgrid]      = mm;
    info[AC_reduction_tile_dimensions] = n;
    info.ngrid_products.xy  = nx * ny;
    info.ngrid_products.xz  = nx * nz;
    info.ngrid_products.yz  = ny * nz;
    info.ngrid_products.xyz = nx * ny * nz;
    if (p) {
        info[AC_ds]         = (AcReal3){p->ds[0], p->ds[1], p->ds[2]};
        info[AC_nu_visc]    = p->nu_visc;
        info[AC_eta]        = p->eta;
        info[AC_cs_sound]   = p->cs_sound;
        info[AC_gamma]      = p->gamma;
        info[AC_cp_sound]   = p->cp_sound;
        info[AC_lnrho0]     = p->lnrho0;
        info[AC_lnT0]       = p->lnT0;
        info[AC_mu0]        = p->mu0;
        info[AC_zeta]       = p->zeta;
        info[AC_K_heatcond] = p->K_heatcond;
        info[AC_cs2_sound]  = p->cs_sound * p->cs_sound;
        info[AC_forcing_magnitude] = p->f_magnitude;
        info[AC_forcing_phase]     = p->f_phase;
        info[AC_kaver]             = p->f_kaver;
        info[AC_k_forcex]          = p->f_k[0];
        info[AC_k_forcey]          = p->f_k[1];
        info[AC_k_forcez]          = p->f_k[2];
        info[AC_ff_hel_rex]        = p->f_re[0];
        info[AC_ff_hel_rey]        = p->f_re[1];
        info[AC_ff_hel_rez]        = p->f_re[2];
        info[AC_ff_hel_imx]        = p->f_im[0];
        info[AC_ff_hel_imy]        = p->f_im[1];
        info[AC_ff_hel_imz]        = p->f_im[2];
    }
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w)
        mesh.vertex_buffer[w] = fields[w];
    return mesh;
}

extern "C" int
ref_integrate(double* const* fields, const int nx, const int ny, const int nz,
              const OracleParams* p, const double dt, const int nsteps)
{
    AcMesh mesh = make_mesh(fields, nx, ny, nz, p);
    for (int s = 0; s < nsteps; ++s)
        if (acHostIntegrateStep(mesh, dt) != AC_SUCCESS)
            return 1;
    return 0;
}

extern "C" int
ref_periodic_bounds(double* const* fields, const int nx, const int ny, const int nz)
{
    AcMesh mesh = make_mesh(fields, nx, ny, nz, NULL);
    return acHostMeshApplyPeriodicBounds(&mesh) == AC_SUCCESS ? 0 : 1;
}

/* kind: 1 = scalar (a), 3 = vector (a,b,c), 4 = vector+scalar (a,b,c,d). */
extern "C" double
ref_reduce(double* const* fields, const int nx, const int ny, const int nz, const int kind,
           const int rtype, const int a, const int b, const int c, const int d)
{
    AcMesh mesh = make_mesh(fields, nx, ny, nz, NULL);
    const AcReduction r = ref_rtypes[rtype];
    if (kind == 1)
        return acHostReduceScal(mesh, r, (VertexBufferHandle)a);
    if (kind == 3)
        return acHostReduceVec(mesh, r, (VertexBufferHandle)a, (VertexBufferHandle)b,
                               (VertexBufferHandle)c);
    return acHostReduceVecScal(mesh, r, (VertexBufferHandle)a, (VertexBufferHandle)b,
                               (VertexBufferHandle)c, (VertexBufferHandle)d);
}

/* Per-point error record of the reference (ulp, abs, rel) for one pair of values. */
extern "C" void
ref_get_error(const double model, const double candidate, long double* out3)
{
    const Error e = acGetError(model, candidate);
    out3[0]       = e.ulp_error;
    out3[1]       = e.abs_error;
    out3[2]       = e.rel_error;
}

/* acVerifyMeshWithMaximumError over all fields; returns 0 when every field passes. */
extern "C" int
ref_verify(double* const* model, double* const* candidate, const int nx, const int ny,
           const int nz, const double max_ulp_error)
{
    AcMesh m = make_mesh(model, nx, ny, nz, NULL);
    AcMesh c = make_mesh(candidate, nx, ny, nz, NULL);
    return acVerifyMeshWithMaximumError("oracle", m, c, (long double)max_ulp_error) ==
                   AC_SUCCESS
               ? 0
               : 1;
}

/* The reference's snapshot writer and reader: data-format.csv and
 * <field>-<id>.dat in the current directory.  Returns 0 on success. */
extern "C" int
ref_write_to_file(double* const* fields, const int nx, const int ny, const int nz,
                  const unsigned long id)
{
    AcMesh mesh = make_mesh(fields, nx, ny, nz, NULL);
    return acHostMeshWriteToFile(mesh, (size_t)id) == AC_SUCCESS ? 0 : 1;
}

extern "C" int
ref_read_from_file(double* const* fields, const int nx, const int ny, const int nz,
                   const unsigned long id)
{
    AcMesh mesh = make_mesh(fields, nx, ny, nz, NULL);
    return acHostMeshReadFromFile((size_t)id, &mesh) == AC_SUCCESS ? 0 : 1;
}

#if LFORCING
/* src/utils/astaroth_forcing.cc:158-216, compiled into the LFORCING=1 build */
void helical_forcing_special_vector(AcReal3* ff_hel_re, AcReal3* ff_hel_im, const AcReal3 k_force,
                                    const AcReal3 e_force, const AcReal relhel);

/* ff_hel_re and ff_hel_im of wave vector k and basis vector e */
extern "C" void
ref_forcing_special_vector(const double* k, const double* e, const double relhel, double* re,
                           double* im)
{
    AcReal3 r, i;
    helical_forcing_special_vector(&r, &i, (AcReal3){k[0], k[1], k[2]}, (AcReal3){e[0], e[1], e[2]},
                                   relhel);
    re[0] = r.x;
    re[1] = r.y;
    re[2] = r.z;
    im[0] = i.x;
    im[1] = i.y;
    im[2] = i.z;
}
#endif

