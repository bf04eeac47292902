/*
 * Host-side helpers of the astaroth_b200 C ABI: parameter derivation, the
 * default configuration, the `.conf` reader, host mesh allocation, seeded
 * initial conditions and the CFL timestep formula.  Plain C11, no CUDA.
 */
#include <ctype.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "astaroth_b200.h"

static int
valid_dims(const AcMeshInfo* info)
{
    const int3 n = info->int3_params[AC_ngrid];
    return n.x > 0 && n.y > 0 && n.z > 0;
}

/* Derived parameters; mirrors what acHostUpdateParams computes in
 * src/core/update_params/update_params.cc and acc-runtime/built-in/variables.h:1-200
 * for a single device (nlocal = ngrid, no multi-GPU offset). */
AcResult
acHostUpdateParams(AcMeshInfo* info)
{
    if (!info || !valid_dims(info))
        return AC_FAILURE;
    const int3 n = info->int3_params[AC_ngrid];
    int3 nl      = info->int3_params[AC_nlocal];
    if (nl.x <= 0 || nl.y <= 0 || nl.z <= 0)
        nl = n;
    info->int3_params[AC_nlocal] = nl;
    const int3 nmin              = {NGHOST, NGHOST, NGHOST};
    info->int3_params[AC_nmin]   = nmin;
    const int3 nlmax = {nl.x + NGHOST, nl.y + NGHOST, nl.z + NGHOST};
    const int3 ngmax = {n.x + NGHOST, n.y + NGHOST, n.z + NGHOST};
    const int3 ml    = {nl.x + 2 * NGHOST, nl.y + 2 * NGHOST, nl.z + 2 * NGHOST};
    const int3 mg    = {n.x + 2 * NGHOST, n.y + 2 * NGHOST, n.z + 2 * NGHOST};
    info->int3_params[AC_nlocal_max] = nlmax;
    info->int3_params[AC_ngrid_max]  = ngmax;
    info->int3_params[AC_mlocal]     = ml;
    info->int3_params[AC_mgrid]      = mg;

    const AcReal3 ds = info->real3_params[AC_ds];
    if (!(ds.x > 0) || !(ds.y > 0) || !(ds.z > 0))
        return AC_FAILURE;
    const AcReal3 inv  = {1.0 / ds.x, 1.0 / ds.y, 1.0 / ds.z};
    const AcReal3 inv2 = {inv.x * inv.x, inv.y * inv.y, inv.z * inv.z};
    const AcReal3 len  = {ds.x * n.x, ds.y * n.y, ds.z * n.z};
    info->real3_params[AC_inv_ds]   = inv;
    info->real3_params[AC_inv_ds_2] = inv2;
    info->real3_params[AC_len]      = len;
    const AcReal cs                 = info->real_params[AC_cs_sound];
    info->real_params[AC_cs2_sound] = cs * cs;
    AcReal dsmin                    = ds.x < ds.y ? ds.x : ds.y;
    dsmin                           = dsmin < ds.z ? dsmin : ds.z;
    info->real_params[AC_dsmin]     = dsmin;
    return AC_SUCCESS;
}

/* Defaults of config/astaroth.conf (:45-70) for the parameters this module
 * reads, on a periodic [0, 2 pi)^3 box. */
AcResult
acHostMeshInfoDefault(const int nx, const int ny, const int nz, AcMeshInfo* info)
{
    if (!info || nx <= 0 || ny <= 0 || nz <= 0)
        return AC_FAILURE;
    memset(info, 0, sizeof(*info));
    const int3 n                  = {nx, ny, nz};
    info->int3_params[AC_ngrid]   = n;
    info->int3_params[AC_nlocal]  = n;
    const double two_pi           = 6.283185307179586476925286766559;
    const AcReal3 ds              = {two_pi / nx, two_pi / ny, two_pi / nz};
    info->real3_params[AC_ds]     = ds;
    info->real_params[AC_nu_visc] = 2e-5;
    info->real_params[AC_cs_sound]  = 1.0;
    info->real_params[AC_zeta]      = 0.01;
    info->real_params[AC_eta]       = 5e-5;
    info->real_params[AC_mu0]       = 1.4;
    info->real_params[AC_chi]       = 0.0001;
    info->real_params[AC_cp_sound]  = 1.0;
    info->real_params[AC_gamma]     = 0.5;
    info->real_params[AC_lnT0]      = 1.2;
    info->real_params[AC_lnrho0]    = 1.3;
    info->real_params[AC_K_heatcond] = 1e-3;
    info->real_params[AC_cdt]       = 0.4;
    info->real_params[AC_cdtv]      = 0.3;
    /* forcing: config/astaroth.conf:58-61 */
    info->real_params[AC_relhel]            = 0.0;
    info->real_params[AC_forcing_magnitude] = 1e-5;
    info->real_params[AC_kmin]              = 0.8;
    info->real_params[AC_kmax]              = 1.2;
    info->real_params[AC_switch_forcing]    = 0.0;
    return acHostUpdateParams(info);
}

/* ---- `.conf` reader: `KEY = value` and `KEY = {a,b,c}`, line and block comments ---- */

typedef struct {
    const char* name;
    int kind; /* 0 int, 1 int3, 2 real, 3 real3 */
    int index;
} ParamName;

static const ParamName param_names[] = {
    {"AC_precision", 0, AC_precision},
    {"AC_additive_timestep", 0, AC_additive_timestep},
    {"AC_upwind", 0, AC_upwind},
    {"AC_lforcing", 0, AC_lforcing},
    {"AC_lbfield", 0, AC_lbfield},
    {"AC_ngrid", 1, AC_ngrid},
    {"AC_nlocal", 1, AC_nlocal},
    {"AC_nu_visc", 2, AC_nu_visc},
    {"AC_eta", 2, AC_eta},
    {"AC_cs_sound", 2, AC_cs_sound},
    {"AC_gamma", 2, AC_gamma},
    {"AC_cp_sound", 2, AC_cp_sound},
    {"AC_lnrho0", 2, AC_lnrho0},
    {"AC_lnT0", 2, AC_lnT0},
    {"AC_mu0", 2, AC_mu0},
    {"AC_zeta", 2, AC_zeta},
    {"AC_K_heatcond", 2, AC_K_heatcond},
    {"AC_cdt", 2, AC_cdt},
    {"AC_cdtv", 2, AC_cdtv},
    {"AC_chi", 2, AC_chi},
    {"AC_relhel", 2, AC_relhel},
    {"AC_forcing_magnitude", 2, AC_forcing_magnitude},
    {"AC_kmin", 2, AC_kmin},
    {"AC_kmax", 2, AC_kmax},
    {"AC_switch_forcing", 2, AC_switch_forcing},
    {"AC_ds", 3, AC_ds},
};

static char*
trim(char* s)
{
    while (*s && isspace((unsigned char)*s))
        ++s;
    char* e = s + strlen(s);
    while (e > s && isspace((unsigned char)e[-1]))
        *--e = '\0';
    return s;
}

static int
parse_bool_or_double(const char* v, double* out)
{
    if (!strcmp(v, "T") || !strcmp(v, "True") || !strcmp(v, "true")) {
        *out = 1;
        return 1;
    }
    if (!strcmp(v, "F") || !strcmp(v, "False") || !strcmp(v, "false")) {
        *out = 0;
        return 1;
    }
    char* end;
    *out = strtod(v, &end);
    return end != v;
}

AcResult
acLoadConfig(const char* path, AcMeshInfo* info)
{
    if (!path || !info)
        return AC_FAILURE;
    FILE* fp = fopen(path, "r");
    if (!fp)
        return AC_FAILURE;
    char line[4096];
    int in_block_comment = 0;
    while (fgets(line, sizeof(line), fp)) {
        char* s = line;
        if (in_block_comment) {
            char* e = strstr(s, "*/");
            if (!e)
                continue;
            in_block_comment = 0;
            s                = e + 2;
        }
        char* c = strstr(s, "/*");
        if (c) {
            char* e = strstr(c + 2, "*/");
            if (!e)
                in_block_comment = 1;
            *c = '\0';
        }
        c = strstr(s, "//");
        if (c)
            *c = '\0';
        char* eq = strchr(s, '=');
        if (!eq)
            continue;
        *eq       = '\0';
        char* key = trim(s);
        char* val = trim(eq + 1);
        for (size_t p = 0; p < sizeof(param_names) / sizeof(param_names[0]); ++p) {
            if (strcmp(key, param_names[p].name))
                continue;
            const ParamName* pn = &param_names[p];
            if (pn->kind == 1 || pn->kind == 3) {
                double v[3] = {0, 0, 0};
                char* q     = val;
                while (*q == '{' || isspace((unsigned char)*q))
                    ++q;
                for (int t = 0; t < 3; ++t) {
                    char* end;
                    v[t] = strtod(q, &end);
                    q    = end;
                    while (*q == ',' || isspace((unsigned char)*q))
                        ++q;
                }
                if (pn->kind == 1) {
                    const int3 iv = {(int)v[0], (int)v[1], (int)v[2]};
                    info->int3_params[pn->index] = iv;
                }
                else {
                    const AcReal3 rv = {v[0], v[1], v[2]};
                    info->real3_params[pn->index] = rv;
                }
            }
            else {
                double v;
                if (!parse_bool_or_double(val, &v))
                    break;
                if (pn->kind == 0)
                    info->int_params[pn->index] = (int)v;
                else
                    info->real_params[pn->index] = v;
            }
            break;
        }
    }
    fclose(fp);
    return acHostUpdateParams(info);
}

/* ---- host meshes ---- */

static size_t
mesh_cells(const AcMeshInfo* info)
{
    const int3 m = info->int3_params[AC_mlocal];
    return (size_t)m.x * (size_t)m.y * (size_t)m.z;
}

AcResult
acHostMeshCreate(const AcMeshInfo info, AcMesh* mesh)
{
    if (!mesh)
        return AC_FAILURE;
    memset(mesh, 0, sizeof(*mesh));
    mesh->info = info;
    if (acHostUpdateParams(&mesh->info) != AC_SUCCESS)
        return AC_FAILURE;
    const size_t n = mesh_cells(&mesh->info);
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w) {
        mesh->vertex_buffer[w] = (AcReal*)calloc(n, sizeof(AcReal));
        if (!mesh->vertex_buffer[w]) {
            acHostMeshDestroy(mesh);
            return AC_FAILURE;
        }
    }
    return AC_SUCCESS;
}

AcResult
acHostMeshDestroy(AcMesh* mesh)
{
    if (!mesh)
        return AC_FAILURE;
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w) {
        free(mesh->vertex_buffer[w]);
        mesh->vertex_buffer[w] = NULL;
    }
    return AC_SUCCESS;
}

/* ---- seeded initial conditions ---- */

static inline uint64_t
splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

/* 53-bit uniform in [0, 1). */
static inline double
u01(const uint64_t x)
{
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

AcResult
acHostMeshRandomizeSeeded(AcMesh* mesh, const unsigned long long seed, const AcReal amp_scalar,
                          const AcReal sigma_uu, const AcReal sigma_aa)
{
    if (!mesh)
        return AC_FAILURE;
    const int3 m     = mesh->info.int3_params[AC_mlocal];
    const size_t n   = (size_t)m.x * (size_t)m.y * (size_t)m.z;
    const uint64_t base = splitmix64((uint64_t)seed * 0xD1B54A32D192ED03ull + 0x5851F42D4C957F2Dull);
    const double two_pi = 6.283185307179586476925286766559;
    for (int w = 0; w < NUM_VTXBUF_HANDLES; ++w) {
        AcReal* f = mesh->vertex_buffer[w];
        if (!f)
            continue; /* fields without a buffer are skipped */
        const int gaussian = (w >= VTXBUF_UUX && w <= VTXBUF_AZ);
        const double sigma = (w <= VTXBUF_UUZ) ? sigma_uu : sigma_aa;
        const uint64_t fbase = base + (uint64_t)w * 0x9E3779B97F4A7C15ull * 2ull * (uint64_t)n;
#pragma omp parallel for schedule(static)
        for (long long idx = 0; idx < (long long)n; ++idx) {
            const uint64_t c  = fbase + 2ull * (uint64_t)idx;
            const uint64_t r1 = splitmix64(c);
            if (!gaussian) {
                f[idx] = amp_scalar * (2.0 * u01(r1) - 1.0);
            }
            else {
                const uint64_t r2 = splitmix64(c + 1ull);
                const double a    = 1.0 - u01(r1); /* (0, 1] */
                const double b    = u01(r2);
                f[idx]            = sigma * sqrt(-2.0 * log(a)) * cos(two_pi * b);
            }
        }
    }
    return AC_SUCCESS;
}

/* ---- timestep: samples/standalone_mpi/main.cc:396-441 (maximum form) ----
 * The reference evaluates this in long double with chi = 0 (its
 * "TODO not calculated"), no hyperdiffusion, no shock and no ambipolar term. */
AcReal
acHostTimestepFromMaxima(const AcMeshInfo info, const AcReal uu_max, const AcReal alfven_max)
{
    const long double cdt   = info.real_params[AC_cdt];
    const long double cdtv  = info.real_params[AC_cdtv];
    const long double dsmin = info.real_params[AC_dsmin];
    const long double cs2   = (long double)info.real_params[AC_cs_sound] *
                            (long double)info.real_params[AC_cs_sound];
    const long double nu    = info.real_params[AC_nu_visc];
    const long double eta   = info.real_params[AC_eta];
    const long double chi   = 0;
    const long double gamma = info.real_params[AC_gamma];
    const long double va    = alfven_max;
    const long double advec_dt = cdt * dsmin / (fabsl((long double)uu_max) + sqrtl(cs2 + va * va));
    long double visc           = nu > eta ? nu : eta;
    visc                       = visc > gamma * chi ? visc : gamma * chi;
    const long double diffus_dt = visc > 0 ? cdtv * dsmin * dsmin / visc : (long double)INFINITY;
    return (AcReal)(advec_dt < diffus_dt ? advec_dt : diffus_dt);
}

/* ---- solenoidal Fourier-mode velocity ----
 * u(x) = sum_m a_m sin(k_m . x + phi_m), a_m parallel to k_m x e_m with
 * |a_m| = amplitude / sqrt(nmodes); div u = 0 analytically.  k_m are integer
 * vectors (in units of 2 pi / L) with 1 <= |k_m| <= kmax.  Evaluated with
 * per-axis phase tables, so the cost per cell and mode is a complex multiply. */
AcResult
acHostMeshSolenoidalModes(AcMesh* mesh, const unsigned long long seed, const int nmodes,
                          const int kmax, const AcReal amplitude)
{
    if (!mesh || nmodes <= 0 || kmax < 1)
        return AC_FAILURE;
    AcMeshInfo* info = &mesh->info;
    if (acHostUpdateParams(info) != AC_SUCCESS)
        return AC_FAILURE;
    const int3 m   = info->int3_params[AC_mlocal];
    const int3 n   = info->int3_params[AC_nlocal];
    const AcReal3 ds = info->real3_params[AC_ds];
    const double two_pi = 6.283185307179586476925286766559;
    int* kv     = (int*)malloc(sizeof(int) * 3 * (size_t)nmodes);
    double* av  = (double*)malloc(sizeof(double) * 3 * (size_t)nmodes);
    double* ph  = (double*)malloc(sizeof(double) * (size_t)nmodes);
    if (!kv || !av || !ph) {
        free(kv);
        free(av);
        free(ph);
        return AC_FAILURE;
    }
    uint64_t ctr = splitmix64((uint64_t)seed ^ 0x632BE59BD9B4E019ull);
    for (int md = 0; md < nmodes; ++md) {
        for (;;) {
            int k[3];
            for (int a = 0; a < 3; ++a)
                k[a] = (int)(splitmix64(ctr++) % (uint64_t)(2 * kmax + 1)) - kmax;
            const int k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
            if (k2 == 0 || k2 > kmax * kmax)
                continue;
            double e[3];
            for (int a = 0; a < 3; ++a)
                e[a] = 2.0 * u01(splitmix64(ctr++)) - 1.0;
            const double c[3] = {k[1] * e[2] - k[2] * e[1], k[2] * e[0] - k[0] * e[2],
                                 k[0] * e[1] - k[1] * e[0]};
            const double cn = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
            if (cn < 1e-3)
                continue;
            const double s = amplitude / sqrt((double)nmodes) / cn;
            for (int a = 0; a < 3; ++a) {
                kv[3 * md + a] = k[a];
                av[3 * md + a] = s * c[a];
            }
            ph[md] = two_pi * u01(splitmix64(ctr++));
            break;
        }
    }
    const double L[3] = {ds.x * n.x, ds.y * n.y, ds.z * n.z};
    const int mm[3]   = {m.x, m.y, m.z};
    const double dd[3] = {ds.x, ds.y, ds.z};
    /* tables: t[a][md][i] = exp(i k x_i) as (cos, sin); the phase joins the z table */
    double* tab[3];
    for (int a = 0; a < 3; ++a) {
        tab[a] = (double*)malloc(sizeof(double) * 2 * (size_t)nmodes * (size_t)mm[a]);
        if (!tab[a]) {
            for (int b = 0; b < a; ++b)
                free(tab[b]);
            free(kv);
            free(av);
            free(ph);
            return AC_FAILURE;
        }
        for (int md = 0; md < nmodes; ++md)
            for (int i = 0; i < mm[a]; ++i) {
                const double x   = (i - NGHOST) * dd[a];
                const double ang = two_pi / L[a] * kv[3 * md + a] * x + (a == 2 ? ph[md] : 0.0);
                tab[a][2 * ((size_t)md * mm[a] + i)]     = cos(ang);
                tab[a][2 * ((size_t)md * mm[a] + i) + 1] = sin(ang);
            }
    }
    AcReal* ux = mesh->vertex_buffer[VTXBUF_UUX];
    AcReal* uy = mesh->vertex_buffer[VTXBUF_UUY];
    AcReal* uz = mesh->vertex_buffer[VTXBUF_UUZ];
    if (!ux || !uy || !uz) {
        for (int a = 0; a < 3; ++a)
            free(tab[a]);
        free(kv);
        free(av);
        free(ph);
        return AC_FAILURE;
    }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < m.z; ++k) {
        double* cyz = (double*)malloc(sizeof(double) * 2 * (size_t)nmodes);
        for (int j = 0; j < m.y; ++j) {
            for (int md = 0; md < nmodes; ++md) {
                const double* ty = &tab[1][2 * ((size_t)md * m.y + j)];
                const double* tz = &tab[2][2 * ((size_t)md * m.z + k)];
                cyz[2 * md]     = ty[0] * tz[0] - ty[1] * tz[1];
                cyz[2 * md + 1] = ty[0] * tz[1] + ty[1] * tz[0];
            }
            const size_t row = (size_t)m.x * ((size_t)j + (size_t)m.y * (size_t)k);
            for (int i = 0; i < m.x; ++i) {
                double vx = 0, vy = 0, vz = 0;
                for (int md = 0; md < nmodes; ++md) {
                    const double* tx = &tab[0][2 * ((size_t)md * m.x + i)];
                    const double s   = tx[0] * cyz[2 * md + 1] + tx[1] * cyz[2 * md];
                    vx += av[3 * md] * s;
                    vy += av[3 * md + 1] * s;
                    vz += av[3 * md + 2] * s;
                }
                ux[row + i] = vx;
                uy[row + i] = vy;
                uz[row + i] = vz;
            }
        }
        free(cyz);
    }
    for (int a = 0; a < 3; ++a)
        free(tab[a]);
    free(kv);
    free(av);
    free(ph);
    return AC_SUCCESS;
}

/* ---- snapshots in the reference's host format: src/utils/memory.cc:182-247 ----
 * data-format.csv ("use_double, mx, my, mz" and one line of values) and one
 * raw file <field name>-<id, 5 digits>.dat per field holding every cell
 * (halos included, x fastest), in the current directory.  The format is kept
 * so that files written by either code read in the other. */
static const char kDataFormat[] = "data-format.csv";
static const char* const kFieldNames[NUM_VTXBUF_HANDLES] = {
    "VTXBUF_LNRHO", "VTXBUF_UUX", "VTXBUF_UUY", "VTXBUF_UUZ",
    "VTXBUF_AX",    "VTXBUF_AY",  "VTXBUF_AZ",  "VTXBUF_ENTROPY"};

static int
grid_mm(const AcMeshInfo* in, int3* mm)
{
    AcMeshInfo info = *in;
    if (acHostUpdateParams(&info) != AC_SUCCESS)
        return 0;
    *mm = info.int3_params[AC_mgrid];
    return 1;
}

AcResult
acHostMeshWriteToFile(const AcMesh mesh, const size_t id)
{
    int3 mm;
    if (!grid_mm(&mesh.info, &mm))
        return AC_FAILURE;
    for (int q = 0; q < NUM_VTXBUF_HANDLES; ++q)
        if (!mesh.vertex_buffer[q])
            return AC_NOT_ALLOCATED;
    FILE* header = fopen(kDataFormat, "w");
    if (!header)
        return AC_FAILURE;
    fprintf(header, "use_double, mx, my, mz\n");
    fprintf(header, "%d, %ld, %ld, %ld\n", (int)(sizeof(AcReal) == 8), (long)mm.x, (long)mm.y,
            (long)mm.z);
    if (fclose(header) != 0)
        return AC_FAILURE;
    const size_t count = (size_t)mm.x * (size_t)mm.y * (size_t)mm.z;
    for (int q = 0; q < NUM_VTXBUF_HANDLES; ++q) {
        char path[4096];
        const int n = snprintf(path, sizeof(path), "%s-%.5lu.dat", kFieldNames[q],
                               (unsigned long)id);
        if (n < 0 || (size_t)n >= sizeof(path))
            return AC_FAILURE;
        FILE* fp = fopen(path, "wb");
        if (!fp)
            return AC_FAILURE;
        const size_t written = fwrite(mesh.vertex_buffer[q], sizeof(AcReal), count, fp);
        if (fclose(fp) != 0 || written != count)
            return AC_FAILURE;
    }
    return AC_SUCCESS;
}

AcResult
acHostMeshReadFromFile(const size_t id, AcMesh* mesh)
{
    if (!mesh)
        return AC_FAILURE;
    int3 mm;
    if (!grid_mm(&mesh->info, &mm))
        return AC_FAILURE;
    FILE* header = fopen(kDataFormat, "r");
    if (!header)
        return AC_FAILURE;
    char line[4096];
    int use_double = -1, mx = -1, my = -1, mz = -1;
    const int ok = fgets(line, sizeof(line), header) != NULL &&
                   fscanf(header, "%d, %d, %d, %d", &use_double, &mx, &my, &mz) == 4;
    fclose(header);
    if (!ok || use_double != (int)(sizeof(AcReal) == 8) || mx != mm.x || my != mm.y ||
        mz != mm.z) {
        fprintf(stderr, "astaroth_b200: %s does not describe this mesh\n", kDataFormat);
        return AC_FAILURE;
    }
    const size_t count = (size_t)mm.x * (size_t)mm.y * (size_t)mm.z;
    for (int q = 0; q < NUM_VTXBUF_HANDLES; ++q) {
        if (!mesh->vertex_buffer[q])
            return AC_NOT_ALLOCATED;
        char path[4096];
        const int n = snprintf(path, sizeof(path), "%s-%.5lu.dat", kFieldNames[q],
                               (unsigned long)id);
        if (n < 0 || (size_t)n >= sizeof(path))
            return AC_FAILURE;
        FILE* fp = fopen(path, "rb");
        if (!fp)
            return AC_FAILURE;
        const size_t got = fread(mesh->vertex_buffer[q], sizeof(AcReal), count, fp);
        fclose(fp);
        if (got != count)
            return AC_FAILURE;
    }
    return AC_SUCCESS;
}

/* ---- forcing parameters: src/utils/astaroth_forcing.cc:84-256 ----
 * The reference draws a wave vector from the integer shell kmin <= |k| <= kmax,
 * the angle phi of the helical basis vector and the phase with its own random
 * generator; acHostForcingParams takes those three draws as arguments and
 * computes the rest as the reference does.  acHostGenerateForcingParams makes
 * the draws from a counter-based generator (splitmix64 of seed and step), so a
 * run is reproducible; its draws differ from the reference's generator. */
static AcReal3
v3(const double x, const double y, const double z)
{
    const AcReal3 r = {x, y, z};
    return r;
}

static AcReal3
cross3(const AcReal3 a, const AcReal3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

static AcReal3
normalized3(const AcReal3 a)
{
    const double n = sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    return v3(a.x / n, a.y / n, a.z / n);
}

AcResult
acHostForcingParams(const AcReal3 k_force, const AcReal phi, const AcReal phase, AcMeshInfo* info)
{
    if (!info)
        return AC_FAILURE;
    const double kk = k_force.x * k_force.x + k_force.y * k_force.y + k_force.z * k_force.z;
    if (!(kk > 0.0))
        return AC_FAILURE;
    const double relhel = info->real_params[AC_relhel];
    /* e: a unit vector perpendicular to k, rotated by phi about k
     * (helical_forcing_e_generator, astaroth_forcing.cc:137-155) */
    AcReal3 e = (k_force.y == 0.0 && k_force.z == 0.0) ? v3(0, 1, 0) : v3(1, 0, 0);
    const AcReal3 kxe   = normalized3(cross3(k_force, e));
    const AcReal3 kxkxe = normalized3(cross3(k_force, kxe));
    e = v3(cos(phi) * kxe.x + sin(phi) * kxkxe.x, cos(phi) * kxe.y + sin(phi) * kxkxe.y,
           cos(phi) * kxe.z + sin(phi) * kxkxe.z);
    /* helical_forcing_special_vector, astaroth_forcing.cc:158-216 (Pencil Code
     * forcing_hel_both): f_im = |k| (k x e) / D, f_re = relhel k x (k x e) / D */
    const AcReal3 kdote = v3(k_force.x * e.x, k_force.y * e.y, k_force.z * e.z);
    const AcReal3 ke    = cross3(k_force, e);
    const AcReal3 kke   = cross3(k_force, ke);
    const double kabs   = sqrt(kk);
    const double den    = sqrt(1.0 + relhel * relhel) * kabs *
                       sqrt(kabs * kabs -
                            (kdote.x * kdote.x + kdote.y * kdote.y + kdote.z * kdote.z));
    double* r                = info->real_params;
    r[AC_ff_hel_imx]         = kabs * ke.x / den;
    r[AC_ff_hel_imy]         = kabs * ke.y / den;
    r[AC_ff_hel_imz]         = kabs * ke.z / den;
    r[AC_ff_hel_rex]         = relhel * kke.x / den;
    r[AC_ff_hel_rey]         = relhel * kke.y / den;
    r[AC_ff_hel_rez]         = relhel * kke.z / den;
    r[AC_k_forcex]           = k_force.x;
    r[AC_k_forcey]           = k_force.y;
    r[AC_k_forcez]           = k_force.z;
    r[AC_forcing_phase]      = phase;
    r[AC_kaver]              = (r[AC_kmax] - r[AC_kmin]) / 2.0;
    return AC_SUCCESS;
}

AcResult
acHostGenerateForcingParams(const unsigned long long seed, const unsigned long long step,
                            AcMeshInfo* info)
{
    if (!info)
        return AC_FAILURE;
    const double kmin = info->real_params[AC_kmin], kmax = info->real_params[AC_kmax];
    /* the integer shell of helical_forcing_k_generator, astaroth_forcing.cc:84-133 */
    const int min_int = (int)ceil(kmin), max_int = (int)floor(kmax);
    const double min2 = kmin * kmin, max2 = kmax * kmax;
    const int min2i = min_int * min_int, max2i = max_int * max_int;
    long count = 0;
    for (int pass = 0; pass < 2; ++pass) {
        long pick = -1, n = 0;
        if (pass == 1) {
            if (count == 0)
                return AC_FAILURE;
            const uint64_t c = splitmix64((uint64_t)seed * 0x9E3779B97F4A7C15ull + 3ull * step);
            pick             = (long)(c % (uint64_t)count);
        }
        for (int x = -max_int; x <= max_int; ++x)
            for (int y = -max_int; y <= max_int; ++y)
                for (int z = -max_int; z <= max_int; ++z) {
                    const int d2 = x * x + y * y + z * z;
                    if ((min2 <= d2 || min2i == d2) && (max2 >= d2 || max2i == d2)) {
                        if (pass == 1 && n == pick) {
                            const double two_pi = 6.283185307179586476925286766559;
                            const uint64_t b = (uint64_t)seed * 0x9E3779B97F4A7C15ull + 3ull * step;
                            const double phi   = two_pi * u01(splitmix64(b + 1));
                            const double phase = two_pi * u01(splitmix64(b + 2));
                            return acHostForcingParams(v3(x, y, z), phi, phase, info);
                        }
                        ++n;
                    }
                }
        count = n;
    }
    return AC_FAILURE;
}

