/*
 * Test infrastructure only: the CPU oracle for the MHD integration hot path.
 *
 * A C restatement, in x87 long double, of Astaroth's host model solver for the
 * 8-field system (lnrho, uu, aa, entropy; LENTROPY=1, LMAGNETIC=1, LUPWD=0,
 * LBFIELD=0, STENCIL_ORDER=6).  The product library never calls or links this
 * file; tests, __graft_entry__.smoke() and bench.py's CPU baseline use it as
 * the checker.
 *
 * The arithmetic follows the reference's order of operations on purpose, so
 * that this file and the reference model compiled by oracle/Makefile (from
 * its own sources) agree bit for bit; the tests check that.  Each function
 * names the reference lines it restates.
 *
 * Layout: one array per field, x fastest, idx = i + mx*(j + my*k), with
 * mx = nx + 6 etc. and the interior at [3, n+3) on every axis.
 */
#define _GNU_SOURCE /* M_PIl, as the reference model uses (modelsolver.cc:83) */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#include "oracle_params.h"

typedef long double R; /* the model's Scalar, src/utils/modelsolver.cc:68 */
typedef struct {
    R x, y, z;
} V3;

enum { LNRHO = 0, UUX, UUY, UUZ, AX, AY, AZ, ENTROPY, NFIELDS };
#define HALO 3

typedef struct {
    int nx, ny, nz, mx, my, mz;
} Dims;

static inline size_t
at(const Dims* d, const int i, const int j, const int k)
{
    return (size_t)i + (size_t)d->mx * ((size_t)j + (size_t)d->my * (size_t)k);
}

/* ---------------------------------------------------------------------------
 * Stencils: src/utils/modelsolver.cc:190-299 (6th order).  p[3] is the centre.
 * ------------------------------------------------------------------------- */
static inline R
d1(const R p[7], const R inv_ds)
{
    const R c1 = (R)3.0 / (R)4.0, c2 = (R)-3.0 / (R)20.0, c3 = (R)1.0 / (R)60.0;
    R s = 0;
    s += c1 * (p[4] - p[2]);
    s += c2 * (p[5] - p[1]);
    s += c3 * (p[6] - p[0]);
    return s * inv_ds;
}

static inline R
d2(const R p[7], const R inv_ds)
{
    const R c0 = (R)-49.0 / (R)18.0, c1 = (R)3.0 / (R)2.0, c2 = (R)-3.0 / (R)20.0,
            c3 = (R)1.0 / (R)90.0;
    R s = c0 * p[3];
    s += c1 * (p[4] + p[2]);
    s += c2 * (p[5] + p[1]);
    s += c3 * (p[6] + p[0]);
    return s * inv_ds * inv_ds;
}

/* Upwinding stencil (a scaled 6th derivative), der6x_upwd of
 * modelsolver.cc:424-492 with the same order of operations. */
static inline R
d6up(const R p[7], const R inv_ds)
{
    return (R)(1.0 / 60.0) * inv_ds *
           (-(R)(20.0) * p[3] + (R)(15.0) * (p[4] + p[2]) - (R)(6.0) * (p[5] + p[1]) + p[6] +
            p[0]);
}

/* Diagonal cross stencil: a runs along (+,+), b along (+,-). */
static inline R
dmix(const R a[7], const R b[7], const R inv_a, const R inv_b)
{
    const R fac = (R)1. / (R)720.;
    const R e1 = (R)(270.0) * fac, e2 = (R)(-27.0) * fac, e3 = (R)(2.0) * fac;
    R s = (R)(0.);
    s += e1 * (a[4] + a[2] - b[4] - b[2]);
    s += e2 * (a[5] + a[1] - b[5] - b[1]);
    s += e3 * (a[6] + a[0] - b[6] - b[0]);
    return s * inv_a * inv_b;
}

/* Per-field derivative record (ScalarData of modelsolver.cc:509-531): value,
 * gradient and the symmetric Hessian h[r][c]. */
typedef struct {
    R v;
    V3 g;
    R h[3][3];
    V3 up; /* upwinding derivatives (modelsolver.cc:501-506), LUPWD only */
} Deriv;

static void
derivs(const double* f, const Dims* d, const int i, const int j, const int k, const R inv[3],
       const int need_mixed, Deriv* out)
{
    R px[7], py[7], pz[7];
    for (int o = 0; o < 7; ++o) {
        px[o] = (R)f[at(d, i + o - 3, j, k)];
        py[o] = (R)f[at(d, i, j + o - 3, k)];
        pz[o] = (R)f[at(d, i, j, k + o - 3)];
    }
    out->v   = (R)f[at(d, i, j, k)];
    out->g.x = d1(px, inv[0]);
    out->g.y = d1(py, inv[1]);
    out->g.z = d1(pz, inv[2]);
    out->h[0][0] = d2(px, inv[0]);
    out->h[1][1] = d2(py, inv[1]);
    out->h[2][2] = d2(pz, inv[2]);
    out->up.x    = d6up(px, inv[0]);
    out->up.y    = d6up(py, inv[1]);
    out->up.z    = d6up(pz, inv[2]);
    if (need_mixed) {
        R a[7], b[7];
        for (int o = 0; o < 7; ++o) {
            a[o] = (R)f[at(d, i + o - 3, j + o - 3, k)];
            b[o] = (R)f[at(d, i + o - 3, j + 3 - o, k)];
        }
        out->h[0][1] = out->h[1][0] = dmix(a, b, inv[0], inv[1]);
        for (int o = 0; o < 7; ++o) {
            a[o] = (R)f[at(d, i + o - 3, j, k + o - 3)];
            b[o] = (R)f[at(d, i + o - 3, j, k + 3 - o)];
        }
        out->h[0][2] = out->h[2][0] = dmix(a, b, inv[0], inv[2]);
        for (int o = 0; o < 7; ++o) {
            a[o] = (R)f[at(d, i, j + o - 3, k + o - 3)];
            b[o] = (R)f[at(d, i, j + o - 3, k + 3 - o)];
        }
        out->h[1][2] = out->h[2][1] = dmix(a, b, inv[1], inv[2]);
    }
}

/* ---------------------------------------------------------------------------
 * Vector helpers and operators: modelsolver.cc:627-745.
 * ------------------------------------------------------------------------- */
static inline R
dot3(const V3 a, const V3 b)
{
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
static inline V3
cross3(const V3 a, const V3 b)
{
    V3 c;
    c.x = a.y * b.z - a.z * b.y;
    c.y = a.z * b.x - a.x * b.z;
    c.z = a.x * b.y - a.y * b.x;
    return c;
}
static inline V3
add3(const V3 a, const V3 b)
{
    V3 r = {a.x + b.x, a.y + b.y, a.z + b.z};
    return r;
}
static inline V3
sub3(const V3 a, const V3 b)
{
    V3 r = {a.x - b.x, a.y - b.y, a.z - b.z};
    return r;
}
static inline V3
scale3(const R s, const V3 a)
{
    V3 r = {s * a.x, s * a.y, s * a.z};
    return r;
}
static inline V3
neg3(const V3 a)
{
    V3 r = {-a.x, -a.y, -a.z};
    return r;
}
static inline R
lap(const Deriv* f)
{
    return f->h[0][0] + f->h[1][1] + f->h[2][2];
}
static inline V3
lapvec(const Deriv v[3])
{
    V3 r = {lap(&v[0]), lap(&v[1]), lap(&v[2])};
    return r;
}
static inline V3
vecvalue(const Deriv v[3])
{
    V3 r = {v[0].v, v[1].v, v[2].v};
    return r;
}
static inline R
divergence(const Deriv v[3])
{
    return v[0].g.x + v[1].g.y + v[2].g.z;
}
static inline V3
curl(const Deriv v[3])
{
    V3 r = {v[2].g.y - v[1].g.z, v[0].g.z - v[2].g.x, v[1].g.x - v[0].g.y};
    return r;
}
/* gradient_of_divergence, modelsolver.cc:685-693 */
static inline V3
graddiv(const Deriv v[3])
{
    V3 r = {v[0].h[0][0] + v[1].h[0][1] + v[2].h[0][2],
            v[0].h[1][0] + v[1].h[1][1] + v[2].h[1][2],
            v[0].h[2][0] + v[1].h[2][1] + v[2].h[2][2]};
    return r;
}
/* (grad v) x: rows are the gradients of the components (mul(gradients(v), x)). */
static inline V3
gradmul(const Deriv v[3], const V3 x)
{
    V3 r = {dot3(v[0].g, x), dot3(v[1].g, x), dot3(v[2].g, x)};
    return r;
}
/* Traceless rate of strain, modelsolver.cc:696-720; S[r] are rows. */
static void
strain(const Deriv u[3], V3 S[3])
{
    S[0].x = (R)(2. / 3.) * u[0].g.x - (R)(1. / 3.) * (u[1].g.y + u[2].g.z);
    S[0].y = (R)(1. / 2.) * (u[0].g.y + u[1].g.x);
    S[0].z = (R)(1. / 2.) * (u[0].g.z + u[2].g.x);
    S[1].y = (R)(2. / 3.) * u[1].g.y - (R)(1. / 3.) * (u[0].g.x + u[2].g.z);
    S[1].z = (R)(1. / 2.) * (u[1].g.z + u[2].g.y);
    S[2].z = (R)(2. / 3.) * u[2].g.z - (R)(1. / 3.) * (u[0].g.x + u[1].g.y);
    S[1].x = S[0].y;
    S[2].x = S[0].z;
    S[2].y = S[1].z;
}
static inline R
contract(const V3 S[3])
{
    R r = 0;
    for (int i = 0; i < 3; ++i)
        r += dot3(S[i], S[i]);
    return r;
}

/* ---------------------------------------------------------------------------
 * Right-hand sides: continuity modelsolver.cc:772-781, momentum :805-875,
 * induction :877-895, lnT/heat conduction/entropy :897-964.
 * ------------------------------------------------------------------------- */
static void
rates(const double* const* f, const Dims* d, const int i, const int j, const int k,
      const OracleParams* p, R out[NFIELDS])
{
    const R inv[3] = {(R)1. / (R)p->ds[0], (R)1. / (R)p->ds[1], (R)1. / (R)p->ds[2]};
    Deriv lnrho, ss, uu[3], aa[3];
    derivs(f[LNRHO], d, i, j, k, inv, 0, &lnrho);
    derivs(f[ENTROPY], d, i, j, k, inv, 0, &ss);
    for (int c = 0; c < 3; ++c) {
        derivs(f[UUX + c], d, i, j, k, inv, 1, &uu[c]);
        derivs(f[AX + c], d, i, j, k, inv, 1, &aa[c]);
    }
    const R nu = p->nu_visc, eta = p->eta, cs = p->cs_sound, gamma = p->gamma,
            cp = p->cp_sound, lnrho0 = p->lnrho0, lnT0 = p->lnT0, mu0 = p->mu0,
            zeta = p->zeta, K = p->K_heatcond;
    const V3 u = vecvalue(uu);
    /* |u| (vecvalue_abs, modelsolver.cc:579-586) for the LUPWD terms */
    const V3 au = {fabsl(u.x), fabsl(u.y), fabsl(u.z)};

    /* continuity; with LUPWD + dot(|u|, upwd(lnrho)) before the divergence */
    if (p->upwind)
        out[LNRHO] = -dot3(u, lnrho.g) + dot3(au, lnrho.up) - divergence(uu);
    else
        out[LNRHO] = -dot3(u, lnrho.g) - divergence(uu);

    /* induction (gauge without grad div A) */
    {
        const V3 B   = curl(aa);
        const V3 ind = add3(cross3(u, B), scale3(eta, lapvec(aa)));
        out[AX]      = ind.x;
        out[AY]      = ind.y;
        out[AZ]      = ind.z;
    }

    /* momentum */
    {
        V3 S[3];
        strain(uu, S);
        const R cs2_sound = cs * cs;
        const R cs2 =
            cs2_sound * expl(gamma * ss.v / cp + (gamma - 1) * (lnrho.v - lnrho0));
        const V3 jj      = scale3((R)(1.) / mu0, sub3(graddiv(aa), lapvec(aa)));
        const V3 B       = curl(aa);
        const R inv_rho  = (R)(1.) / expl(lnrho.v);
        const V3 pgrad   = add3(scale3((R)(1.) / cp, ss.g), lnrho.g);
        const V3 SgL     = {dot3(S[0], lnrho.g), dot3(S[1], lnrho.g), dot3(S[2], lnrho.g)};
        const V3 visc    = add3(add3(lapvec(uu), scale3((R)(1. / 3.), graddiv(uu))),
                                scale3((R)(2.), SgL));
        V3 m = sub3(neg3(gradmul(uu, u)), scale3(cs2, pgrad));
        if (p->upwind) { /* + mul(gradients_upwd(uu), |u|), modelsolver.cc:837-841 */
            const V3 up = {dot3(uu[0].up, au), dot3(uu[1].up, au), dot3(uu[2].up, au)};
            m           = add3(m, up);
        }
        m    = add3(m, scale3(inv_rho, cross3(jj, B)));
        m    = add3(m, scale3(nu, visc));
        m    = add3(m, scale3(zeta, graddiv(uu)));
        out[UUX] = m.x;
        out[UUY] = m.y;
        out[UUZ] = m.z;
    }

    /* entropy */
    {
        V3 S[3];
        strain(uu, S);
        const R lnT    = lnT0 + gamma * ss.v / cp + (gamma - (R)(1.)) * (lnrho.v - lnrho0);
        const R inv_pT = (R)(1.) / (expl(lnrho.v) * expl(lnT));
        const V3 jj    = scale3((R)(1.) / mu0, sub3(graddiv(aa), lapvec(aa)));
        const R divu   = divergence(uu);
        const R rhs    = (R)(0.0) - (R)(0.0) + eta * mu0 * dot3(jj, jj) +
                      (R)(2.) * expl(lnrho.v) * nu * contract(S) +
                      zeta * expl(lnrho.v) * divu * divu;
        /* heat_conduction */
        const R inv_cp   = (R)(1.) / cp;
        const V3 gln_chi = neg3(lnrho.g);
        const R first    = gamma * inv_cp * lap(&ss) + (gamma - (R)(1.)) * lap(&lnrho);
        const V3 second  = add3(scale3(gamma * inv_cp, ss.g), scale3(gamma - (R)(1.), lnrho.g));
        const V3 third   = add3(scale3(gamma, add3(scale3(inv_cp, ss.g), lnrho.g)), gln_chi);
        const R chi      = K / (expl(lnrho.v) * cp);
        const R heat     = cp * chi * (first + dot3(second, third));
        out[ENTROPY]     = -dot3(u, ss.g) + inv_pT * rhs + heat;
    }
}

/* ---------------------------------------------------------------------------
 * Helical forcing added to u in substep 2: forcing() and helical_forcing() of
 * modelsolver.cc:1003-1076, applied as in :1162-1168, with the same order of
 * operations in long double.  The scale is cs * magnitude * sqrt(kaver cs) as
 * in the device code (mhdsolver.ac:318-319); the host model leaves the
 * magnitude out, so the two agree bit for bit at magnitude 1.
 * ------------------------------------------------------------------------- */
static void
forcing_vec(const OracleParams* p, const Dims* d, const int i, const int j, const int k,
            const R dt, R out[3])
{
    const R ds[3] = {(R)p->ds[0], (R)p->ds[1], (R)p->ds[2]};
    const int n[3] = {d->nx, d->ny, d->nz};
    R xx[3]        = {(R)(i - HALO) * ds[0], (R)(j - HALO) * ds[1], (R)(k - HALO) * ds[2]};
    for (int a = 0; a < 3; ++a)
        xx[a] = xx[a] * ((R)2.0 * M_PIl / (ds[a] * n[a]));
    const R phi     = (R)p->f_phase;
    const R cos_phi = cosl(phi);
    const R sin_phi = sinl(phi);
    const R kx      = (R)p->f_k[0] * xx[0] + (R)p->f_k[1] * xx[1] + (R)p->f_k[2] * xx[2];
    const R ckx     = cosl(kx);
    const R skx     = sinl(kx);
    const R re      = ckx * cos_phi - skx * sin_phi;
    const R im      = ckx * sin_phi + skx * cos_phi;
    const R cs2     = (R)(p->cs_sound * p->cs_sound); /* AC_cs2_sound, a double param */
    const R cs      = sqrtl(cs2);
    const R NN      = cs * (R)p->f_magnitude * sqrtl((R)p->f_kaver * cs);
    int ok          = 1;
    for (int a = 0; a < 3; ++a) {
        const R f = (R)p->f_re[a] * re - (R)p->f_im[a] * im;
        out[a]    = sqrtl(dt) * NN * f;
        ok        = ok && !isnan(out[a]) && !isinf(out[a]);
    }
    if (!ok)
        out[0] = out[1] = out[2] = 0;
}

/* ---------------------------------------------------------------------------
 * Periodic halo fill: src/utils/memory.cc:76-149 (every field communicated).
 * ------------------------------------------------------------------------- */
static void
periodic(double* const* f, const Dims* d)
{
    for (int w = 0; w < NFIELDS; ++w)
        for (int k = 0; k < d->mz; ++k)
            for (int j = 0; j < d->my; ++j)
                for (int i = 0; i < d->mx; ++i) {
                    if (i >= HALO && i < d->nx + HALO && j >= HALO && j < d->ny + HALO &&
                        k >= HALO && k < d->nz + HALO)
                        continue;
                    const int is = (i - HALO + d->nx) % d->nx + HALO;
                    const int js = (j - HALO + d->ny) % d->ny + HALO;
                    const int ks = (k - HALO + d->nz) % d->nz + HALO;
                    f[w][at(d, i, j, k)] = f[w][at(d, is, js, ks)];
                }
}

static Dims
mkdims(const int nx, const int ny, const int nz)
{
    Dims d = {nx, ny, nz, nx + 2 * HALO, ny + 2 * HALO, nz + 2 * HALO};
    return d;
}

int
oracle_periodic_bounds(double* const* f, const int nx, const int ny, const int nz)
{
    const Dims d = mkdims(nx, ny, nz);
    periodic(f, &d);
    return 0;
}

/* ---------------------------------------------------------------------------
 * One RK3 step, two passes per substep: src/utils/modelsolver.cc:1078-1175
 * (alpha/beta steps) and :1214-1272 (driver).  w is stored in double between
 * the passes, as the reference's intermediate mesh is.
 * ------------------------------------------------------------------------- */
int
oracle_integrate(double* const* f, const int nx, const int ny, const int nz,
                 const OracleParams* p, const double dt, const int nsteps)
{
    const Dims d     = mkdims(nx, ny, nz);
    const size_t cnt = (size_t)d.mx * d.my * d.mz;
    double* w[NFIELDS];
    for (int q = 0; q < NFIELDS; ++q) {
        w[q] = (double*)calloc(cnt, sizeof(double));
        if (!w[q])
            return 1;
    }
    const R alpha[3] = {(R)(.0), (R)(-5. / 9.), (R)(-153. / 128.)};
    const R beta[3]  = {(R)(1. / 3.), (R)(15. / 16.), (R)(8. / 15.)};
    for (int step = 0; step < nsteps; ++step) {
        for (int s = 0; s < 3; ++s) {
            periodic(f, &d);
#pragma omp parallel for schedule(static)
            for (int k = HALO; k < nz + HALO; ++k)
                for (int j = HALO; j < ny + HALO; ++j)
                    for (int i = HALO; i < nx + HALO; ++i) {
                        R r[NFIELDS];
                        rates((const double* const*)f, &d, i, j, k, p, r);
                        const size_t idx = at(&d, i, j, k);
                        for (int q = 0; q < NFIELDS; ++q)
                            w[q][idx] = s == 0 ? (double)(r[q] * (R)dt)
                                               : (double)(alpha[s] * (R)w[q][idx] + r[q] * (R)dt);
                    }
#pragma omp parallel for schedule(static)
            for (int k = HALO; k < nz + HALO; ++k)
                for (int j = HALO; j < ny + HALO; ++j)
                    for (int i = HALO; i < nx + HALO; ++i) {
                        const size_t idx = at(&d, i, j, k);
                        for (int q = 0; q < NFIELDS; ++q)
                            f[q][idx] += (double)(beta[s] * (R)w[q][idx]);
                        if (s == 2 && p->forcing) {
                            R fu[3];
                            forcing_vec(p, &d, i, j, k, (R)dt, fu);
                            for (int c = 0; c < 3; ++c)
                                f[UUX + c][idx] = (double)((R)f[UUX + c][idx] + fu[c]);
                        }
                    }
        }
    }
    for (int q = 0; q < NFIELDS; ++q)
        free(w[q]);
    return 0;
}

/* The rates of change (RHS) at every interior cell, rounded to double, written
 * to out[q] at the same index.  Halos of f must be filled by the caller. */
int
oracle_rates(const double* const* f, const int nx, const int ny, const int nz,
             const OracleParams* p, double* const* out)
{
    const Dims d = mkdims(nx, ny, nz);
#pragma omp parallel for schedule(static)
    for (int k = HALO; k < nz + HALO; ++k)
        for (int j = HALO; j < ny + HALO; ++j)
            for (int i = HALO; i < nx + HALO; ++i) {
                R r[NFIELDS];
                rates(f, &d, i, j, k, p, r);
                for (int q = 0; q < NFIELDS; ++q)
                    out[q][at(&d, i, j, k)] = (double)r[q];
            }
    return 0;
}

/* ---------------------------------------------------------------------------
 * Reductions: src/utils/modelreduce.cc:52-340 with the reduction types of
 * stdlib/reduction.h:1-8.  rtype: 0 MAX, 1 MIN, 2 SUM, 3 RMS, 4 RMS_EXP,
 * 5 ALFVEN_MAX, 6 ALFVEN_MIN, 7 ALFVEN_RMS.  kind: 1 scalar, 3 vector,
 * 4 vector + scalar.  Sequential sum in (k, j, i) order, as the reference.
 * ------------------------------------------------------------------------- */
enum { MAP_VALUE, MAP_SQUARE, MAP_EXP_SQUARE, MAP_NORM, MAP_ALF_NORM, MAP_ALF_SQUARE };
enum { OP_MAX, OP_MIN, OP_SUM };

static inline R
map_value(const int map, const int kind, const R a, const R b, const R c, const R dd)
{
    if (kind == 1) {
        if (map == MAP_VALUE)
            return a;
        if (map == MAP_SQUARE)
            return a * a;
        return expl(a) * expl(a);
    }
    if (kind == 3) {
        if (map == MAP_NORM)
            return sqrtl(a * a + b * b + c * c);
        if (map == MAP_SQUARE)
            return a * a + b * b + c * c;
        return expl(a) * expl(a) + expl(b) * expl(b) + expl(c) * expl(c);
    }
    if (map == MAP_ALF_NORM)
        return sqrtl(a * a + b * b + c * c) / sqrtl(expl(dd));
    return (a * a + b * b + c * c) / (expl(dd));
}

double
oracle_reduce(const double* const* f, const int nx, const int ny, const int nz, const int kind,
              const int rtype, const int a, const int b, const int c, const int dvi)
{
    static const int ops[8]  = {OP_MAX, OP_MIN, OP_SUM, OP_SUM, OP_SUM, OP_MAX, OP_MIN, OP_SUM};
    static const int rms[8]  = {0, 0, 0, 1, 1, 0, 0, 1};
    static const int scal[8] = {MAP_VALUE, MAP_VALUE, MAP_VALUE, MAP_SQUARE, MAP_EXP_SQUARE,
                                -1, -1, -1};
    static const int vec[8]  = {MAP_NORM, MAP_NORM, MAP_NORM, MAP_SQUARE, MAP_EXP_SQUARE,
                                -1, -1, -1};
    static const int alf[8]  = {-1, -1, -1, -1, -1, MAP_ALF_NORM, MAP_ALF_NORM, MAP_ALF_SQUARE};
    if (rtype < 0 || rtype > 7)
        return NAN;
    const int map = kind == 1 ? scal[rtype] : kind == 3 ? vec[rtype] : alf[rtype];
    if (map < 0)
        return NAN;
    const Dims d = mkdims(nx, ny, nz);
    const double* fa = f[a];
    const double* fb = kind >= 3 ? f[b] : fa;
    const double* fc = kind >= 3 ? f[c] : fa;
    const double* fd = kind == 4 ? f[dvi] : fa;
    const int op     = ops[rtype];
    R res;
    {
        const size_t i0 = at(&d, HALO, HALO, HALO);
        res = op == OP_SUM ? (R)0
                           : map_value(map, kind, (R)fa[i0], (R)fb[i0], (R)fc[i0], (R)fd[i0]);
    }
    for (int k = HALO; k < nz + HALO; ++k)
        for (int j = HALO; j < ny + HALO; ++j)
            for (int i = HALO; i < nx + HALO; ++i) {
                const size_t idx = at(&d, i, j, k);
                const R v = map_value(map, kind, (R)fa[idx], (R)fb[idx], (R)fc[idx], (R)fd[idx]);
                if (op == OP_SUM)
                    res = res + v;
                else if (op == OP_MAX)
                    res = res > v ? res : v;
                else
                    res = res < v ? res : v;
            }
    if (rms[rtype]) {
        const int npts = nx * ny * nz;
        const R inv_n  = (R)1.0 / npts;
        return (double)sqrtl(inv_n * res);
    }
    return (double)res;
}

/* ---------------------------------------------------------------------------
 * Seeded initial condition of the benchmark workloads, for callers of the
 * oracle that must not load the product library (the CPU baseline).  The
 * reference has no seeded Gaussian initial condition (its acHostMeshRandomize
 * is rand()/RAND_MAX, src/core/astaroth.cc:383-400); this is the project's
 * counter-based definition: splitmix64 of (seed, field, cell index), a 53-bit
 * uniform, and Box-Muller for the Gaussian fields.  lnrho and entropy ~
 * U(-amp, amp); uu ~ N(0, sigma_uu^2); aa ~ N(0, sigma_aa^2); every cell of
 * the (nx+6)(ny+6)(nz+6) arrays, halos included.  The tests check its bytes
 * against the input hashes of the golden vectors.
 * ------------------------------------------------------------------------- */
static inline unsigned long long
sm64(unsigned long long x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

static inline double
unit53(const unsigned long long x)
{
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
}

int
oracle_seeded_mesh(double* const* f, const int nx, const int ny, const int nz,
                   const unsigned long long seed, const double amp_scalar, const double sigma_uu,
                   const double sigma_aa)
{
    const Dims d  = mkdims(nx, ny, nz);
    const size_t n = (size_t)d.mx * (size_t)d.my * (size_t)d.mz;
    const unsigned long long base =
        sm64(seed * 0xD1B54A32D192ED03ull + 0x5851F42D4C957F2Dull);
    const double two_pi = 6.283185307179586476925286766559;
    for (int w = 0; w < NFIELDS; ++w) {
        double* a = f[w];
        if (!a)
            continue;
        const int gaussian = w >= UUX && w <= AZ;
        const double sigma = w <= UUZ ? sigma_uu : sigma_aa;
        const unsigned long long fbase =
            base + (unsigned long long)w * 0x9E3779B97F4A7C15ull * 2ull * (unsigned long long)n;
#pragma omp parallel for schedule(static)
        for (long long idx = 0; idx < (long long)n; ++idx) {
            const unsigned long long c = fbase + 2ull * (unsigned long long)idx;
            const unsigned long long r1 = sm64(c);
            if (!gaussian) {
                a[idx] = amp_scalar * (2.0 * unit53(r1) - 1.0);
            }
            else {
                const double u = 1.0 - unit53(r1); /* (0, 1] */
                const double v = unit53(sm64(c + 1ull));
                a[idx]         = sigma * sqrt(-2.0 * log(u)) * cos(two_pi * v);
            }
        }
    }
    return 0;
}
