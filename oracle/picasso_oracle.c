/*
 * ORACLE -- test infrastructure only.  Nothing in the product links or calls
 * this file; the tests, the smoke check and the CPU-baseline leg of the
 * benchmark use it as the checker.
 *
 * A CPU, FP64, particle-serial restatement of the reference's transfer path:
 *   - spline evaluation: Picasso::createSpline
 *     (src/Picasso_ParticleInterpolation.hpp:88-105) calls
 *     Cabana::Grid::evaluateSpline (Cabana 0.6.1, Cabana_Grid_Splines.hpp; a
 *     third-party dependency that is not vendored in the reference tree).  Its
 *     published algorithm is restated here: entity-0 coordinate low_x, cell
 *     size dx = coord(1) - coord(0), logical position x0 = (x - low_x)/dx
 *     (+1/2 for even orders), stencil start from the integer part of x0,
 *     uniform B-spline weights of order 1/2/3 and their derivatives / dx, and
 *     physical distance d = entity coordinate - particle position.
 *   - APIC p2g / g2p: src/Picasso_APIC.hpp:55-544, loop order i -> j -> k and
 *     component order as written there.
 *   - PolyPIC linear p2g / g2p: src/Picasso_PolyPIC.hpp:39-359.
 *   - 3x3 determinant and cofactor inverse:
 *     src/Picasso_BatchedLinearAlgebra.hpp:4337-4350, 4626-4686.
 *   - PolyPIC quadratic (27 modes): NOT in the reference (only a 2-D
 *     derivation, doc/polypic/polypic_2d_quadratic.nb).  Defined here as the
 *     tensor product of the per-dimension weight-orthogonal modes
 *     {1, r, r^2 - h^2/4 - alpha r} of that derivation (Fu, Yang, Jiang,
 *     Teran 2017, "A polynomial particle-in-cell method"); parity unpinned.
 *   - cell sort, grid velocity update, advection: not in the reference; the
 *     oracle defines them (parity unpinned).
 *
 * The descriptor structs are the ones of include/picasso_b200.h; all pointers
 * here are host pointers and every array is FP64.
 */
#include "../include/picasso_b200.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAXK 4

typedef struct orc_spline_data {
    int order, nk;
    int s[3][ORC_MAXK];     /* stencil entity indices (unwrapped) */
    double w[3][ORC_MAXK];  /* weights */
    double g[3][ORC_MAXK];  /* weight gradients (physical) */
    double d[3][ORC_MAXK];  /* physical distance entity - particle */
    double dx[3];           /* physical cell size */
    double x0[3];           /* logical position */
} orc_spline_data;

/* ---------------------------------------------------------------------- */
/* descriptors                                                            */
/* ---------------------------------------------------------------------- */
static void entity_offset(int loc, double off[3])
{
    for (int d = 0; d < 3; ++d) off[d] = 0.0;
    if (loc == PICASSO_CELL) {
        off[0] = off[1] = off[2] = 0.5;
    } else if (loc >= PICASSO_FACE_I && loc <= PICASSO_FACE_K) {
        int dim = loc - PICASSO_FACE_I;
        for (int d = 0; d < 3; ++d) off[d] = (d == dim) ? 0.0 : 0.5;
    } else if (loc >= PICASSO_EDGE_I && loc <= PICASSO_EDGE_K) {
        int dim = loc - PICASSO_EDGE_I;
        for (int d = 0; d < 3; ++d) off[d] = (d == dim) ? 0.5 : 0.0;
    }
}

static int staggered_dim(int loc)
{
    if (loc >= PICASSO_FACE_I && loc <= PICASSO_FACE_K) return loc - PICASSO_FACE_I;
    if (loc >= PICASSO_EDGE_I && loc <= PICASSO_EDGE_K) return loc - PICASSO_EDGE_I;
    return -1;
}

static inline int64_t pf_index(const picasso_particle_field* f, int64_t p, int c)
{
    if (f->vector_shift >= 62) return p + (int64_t)c * f->comp_stride;
    int64_t mask = ((int64_t)1 << f->vector_shift) - 1;
    return (p >> f->vector_shift) * f->tile_stride + (int64_t)c * f->comp_stride + (p & mask);
}
static inline double pget(const picasso_particle_field* f, int64_t p, int c)
{
    return ((const double*)f->data)[pf_index(f, p, c)];
}
static inline void pset(const picasso_particle_field* f, int64_t p, int c, double v)
{
    ((double*)f->data)[pf_index(f, p, c)] = v;
}
static inline double* gref(const picasso_grid_field* f, int i, int j, int k, int c)
{
    return (double*)f->data + (int64_t)i * f->stride[0] + (int64_t)j * f->stride[1] +
           (int64_t)k * f->stride[2] + (int64_t)c * f->stride[3];
}

/* Periodic wrap / bounds check of one stencil index (see picasso_mesh). */
static inline int resolve(const picasso_mesh* m, int d, int s, int* out)
{
    if (m->periodic[d]) {
        int n = m->own_extent[d];
        int r = (s - m->own_begin[d]) % n;
        if (r < 0) r += n;
        *out = m->own_begin[d] + r;
        return 1;
    }
    if (s < 0 || s >= m->extent[d]) return 0;
    *out = s;
    return 1;
}

/* ---------------------------------------------------------------------- */
/* spline (Cabana::Grid::evaluateSpline restated)                         */
/* ---------------------------------------------------------------------- */
int oracle_spline(const picasso_spline* sp, const double x[3], orc_spline_data* sd)
{
    double off[3];
    entity_offset(sp->location, off);
    int order = sp->order;
    if (order < 1 || order > 3) return PICASSO_ERR_INVALID_ARGUMENT;
    sd->order = order;
    sd->nk = order + 1;
    for (int d = 0; d < 3; ++d) {
        double cs = sp->mesh.cell_size[d];
        double lo = sp->mesh.low_corner[d] + (0.0 + off[d]) * cs;
        double lo1 = sp->mesh.low_corner[d] + (1.0 + off[d]) * cs;
        double dx = lo1 - lo;
        double rdx = 1.0 / dx;
        double x0 = (x[d] - lo) * rdx + ((order % 2 == 0) ? 0.5 : 0.0);
        int s0 = (int)floor(x0);
        double t = x0 - (double)s0;
        sd->dx[d] = dx;
        sd->x0[d] = x0;
        if (order == 1) {
            sd->s[d][0] = s0;
            sd->s[d][1] = s0 + 1;
            sd->w[d][0] = 1.0 - t;
            sd->w[d][1] = t;
            sd->g[d][0] = -rdx;
            sd->g[d][1] = rdx;
        } else if (order == 2) {
            double xn = t - 0.5; /* particle offset from the centre knot */
            sd->s[d][0] = s0 - 1;
            sd->s[d][1] = s0;
            sd->s[d][2] = s0 + 1;
            sd->w[d][0] = 0.5 * xn * xn - 0.5 * xn + 0.125;
            sd->w[d][1] = 0.75 - xn * xn;
            sd->w[d][2] = 0.5 * xn * xn + 0.5 * xn + 0.125;
            sd->g[d][0] = (xn - 0.5) * rdx;
            sd->g[d][1] = -2.0 * xn * rdx;
            sd->g[d][2] = (xn + 0.5) * rdx;
        } else {
            double u = 1.0 - t;
            sd->s[d][0] = s0 - 1;
            sd->s[d][1] = s0;
            sd->s[d][2] = s0 + 1;
            sd->s[d][3] = s0 + 2;
            sd->w[d][0] = u * u * u / 6.0;
            sd->w[d][1] = 2.0 / 3.0 - t * t + 0.5 * t * t * t;
            sd->w[d][2] = 2.0 / 3.0 - u * u + 0.5 * u * u * u;
            sd->w[d][3] = t * t * t / 6.0;
            sd->g[d][0] = -0.5 * u * u * rdx;
            sd->g[d][1] = (-2.0 * t + 1.5 * t * t) * rdx;
            sd->g[d][2] = (2.0 * u - 1.5 * u * u) * rdx;
            sd->g[d][3] = 0.5 * t * t * rdx;
        }
        for (int n = 0; n < sd->nk; ++n) sd->d[d][n] = lo + sd->s[d][n] * dx - x[d];
    }
    return PICASSO_OK;
}

/* Resolve the whole stencil; returns 0 if any index leaves the mesh. */
static int resolve_stencil(const picasso_mesh* m, orc_spline_data* sd, int idx[3][ORC_MAXK])
{
    for (int d = 0; d < 3; ++d)
        for (int n = 0; n < sd->nk; ++n)
            if (!resolve(m, d, sd->s[d][n], &idx[d][n])) return 0;
    return 1;
}

static void particle_position(const picasso_particle_field* x, int64_t p, double xp[3])
{
    for (int d = 0; d < 3; ++d) xp[d] = pget(x, p, d);
}

/* ---------------------------------------------------------------------- */
/* APIC                                                                   */
/* ---------------------------------------------------------------------- */
static double inertial_scaling(const orc_spline_data* sd)
{
    /* Picasso_APIC.hpp:33-47 */
    if (sd->order == 2) return 4.0 / (sd->dx[0] * sd->dx[0]);
    return 3.0 / (sd->dx[0] * sd->dx[0]);
}

/* One particle of APIC::p2g into the given grid arrays. */
static void apic_p2g_particle(const orc_spline_data* sd, int idx[3][ORC_MAXK], int stag,
                              int ncomp, double m_p, const double c[4][3],
                              const picasso_grid_field* m_i, const picasso_grid_field* mu_i)
{
    int nk = sd->nk;
    int nc = (stag >= 0) ? 3 : ncomp;
    double B[3][3]; /* B_p(d, a) = c_p(1 + a, d)  (APIC.hpp:94-101) */
    for (int d = 0; d < nc; ++d)
        for (int a = 0; a < 3; ++a) B[d][a] = c[1 + a][d];
    if (sd->order >= 2) {
        double D = inertial_scaling(sd);
        double DB[3][3];
        for (int d = 0; d < nc; ++d)
            for (int a = 0; a < 3; ++a) DB[d][a] = D * B[d][a];
        for (int i = 0; i < nk; ++i)
            for (int j = 0; j < nk; ++j)
                for (int k = 0; k < nk; ++k) {
                    double dist[3] = {sd->d[0][i], sd->d[1][j], sd->d[2][k]};
                    double wm = sd->w[0][i] * sd->w[1][j] * sd->w[2][k] * m_p;
                    if (stag < 0) {
                        /* APIC.hpp:121-138 */
                        for (int d = 0; d < ncomp; ++d) {
                            double dbd = 0.0;
                            for (int a = 0; a < 3; ++a) dbd += DB[d][a] * dist[a];
                            *gref(mu_i, idx[0][i], idx[1][j], idx[2][k], d) +=
                                wm * (c[0][d] + dbd);
                        }
                    } else {
                        /* APIC.hpp:219-230: c_p(0,dim) + (D * ~B.row(dim)) * dist */
                        double bd = 0.0;
                        for (int a = 0; a < 3; ++a) bd += DB[stag][a] * dist[a];
                        *gref(mu_i, idx[0][i], idx[1][j], idx[2][k], 0) +=
                            wm * (c[0][stag] + bd);
                    }
                    *gref(m_i, idx[0][i], idx[1][j], idx[2][k], 0) += wm;
                }
    } else {
        /* order 1, gradient form: APIC.hpp:284-318 and :374-401 */
        for (int i = 0; i < nk; ++i)
            for (int j = 0; j < nk; ++j)
                for (int k = 0; k < nk; ++k) {
                    double wm = sd->w[0][i] * sd->w[1][j] * sd->w[2][k] * m_p;
                    double gm[3];
                    gm[0] = sd->g[0][i] * sd->w[1][j] * sd->w[2][k] * m_p;
                    gm[1] = sd->w[0][i] * sd->g[1][j] * sd->w[2][k] * m_p;
                    gm[2] = sd->w[0][i] * sd->w[1][j] * sd->g[2][k] * m_p;
                    if (stag < 0) {
                        for (int d = 0; d < ncomp; ++d) {
                            double bg = 0.0;
                            for (int a = 0; a < 3; ++a) bg += B[d][a] * gm[a];
                            *gref(mu_i, idx[0][i], idx[1][j], idx[2][k], d) +=
                                wm * c[0][d] + bg;
                        }
                    } else {
                        double bg = 0.0;
                        for (int a = 0; a < 3; ++a) bg += B[stag][a] * gm[a];
                        *gref(mu_i, idx[0][i], idx[1][j], idx[2][k], 0) +=
                            wm * c[0][stag] + bg;
                    }
                    *gref(m_i, idx[0][i], idx[1][j], idx[2][k], 0) += wm;
                }
    }
}

static int check_apic(const picasso_spline* sp, int ncomp)
{
    if (sp->order < 1 || sp->order > 3) return PICASSO_ERR_INVALID_ARGUMENT;
    if (staggered_dim(sp->location) >= 0) {
        if (ncomp != 3) return PICASSO_ERR_INVALID_ARGUMENT;
    } else if (ncomp < 1 || ncomp > 3) {
        return PICASSO_ERR_INVALID_ARGUMENT;
    }
    return PICASSO_OK;
}

int oracle_apic_p2g(const picasso_spline* sp, int64_t np, int ncomp,
                    picasso_particle_field x, picasso_particle_field m,
                    picasso_particle_field c, picasso_grid_field m_i,
                    picasso_grid_field mu_i, int64_t* skipped)
{
    int st = check_apic(sp, ncomp);
    if (st) return st;
    int stag = staggered_dim(sp->location);
    int nc = (stag >= 0) ? 3 : ncomp;
    int64_t skip = 0;
    for (int64_t p = 0; p < np; ++p) {
        double xp[3], cp[4][3];
        orc_spline_data sd;
        int idx[3][ORC_MAXK];
        particle_position(&x, p, xp);
        oracle_spline(sp, xp, &sd);
        if (!resolve_stencil(&sp->mesh, &sd, idx)) { ++skip; continue; }
        for (int r = 0; r < 4; ++r)
            for (int d = 0; d < nc; ++d) cp[r][d] = pget(&c, p, r * nc + d);
        apic_p2g_particle(&sd, idx, stag, ncomp, pget(&m, p, 0), cp, &m_i, &mu_i);
    }
    if (skipped) *skipped = skip;
    return PICASSO_OK;
}

static void apic_g2p_particle(const orc_spline_data* sd, int idx[3][ORC_MAXK], int stag,
                              int ncomp, const picasso_grid_field* u_i, double c[4][3])
{
    int nk = sd->nk;
    double u_p[3] = {0, 0, 0};
    double B[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int i = 0; i < nk; ++i)
        for (int j = 0; j < nk; ++j)
            for (int k = 0; k < nk; ++k) {
                double w = sd->w[0][i] * sd->w[1][j] * sd->w[2][k];
                double dist[3] = {sd->d[0][i], sd->d[1][j], sd->d[2][k]};
                if (stag < 0) {
                    /* APIC.hpp:444-460 */
                    double ue[3];
                    for (int d = 0; d < ncomp; ++d)
                        ue[d] = *gref(u_i, idx[0][i], idx[1][j], idx[2][k], d);
                    for (int d = 0; d < ncomp; ++d) u_p[d] = u_p[d] + w * ue[d];
                    for (int d = 0; d < ncomp; ++d)
                        for (int a = 0; a < 3; ++a) B[d][a] += w * ue[d] * dist[a];
                } else {
                    /* APIC.hpp:517-532 */
                    double ue = *gref(u_i, idx[0][i], idx[1][j], idx[2][k], 0);
                    u_p[stag] += w * ue;
                    for (int a = 0; a < 3; ++a) B[stag][a] += w * ue * dist[a];
                }
            }
    int nc = (stag >= 0) ? 3 : ncomp;
    for (int d = 0; d < nc; ++d) {
        c[0][d] = u_p[d];
        c[1][d] = B[d][0];
        c[2][d] = B[d][1];
        c[3][d] = B[d][2];
    }
}

int oracle_apic_g2p(const picasso_spline* sp, int64_t np, int ncomp,
                    picasso_particle_field x, picasso_grid_field u_i,
                    picasso_particle_field c, int64_t* skipped)
{
    int st = check_apic(sp, ncomp);
    if (st) return st;
    int stag = staggered_dim(sp->location);
    int nc = (stag >= 0) ? 3 : ncomp;
    int64_t skip = 0;
    for (int64_t p = 0; p < np; ++p) {
        double xp[3], cp[4][3];
        orc_spline_data sd;
        int idx[3][ORC_MAXK];
        particle_position(&x, p, xp);
        oracle_spline(sp, xp, &sd);
        if (!resolve_stencil(&sp->mesh, &sd, idx)) { ++skip; continue; }
        apic_g2p_particle(&sd, idx, stag, ncomp, &u_i, cp);
        for (int r = 0; r < 4; ++r)
            for (int d = 0; d < nc; ++d) pset(&c, p, r * nc + d, cp[r][d]);
    }
    if (skipped) *skipped = skip;
    return PICASSO_OK;
}

/* ---------------------------------------------------------------------- */
/* 3x3 linear algebra                                                     */
/* ---------------------------------------------------------------------- */
double oracle_det3(const double a[9])
{
    /* BatchedLinearAlgebra.hpp:4344-4349 */
    return a[0] * a[4] * a[8] + a[1] * a[5] * a[6] + a[2] * a[3] * a[7] -
           a[2] * a[4] * a[6] - a[1] * a[3] * a[8] - a[0] * a[5] * a[7];
}

void oracle_inverse3(const double a[9], double inv[9])
{
    /* BatchedLinearAlgebra.hpp:4626-4686: cofactors times (1 / det) */
    double r = 1.0 / oracle_det3(a);
    inv[0] = (a[4] * a[8] - a[5] * a[7]) * r;
    inv[1] = (a[2] * a[7] - a[1] * a[8]) * r;
    inv[2] = (a[1] * a[5] - a[2] * a[4]) * r;
    inv[3] = (a[5] * a[6] - a[3] * a[8]) * r;
    inv[4] = (a[0] * a[8] - a[2] * a[6]) * r;
    inv[5] = (a[2] * a[3] - a[0] * a[5]) * r;
    inv[6] = (a[3] * a[7] - a[4] * a[6]) * r;
    inv[7] = (a[1] * a[6] - a[0] * a[7]) * r;
    inv[8] = (a[0] * a[4] - a[1] * a[3]) * r;
}

void oracle_mat3_inverse(int64_t n, const double* a, double* a_inv, double* det,
                         const double* x, double* y)
{
    for (int64_t b = 0; b < n; ++b) {
        const double* ab = a + 9 * b;
        double inv[9];
        if (det) det[b] = oracle_det3(ab);
        oracle_inverse3(ab, inv);
        if (a_inv) memcpy(a_inv + 9 * b, inv, sizeof(inv));
        if (x && y)
            for (int i = 0; i < 3; ++i) {
                double s = 0.0;
                for (int j = 0; j < 3; ++j) s += inv[3 * i + j] * x[3 * b + j];
                y[3 * b + i] = s;
            }
    }
}

/* ---------------------------------------------------------------------- */
/* PolyPIC                                                                */
/* ---------------------------------------------------------------------- */
/* Mode r <-> per-dimension degrees (a, b, c).  Modes 0..7 are the linear
 * modes in the reference order {1, x, y, z, xy, xz, yz, xyz}
 * (PolyPIC.hpp:109-116); modes 8..26 are the remaining tensor products of
 * degree <= 2 per dimension with at least one quadratic factor, ordered
 * lexicographically in (a, b, c). */
static const int kModeDeg[27][3] = {
    {0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1},
    {1, 1, 1}, {0, 0, 2}, {0, 1, 2}, {0, 2, 0}, {0, 2, 1}, {0, 2, 2}, {1, 0, 2},
    {1, 1, 2}, {1, 2, 0}, {1, 2, 1}, {1, 2, 2}, {2, 0, 0}, {2, 0, 1}, {2, 0, 2},
    {2, 1, 0}, {2, 1, 1}, {2, 1, 2}, {2, 2, 0}, {2, 2, 1}, {2, 2, 2}};

void oracle_polypic_mode_degrees(int out[27][3]) { memcpy(out, kModeDeg, sizeof(kModeDeg)); }

/* Quadratic mode shift alpha = p (h^2 - 4 p^2) / h^2 with p the particle's
 * offset from the centre knot (polypic_2d_quadratic.nb, columns 5/6). */
static double quad_alpha(const orc_spline_data* sd, int d)
{
    double h = sd->dx[d];
    double p = -sd->d[d][1]; /* centre knot distance is -p */
    return p * (h * h - 4.0 * p * p) / (h * h);
}

static double mode1d(int deg, double r, double h, double alpha)
{
    if (deg == 0) return 1.0;
    if (deg == 1) return r;
    return r * r - 0.25 * h * h - alpha * r;
}

static int check_polypic(const picasso_spline* sp, int ncomp)
{
    if (sp->order != 1 && sp->order != 2) return PICASSO_ERR_UNSUPPORTED;
    if (ncomp < 1 || ncomp > 3) return PICASSO_ERR_INVALID_ARGUMENT;
    if (staggered_dim(sp->location) >= 0 && sp->order != 1) return PICASSO_ERR_UNSUPPORTED;
    return PICASSO_OK;
}

int oracle_polypic_p2g(const picasso_spline* sp, int64_t np, int ncomp,
                       picasso_particle_field x, picasso_particle_field m,
                       picasso_particle_field u, picasso_particle_field c,
                       picasso_grid_field mu_i, picasso_grid_field m_i, double dt,
                       int64_t* skipped)
{
    int st = check_polypic(sp, ncomp);
    if (st) return st;
    int stag = staggered_dim(sp->location);
    int nmode = (sp->order == 1) ? 8 : 27;
    /* staggered: a 3-component field contributes column `dim`, a scalar
     * field column 0 (PolyPIC.hpp:181) */
    int col = (stag >= 0) ? ((ncomp == 3) ? stag : 0) : -1;
    int64_t skip = 0;
    for (int64_t p = 0; p < np; ++p) {
        double xp[3];
        orc_spline_data sd;
        int idx[3][ORC_MAXK];
        particle_position(&x, p, xp);
        oracle_spline(sp, xp, &sd);
        if (!resolve_stencil(&sp->mesh, &sd, idx)) { ++skip; continue; }
        double m_p = pget(&m, p, 0);
        /* PolyPIC.hpp:81-87: am_p(a,b) = delta_ab + dt * u_p(1 + a, b) */
        double am[9], ai[9];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                am[3 * a + b] = (a == b) ? 1.0 + dt * pget(&u, p, (1 + a) * 3 + b)
                                         : dt * pget(&u, p, (1 + a) * 3 + b);
        oracle_inverse3(am, ai);
        double cp[27][3];
        for (int r = 0; r < nmode; ++r)
            for (int d = 0; d < ncomp; ++d) cp[r][d] = pget(&c, p, r * ncomp + d);
        double alpha[3] = {0, 0, 0};
        if (sp->order == 2)
            for (int d = 0; d < 3; ++d) alpha[d] = quad_alpha(&sd, d);
        int nk = sd.nk;
        for (int i = 0; i < nk; ++i)
            for (int j = 0; j < nk; ++j)
                for (int k = 0; k < nk; ++k) {
                    double wm = m_p * sd.w[0][i] * sd.w[1][j] * sd.w[2][k];
                    double dist[3] = {sd.d[0][i], sd.d[1][j], sd.d[2][k]};
                    double map[3];
                    for (int a = 0; a < 3; ++a) {
                        double s = 0.0;
                        for (int b = 0; b < 3; ++b) s += ai[3 * a + b] * dist[b];
                        map[a] = s;
                    }
                    double basis[27];
                    if (sp->order == 1) {
                        basis[0] = 1.0;
                        basis[1] = map[0];
                        basis[2] = map[1];
                        basis[3] = map[2];
                        basis[4] = map[0] * map[1];
                        basis[5] = map[0] * map[2];
                        basis[6] = map[1] * map[2];
                        basis[7] = map[0] * map[1] * map[2];
                    } else {
                        for (int r = 0; r < 27; ++r) {
                            double v = 1.0;
                            for (int d = 0; d < 3; ++d)
                                v *= mode1d(kModeDeg[r][d], map[d], sd.dx[d], alpha[d]);
                            basis[r] = v;
                        }
                    }
                    if (col < 0) {
                        for (int d = 0; d < ncomp; ++d) {
                            double s = 0.0;
                            for (int r = 0; r < nmode; ++r) s += cp[r][d] * basis[r];
                            *gref(&mu_i, idx[0][i], idx[1][j], idx[2][k], d) += wm * s;
                        }
                    } else {
                        double s = 0.0;
                        for (int r = 0; r < nmode; ++r) s += cp[r][col] * basis[r];
                        *gref(&mu_i, idx[0][i], idx[1][j], idx[2][k], 0) += wm * s;
                    }
                    *gref(&m_i, idx[0][i], idx[1][j], idx[2][k], 0) += wm;
                }
    }
    if (skipped) *skipped = skip;
    return PICASSO_OK;
}

int oracle_polypic_g2p(const picasso_spline* sp, int64_t np, int ncomp,
                       picasso_particle_field x, picasso_grid_field u_i,
                       picasso_particle_field c, int64_t* skipped)
{
    int st = check_polypic(sp, ncomp);
    if (st) return st;
    int stag = staggered_dim(sp->location);
    int nmode = (sp->order == 1) ? 8 : 27;
    int col = (stag >= 0) ? ((ncomp == 3) ? stag : 0) : -1;
    int64_t skip = 0;
    for (int64_t p = 0; p < np; ++p) {
        double xp[3];
        orc_spline_data sd;
        int idx[3][ORC_MAXK];
        particle_position(&x, p, xp);
        oracle_spline(sp, xp, &sd);
        if (!resolve_stencil(&sp->mesh, &sd, idx)) { ++skip; continue; }
        int nk = sd.nk;
        /* per-dimension mode factors G[d][deg][knot] */
        double G[3][3][ORC_MAXK];
        for (int d = 0; d < 3; ++d)
            for (int n = 0; n < nk; ++n) {
                G[d][0][n] = sd.w[d][n];
                G[d][1][n] = sd.g[d][n];
            }
        if (sp->order == 2) {
            /* weighted least-squares projection onto the orthogonal modes,
             * G = w s_deg(r) / sum_n w s_deg(r)^2.  With q = p / h the
             * denominators are h^2/4 (degree 1) and h^4 (1-4q^2)^2 (3/4-q^2)/4
             * (degree 2, the BTMB diagonal of polypic_2d_quadratic.nb), and
             * the quotients simplify to G1 = 4 w r / h^2 and
             * G2 = {1/(2h^2), -1/h^2, 1/(2h^2)}: the degree-2 quotient is a
             * 0/0 limit at cell faces, so the closed forms are evaluated. */
            for (int d = 0; d < 3; ++d) {
                double h = sd.dx[d], rh2 = 1.0 / (h * h);
                for (int n = 0; n < nk; ++n) G[d][1][n] = 4.0 * sd.w[d][n] * sd.d[d][n] * rh2;
                G[d][2][0] = 0.5 * rh2;
                G[d][2][1] = -rh2;
                G[d][2][2] = 0.5 * rh2;
            }
        }
        double cp[27][3];
        if (col < 0) {
            for (int r = 0; r < nmode; ++r)
                for (int d = 0; d < ncomp; ++d) cp[r][d] = 0.0;
        } else {
            for (int r = 0; r < nmode; ++r)
                for (int d = 0; d < ncomp; ++d) cp[r][d] = pget(&c, p, r * ncomp + d);
            for (int r = 0; r < nmode; ++r) cp[r][col] = 0.0;
        }
        for (int i = 0; i < nk; ++i)
            for (int j = 0; j < nk; ++j)
                for (int k = 0; k < nk; ++k) {
                    double coeff[27];
                    for (int r = 0; r < nmode; ++r)
                        coeff[r] = G[0][kModeDeg[r][0]][i] * G[1][kModeDeg[r][1]][j] *
                                   G[2][kModeDeg[r][2]][k];
                    if (col < 0) {
                        for (int r = 0; r < nmode; ++r)
                            for (int d = 0; d < ncomp; ++d)
                                cp[r][d] += coeff[r] *
                                            *gref(&u_i, idx[0][i], idx[1][j], idx[2][k], d);
                    } else {
                        double ue = *gref(&u_i, idx[0][i], idx[1][j], idx[2][k], 0);
                        for (int r = 0; r < nmode; ++r) cp[r][col] += coeff[r] * ue;
                    }
                }
        for (int r = 0; r < nmode; ++r)
            for (int d = 0; d < ncomp; ++d) pset(&c, p, r * ncomp + d, cp[r][d]);
    }
    if (skipped) *skipped = skip;
    return PICASSO_OK;
}

/* ---------------------------------------------------------------------- */
/* grid update, advection                                                 */
/* ---------------------------------------------------------------------- */
static void owned_box(const picasso_mesh* m, int lo[3], int hi[3])
{
    for (int d = 0; d < 3; ++d) {
        lo[d] = m->periodic[d] ? m->own_begin[d] : 0;
        hi[d] = m->periodic[d] ? m->own_begin[d] + m->own_extent[d] : m->extent[d];
    }
}

int oracle_grid_velocity(const picasso_mesh* mesh, int ncomp, picasso_grid_field m_i,
                         picasso_grid_field mu_i, double thr, picasso_grid_field u_i)
{
    int lo[3], hi[3];
    owned_box(mesh, lo, hi);
    for (int i = lo[0]; i < hi[0]; ++i)
        for (int j = lo[1]; j < hi[1]; ++j)
            for (int k = lo[2]; k < hi[2]; ++k) {
                double m = *gref(&m_i, i, j, k, 0);
                for (int d = 0; d < ncomp; ++d)
                    *gref(&u_i, i, j, k, d) = (m > thr) ? *gref(&mu_i, i, j, k, d) / m : 0.0;
            }
    return PICASSO_OK;
}

/* Grid update of the explicit APIC step, doc/basic/
 * explict_nearly_incompressible_flow.md:20-21: u = (mu + dt f) / m + dt g where
 * m > thr, else 0; then u <- BC(u) with walls along non-periodic dimensions
 * (wall[d][side]: 0 none, 1 no-slip u = 0, 2 free-slip u_d = 0) on the nodes
 * within `width` of the owned range's ends and beyond.  f may be NULL data. */
int oracle_grid_update(const picasso_mesh* mesh, picasso_grid_field m_i,
                       picasso_grid_field mu_i, picasso_grid_field f_i, double dt,
                       const double g[3], double thr, const int wall[6], int width,
                       picasso_grid_field u_i)
{
    int lo[3], hi[3];
    owned_box(mesh, lo, hi);
    for (int i = lo[0]; i < hi[0]; ++i)
        for (int j = lo[1]; j < hi[1]; ++j)
            for (int k = lo[2]; k < hi[2]; ++k) {
                double m = *gref(&m_i, i, j, k, 0);
                double u[3];
                for (int d = 0; d < 3; ++d) {
                    double p = *gref(&mu_i, i, j, k, d);
                    if (f_i.data) p = p + dt * *gref(&f_i, i, j, k, d);
                    u[d] = (m > thr) ? p / m + dt * g[d] : 0.0;
                }
                const int idx[3] = {i, j, k};
                for (int d = 0; d < 3; ++d) {
                    if (mesh->periodic[d]) continue;
                    int side = -1;
                    if (idx[d] < mesh->own_begin[d] + width) side = 0;
                    else if (idx[d] >= mesh->own_begin[d] + mesh->own_extent[d] - width) side = 1;
                    if (side < 0) continue;
                    if (wall[2 * d + side] == 1) u[0] = u[1] = u[2] = 0.0;
                    else if (wall[2 * d + side] == 2) u[d] = 0.0;
                }
                for (int d = 0; d < 3; ++d) *gref(&u_i, i, j, k, d) = u[d];
            }
    return PICASSO_OK;
}

int oracle_advect(const picasso_mesh* mesh, int64_t np, double dt,
                  picasso_particle_field x, picasso_particle_field c)
{
    for (int64_t p = 0; p < np; ++p)
        for (int d = 0; d < 3; ++d) {
            double xn = pget(&x, p, d) + dt * pget(&c, p, d);
            if (mesh->periodic[d]) {
                double lo = mesh->low_corner[d] + mesh->own_begin[d] * mesh->cell_size[d];
                double len = mesh->own_extent[d] * mesh->cell_size[d];
                if (xn < lo) xn += len;
                else if (xn >= lo + len) xn -= len;
            }
            pset(&x, p, d, xn);
        }
    return PICASSO_OK;
}

/* ---------------------------------------------------------------------- */
/* cell sort                                                              */
/* ---------------------------------------------------------------------- */
/* Bin extent per dimension: owned extent along periodic dimensions, full
 * extent otherwise. */
static void bin_extent(const picasso_mesh* m, int nb[3])
{
    for (int d = 0; d < 3; ++d) nb[d] = m->periodic[d] ? m->own_extent[d] : m->extent[d];
}

/* Key of one particle: (tile, bin in tile) of its stencil start, i slowest
 * and k fastest in both.  Particles whose stencil leaves a non-periodic mesh
 * get the key nkeys (one past the last valid key) and so sort last. */
uint32_t oracle_particle_key(const picasso_spline* sp, const double xp[3], const int tile[3])
{
    orc_spline_data sd;
    int nb[3], b[3], nt[3];
    oracle_spline(sp, xp, &sd);
    bin_extent(&sp->mesh, nb);
    for (int d = 0; d < 3; ++d) nt[d] = (nb[d] + tile[d] - 1) / tile[d];
    uint64_t nkeys = (uint64_t)nt[0] * nt[1] * nt[2] * tile[0] * tile[1] * tile[2];
    for (int d = 0; d < 3; ++d) {
        int s = sd.s[d][0];
        if (sp->mesh.periodic[d]) {
            int r = (s - sp->mesh.own_begin[d]) % nb[d];
            if (r < 0) r += nb[d];
            b[d] = r;
        } else {
            if (s < 0 || s > sp->mesh.extent[d] - sd.nk) return (uint32_t)nkeys;
            b[d] = s;
        }
    }
    uint64_t tl = ((uint64_t)(b[0] / tile[0]) * nt[1] + (b[1] / tile[1])) * nt[2] + (b[2] / tile[2]);
    uint64_t ll = ((uint64_t)(b[0] % tile[0]) * tile[1] + (b[1] % tile[1])) * tile[2] + (b[2] % tile[2]);
    return (uint32_t)(tl * (uint64_t)tile[0] * tile[1] * tile[2] + ll);
}

/* Stable counting sort by key (std::stable_sort semantics).  perm[r] =
 * original index of the particle of rank r; tile_offset[t] = first rank of
 * tile t, tile_offset[ntiles] = number of particles inside the mesh. */
int oracle_cell_sort(const picasso_spline* sp, int64_t np, picasso_particle_field x,
                     const int tile[3], uint32_t* key_out, uint32_t* perm,
                     int64_t* tile_offset)
{
    int nb[3], nt[3];
    bin_extent(&sp->mesh, nb);
    for (int d = 0; d < 3; ++d) nt[d] = (nb[d] + tile[d] - 1) / tile[d];
    int64_t ntiles = (int64_t)nt[0] * nt[1] * nt[2];
    int64_t tsize = (int64_t)tile[0] * tile[1] * tile[2];
    int64_t nkeys = ntiles * tsize;
    if (nkeys >= 0xFFFFFFFFll) return PICASSO_ERR_OUT_OF_RANGE;
    uint32_t* key = (uint32_t*)malloc(sizeof(uint32_t) * (np > 0 ? np : 1));
    int64_t* cnt = (int64_t*)calloc((size_t)nkeys + 2, sizeof(int64_t));
    for (int64_t p = 0; p < np; ++p) {
        double xp[3];
        particle_position(&x, p, xp);
        key[p] = oracle_particle_key(sp, xp, tile);
        cnt[key[p] + 1]++;
    }
    for (int64_t k = 1; k <= nkeys + 1; ++k) cnt[k] += cnt[k - 1];
    /* cnt[k] = number of particles with key < k */
    if (tile_offset)
        for (int64_t t = 0; t <= ntiles; ++t) tile_offset[t] = cnt[t * tsize];
    for (int64_t p = 0; p < np; ++p) {
        int64_t r = cnt[key[p]]++;
        perm[r] = (uint32_t)p;
        if (key_out) key_out[r] = key[p];
    }
    free(key);
    free(cnt);
    return PICASSO_OK;
}

/* ---------------------------------------------------------------------- */
/* Multi-threaded APIC step for the CPU baseline.  P2G follows the Kokkos   */
/* OpenMP ScatterView default (one duplicate grid per thread, then a        */
/* reduction over duplicates, GridOperator.hpp:568-591); G2P is a plain     */
/* parallel loop.  Grids are dense (i,j,k,comp) FP64 arrays of the mesh     */
/* extent; only collocated locations.                                       */
/* ---------------------------------------------------------------------- */
int oracle_apic_step_omp(const picasso_spline* sp, int64_t np, int nthreads,
                         picasso_particle_field x, picasso_particle_field m,
                         picasso_particle_field c, double* grid_m, double* grid_mu,
                         double* grid_u, double thr)
{
    if (staggered_dim(sp->location) >= 0) return PICASSO_ERR_UNSUPPORTED;
    const picasso_mesh* mesh = &sp->mesh;
    int64_t nn = (int64_t)mesh->extent[0] * mesh->extent[1] * mesh->extent[2];
    int nt = nthreads > 0 ? nthreads : 1;
#ifdef _OPENMP
    omp_set_num_threads(nt);
#else
    nt = 1;
#endif
    double* dup = (double*)malloc(sizeof(double) * (size_t)nn * 4 * nt);
    if (!dup) return PICASSO_ERR_INVALID_ARGUMENT;
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double* g = dup + (size_t)tid * nn * 4;
        memset(g, 0, sizeof(double) * (size_t)nn * 4);
        picasso_grid_field gm = {g, PICASSO_F64, 0,
                                 {(int64_t)mesh->extent[1] * mesh->extent[2] * 4,
                                  (int64_t)mesh->extent[2] * 4, 4, 1}};
        picasso_grid_field gmu = gm;
        gmu.data = g + 1;
#pragma omp for schedule(static)
        for (int64_t p = 0; p < np; ++p) {
            double xp[3], cp[4][3];
            orc_spline_data sd;
            int idx[3][ORC_MAXK];
            particle_position(&x, p, xp);
            oracle_spline(sp, xp, &sd);
            if (!resolve_stencil(mesh, &sd, idx)) continue;
            for (int r = 0; r < 4; ++r)
                for (int d = 0; d < 3; ++d) cp[r][d] = pget(&c, p, r * 3 + d);
            apic_p2g_particle(&sd, idx, -1, 3, pget(&m, p, 0), cp, &gm, &gmu);
        }
        /* contribute: reduce the duplicates */
#pragma omp for schedule(static)
        for (int64_t n = 0; n < nn; ++n) {
            double s[4] = {0, 0, 0, 0};
            for (int t = 0; t < nt; ++t)
                for (int q = 0; q < 4; ++q) s[q] += dup[((size_t)t * nn + n) * 4 + q];
            grid_m[n] = s[0];
            for (int q = 0; q < 3; ++q) grid_mu[3 * n + q] = s[1 + q];
            for (int q = 0; q < 3; ++q) grid_u[3 * n + q] = (s[0] > thr) ? s[1 + q] / s[0] : 0.0;
        }
        picasso_grid_field gu = {grid_u, PICASSO_F64, 0,
                                 {(int64_t)mesh->extent[1] * mesh->extent[2] * 3,
                                  (int64_t)mesh->extent[2] * 3, 3, 1}};
#pragma omp for schedule(static)
        for (int64_t p = 0; p < np; ++p) {
            double xp[3], cp[4][3];
            orc_spline_data sd;
            int idx[3][ORC_MAXK];
            particle_position(&x, p, xp);
            oracle_spline(sp, xp, &sd);
            if (!resolve_stencil(mesh, &sd, idx)) continue;
            apic_g2p_particle(&sd, idx, -1, 3, &gu, cp);
            for (int r = 0; r < 4; ++r)
                for (int d = 0; d < 3; ++d) pset(&c, p, r * 3 + d, cp[r][d]);
        }
    }
    free(dup);
    return PICASSO_OK;
}
