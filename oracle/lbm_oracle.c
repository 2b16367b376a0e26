/*
 * ORACLE -- test infrastructure only.  Not part of the product path.
 *
 * A plain-C, FP64, single-domain restatement of the coupled thermal
 * lattice-Boltzmann time step of zzhao0930/MPI-Multi-Process-Version
 * (Fortran 90 + MPI).  Each function below names the reference subroutine it
 * restates, as file:line.  Abbreviations used in the citations:
 *   2M = natural-convection_2dim_mono.f90    2B = natural-convection_2dim_block.f90
 *   3M = natural-convection_3dim_mono.f90    3B = natural-convection_3dim_block.f90
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg may load this
 * library, and only as the checker (or as the timed CPU restatement).
 *
 * Semantics: the MPI block decomposition is removed (one domain) and every
 * wall is applied, with one-sided interpolation stencils at both ends of each
 * axis.  That is what the reference computes when every decomposed axis has
 * at least two ranks (2B/3B with dims >= 2); with a single rank on an axis the
 * reference's `if ... elseif` on the rank position applies only one of the two
 * opposite walls (2M:679-694, 3M:919-940), which this restatement does not
 * reproduce.  In 3D the reference never initialises w / wp (3M:256-263); here
 * they start at zero.
 *
 * Arithmetic: every expression keeps the reference's operand order and its
 * divisions (no reciprocal multiplies); build with -ffp-contract=off so that
 * no multiply-add is fused.  gfortran folds x**2.0d0 and x**2 to x*x and
 * (L-1)**3 to (x*x)*x; the same products are written out here.
 *
 * Parity with the Fortran binary itself is pinned separately: the test suite
 * compares this file's outputs against golden fields produced by executing a
 * mechanical translation of the reference's own subroutines, with an emulated
 * MPI of 2x2 ranks (tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int dim, nx, ny, nz, Q, QT;
    long nnode;
    double Ra, Pr, Ma, Thot, Tcold;
    double length_LB, dt;
    double viscosity_LB, kappa, gbeta, tauf, Snu, Sq, sig_k;
    double *x, *y, *z;          /* coordinates 0..n+1, LB units (after mesh()) */
    int *inter_x, *inter_y, *inter_z; /* [(i)*3 + c], i = 1..n, c = 0..2 */
    double omega_U[19], omega_T[7];
    int ex[19], ey[19], ez[19];
    double *f, *f_post, *g, *g_post; /* node-major AoS: [node*Q + a] */
    double *rho, *u, *v, *w, *temp, *F; /* F = Fy (2D) or Fz (3D) */
    double *up, *vp, *wp, *utemp;
    long itc;
} ora_state;

static const int EX2[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};     /* 2M:59 */
static const int EY2[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};     /* 2M:60 */
static const int EX3[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0}; /* 3M:61 */
static const int EY3[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1}; /* 3M:62 */
static const int EZ3[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1}; /* 3M:63 */

/* node index from 1-based (i, j, k) */
#define NID(s, i, j, k) ((long)((i) - 1) + (long)(s)->nx * ((long)((j) - 1) + (long)(s)->ny * (long)((k) - 1)))

/* ------------------------------------------------------------------------ */
/* mesh: 2M:74-134 (3M:122-189)                                              */
/* ------------------------------------------------------------------------ */

/* Raw stretched coordinates x(0..n+1) in [0,1] before the shift/scale.
 * kind 0: the reference's erf grid, 2M:86-88 (constA = stretch, 3.2 there).
 * kind 1: tanh grid 0.5*(1 + tanh(b*(2*xi-1))/tanh(b)), xi = i/(n+1).
 * kind 2: uniform, xi = i/(n+1). */
void ora_grid_raw(int kind, int n, double stretch, double *xr)
{
    for (int i = 0; i <= n + 1; ++i) {
        double xi = (double)i / (double)(n + 1);
        if (kind == 0)
            xr[i] = 0.5 * (erf(stretch * ((double)i / (double)(n + 1) - 0.5)) / erf(0.5 * stretch) + 1.0);
        else if (kind == 1)
            xr[i] = 0.5 * (tanh(stretch * (2.0 * xi - 1.0)) / tanh(stretch) + 1.0);
        else
            xr[i] = xi;
    }
}

/* The shift/scale of 2M:94-116: dx0 = x(1)-x(0) of the x axis, dt0 = dx0,
 * length_LB = 1/dx(1), dt = dt0*length_LB, nodes 1..n shifted by -dx0/2 on
 * every axis, then every coordinate scaled by length_LB.
 * out[0] = dx0, out[1] = length_LB, out[2] = dt.  z may be NULL (2D). */
void ora_mesh(int kind, double stretch, int nx, int ny, int nz,
              double *x, double *y, double *z, double *out)
{
    ora_grid_raw(kind, nx, stretch, x);
    ora_grid_raw(kind, ny, stretch, y);
    if (z) ora_grid_raw(kind, nz, stretch, z);
    double dx1 = x[1] - x[0];
    double dx0 = dx1;
    double dt0 = dx0;
    double length_LB = 1.0 / dx1;
    double dt = dt0 * length_LB;
    for (int i = 1; i <= nx; ++i) x[i] = x[i] - dx0 / 2.0;
    for (int j = 1; j <= ny; ++j) y[j] = y[j] - dx0 / 2.0;
    if (z) for (int k = 1; k <= nz; ++k) z[k] = z[k] - dx0 / 2.0;
    for (int i = 0; i <= nx + 1; ++i) x[i] = x[i] * length_LB;
    for (int j = 0; j <= ny + 1; ++j) y[j] = y[j] * length_LB;
    if (z) for (int k = 0; k <= nz + 1; ++k) z[k] = z[k] * length_LB;
    out[0] = dx0;
    out[1] = length_LB;
    out[2] = dt;
}

/* ------------------------------------------------------------------------ */
/* initial: 2M:136-281 (2B:141-299), 3M:191-345 (3B:229-415)                 */
/* ------------------------------------------------------------------------ */

static void stencil_table(int n, int *t)
{
    /* one-sided at both ends, centred inside: 2B:246-296, 3B:343-412 */
    for (int i = 1; i <= n; ++i) {
        if (i == 1) { t[i * 3 + 0] = i + 1; t[i * 3 + 1] = i; t[i * 3 + 2] = i + 2; }
        else if (i == n) { t[i * 3 + 0] = i - 1; t[i * 3 + 1] = i; t[i * 3 + 2] = i - 2; }
        else { t[i * 3 + 0] = i - 1; t[i * 3 + 1] = i; t[i * 3 + 2] = i + 1; }
    }
}

/* equilibrium of 2M:227-240 / 3M:286-301 at one node */
static void equilibrium(ora_state *s, long id)
{
    double *f = s->f + id * s->Q, *g = s->g + id * s->QT;
    double rho = s->rho[id], u = s->u[id], v = s->v[id], T = s->temp[id];
    if (s->dim == 2) {
        double velocitySquare = u * u + v * v;
        for (int a = 0; a < 9; ++a) {
            double un = u * s->ex[a] + v * s->ey[a];
            f[a] = rho * s->omega_U[a] * (1.0 + 3.0 * un + 4.5 * un * un - 1.5 * velocitySquare);
        }
        for (int a = 0; a < 5; ++a) {
            double un = u * s->ex[a] + v * s->ey[a];
            g[a] = s->omega_T[a] * T * (1.0 + 4.0 * un);
        }
    } else {
        double w = s->w[id];
        double us2 = u * u + v * v + w * w;
        for (int a = 0; a < 19; ++a) {
            double un = u * s->ex[a] + v * s->ey[a] + w * s->ez[a];
            f[a] = s->omega_U[a] * rho * (1.0 + 3.0 * un + 4.5 * un * un - 1.5 * us2);
        }
        for (int a = 0; a < 7; ++a) {
            double un = u * s->ex[a] + v * s->ey[a] + w * s->ez[a];
            g[a] = s->omega_T[a] * T * (1.0 + 6.0 * un);
        }
    }
}

/* x, y, z: coordinates 0..n+1 as produced by ora_mesh (z ignored in 2D). */
ora_state *ora_create(int dim, int nx, int ny, int nz,
                      const double *x, const double *y, const double *z,
                      double dt, double length_LB,
                      double Ra, double Pr, double Ma, double Thot, double Tcold)
{
    ora_state *s = (ora_state *)calloc(1, sizeof(ora_state));
    if (dim != 3) nz = 1;
    s->dim = dim; s->nx = nx; s->ny = ny; s->nz = nz;
    s->Q = dim == 2 ? 9 : 19;
    s->QT = dim == 2 ? 5 : 7;
    s->nnode = (long)nx * ny * nz;
    s->Ra = Ra; s->Pr = Pr; s->Ma = Ma; s->Thot = Thot; s->Tcold = Tcold;
    s->dt = dt; s->length_LB = length_LB;

    /* parameters: 2M:152-162 (2D), 3M:207-229 (3D) */
    s->viscosity_LB = (Ma * (length_LB - 1.0) * sqrt(Pr)) / sqrt(3.0 * Ra);
    s->kappa = s->viscosity_LB / Pr;
    double L1 = length_LB - 1.0;
    s->gbeta = Ra * s->viscosity_LB * s->kappa / ((L1 * L1) * L1);
    s->tauf = s->viscosity_LB * 3.0 + 0.5;
    s->Snu = 1.0 / s->tauf;
    s->Sq = 8.0 * (2.0 - s->Snu) / (8.0 - s->Snu);
    if (dim == 2)
        s->sig_k = 1.0 / (0.5 + 4.0 * (1.0 / s->Snu - 0.5) / (3.0 * Pr));
    else
        s->sig_k = 1.0 / (0.5 + (1.0 / s->Snu - 0.5) / (0.5 * Pr));

    s->x = (double *)malloc(sizeof(double) * (nx + 2));
    s->y = (double *)malloc(sizeof(double) * (ny + 2));
    s->z = (double *)malloc(sizeof(double) * (nz + 2));
    memcpy(s->x, x, sizeof(double) * (nx + 2));
    memcpy(s->y, y, sizeof(double) * (ny + 2));
    if (dim == 3) memcpy(s->z, z, sizeof(double) * (nz + 2));
    else for (int k = 0; k < nz + 2; ++k) s->z[k] = 0.0;

    s->inter_x = (int *)calloc((size_t)(nx + 1) * 3, sizeof(int));
    s->inter_y = (int *)calloc((size_t)(ny + 1) * 3, sizeof(int));
    s->inter_z = (int *)calloc((size_t)(nz + 1) * 3, sizeof(int));
    stencil_table(nx, s->inter_x);
    stencil_table(ny, s->inter_y);
    if (dim == 3) stencil_table(nz, s->inter_z);

    for (int a = 0; a < s->Q; ++a) {
        s->ex[a] = dim == 2 ? EX2[a] : EX3[a];
        s->ey[a] = dim == 2 ? EY2[a] : EY3[a];
        s->ez[a] = dim == 2 ? 0 : EZ3[a];
    }
    if (dim == 2) {
        /* 2M:214-225 */
        s->omega_U[0] = 4.0 / 9.0;
        for (int a = 1; a <= 4; ++a) s->omega_U[a] = 1.0 / 9.0;
        for (int a = 5; a <= 8; ++a) s->omega_U[a] = 1.0 / 36.0;
        s->omega_T[0] = 1.0 / 2.0;
        for (int a = 1; a <= 4; ++a) s->omega_T[a] = 1.0 / 8.0;
    } else {
        /* 3M:273-284 */
        s->omega_U[0] = 1.0 / 3.0;
        for (int a = 1; a <= 6; ++a) s->omega_U[a] = 1.0 / 18.0;
        for (int a = 7; a <= 18; ++a) s->omega_U[a] = 1.0 / 36.0;
        s->omega_T[0] = 1.0 / 2.0;
        for (int a = 1; a <= 6; ++a) s->omega_T[a] = 1.0 / 12.0;
    }

    long N = s->nnode;
    s->f = (double *)calloc((size_t)N * s->Q, sizeof(double));
    s->f_post = (double *)calloc((size_t)N * s->Q, sizeof(double));
    s->g = (double *)calloc((size_t)N * s->QT, sizeof(double));
    s->g_post = (double *)calloc((size_t)N * s->QT, sizeof(double));
    s->rho = (double *)calloc(N, sizeof(double));
    s->u = (double *)calloc(N, sizeof(double));
    s->v = (double *)calloc(N, sizeof(double));
    s->w = (double *)calloc(N, sizeof(double));
    s->temp = (double *)calloc(N, sizeof(double));
    s->F = (double *)calloc(N, sizeof(double));
    s->up = (double *)calloc(N, sizeof(double));
    s->vp = (double *)calloc(N, sizeof(double));
    s->wp = (double *)calloc(N, sizeof(double));
    s->utemp = (double *)calloc(N, sizeof(double));

    /* rho = rho0, u = v = 0, T linear conduction profile: 2M:200-212 (in x),
     * 3M:257-271 (in y) */
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                long id = NID(s, i, j, k);
                s->rho[id] = 1.0;
                if (dim == 2)
                    s->temp[id] = (double)(i - 1) / (double)(nx - 1) * (Tcold - Thot) + Thot;
                else
                    s->temp[id] = (double)(j - 1) / (double)(ny - 1) * (Tcold - Thot) + Thot;
                equilibrium(s, id);
            }
    s->itc = 0;
    return s;
}

/* Replace the macroscopic fields and re-initialise f, g at equilibrium with
 * the formulas of 2M:227-240 / 3M:286-301 (used for the rest-state and
 * noisy initial conditions).  w may be NULL in 2D. */
void ora_set_macro(ora_state *s, const double *rho, const double *u, const double *v,
                   const double *w, const double *T)
{
    long N = s->nnode;
    memcpy(s->rho, rho, sizeof(double) * N);
    memcpy(s->u, u, sizeof(double) * N);
    memcpy(s->v, v, sizeof(double) * N);
    if (w && s->dim == 3) memcpy(s->w, w, sizeof(double) * N);
    memcpy(s->temp, T, sizeof(double) * N);
    for (long id = 0; id < N; ++id) equilibrium(s, id);
}

/* ------------------------------------------------------------------------ */
/* Warm-start initial state (new, no reference counterpart): the equilibrium  */
/* of 2M:227-240 / 3M:286-301 plus the first-order Chapman-Enskog            */
/* non-equilibrium part built from gradients of the given fields:            */
/*   f_a += -3 tau_f dt w_a rho (e_a e_a : grad u - div u / 3)               */
/*   g_a += -tau_T dt wT_a (e_a . grad T),   tau_T = 1 / sig_k               */
/* (tau_f relaxes the second-order moments of the MRT set, sig_k the heat    */
/* flux moments).  Gradients: slope at node m of the quadratic through the   */
/* three nodes of the interpolation stencil (inter_x order, 2B:246-296).     */
/* ------------------------------------------------------------------------ */

/* d/dc at c = xm of the quadratic through (xa, qa), (xm, qm), (xb, qb) */
double ora_slope3(double xa, double qa, double xm, double qm, double xb, double qb)
{
    const double la = (xm - xb) / ((xa - xm) * (xa - xb));
    const double lm = ((xm - xa) + (xm - xb)) / ((xm - xa) * (xm - xb));
    const double lb = (xm - xa) / ((xb - xa) * (xb - xm));
    return (qa * la + qm * lm) + qb * lb;
}

/* stencil partners of node i (1..n) along one axis */
static void stencil_ab(int i, int n, int *a, int *b)
{
    if (i == 1) { *a = i + 1; *b = i + 2; }
    else if (i == n) { *a = i - 1; *b = i - 2; }
    else { *a = i - 1; *b = i + 1; }
}

/* gradient (d/dx, d/dy, d/dz) of field q at node (i, j, k) */
static void grad3(const ora_state *s, const double *q, int i, int j, int k, double out[3])
{
    int a, b;
    stencil_ab(i, s->nx, &a, &b);
    out[0] = ora_slope3(s->x[a], q[NID(s, a, j, k)], s->x[i], q[NID(s, i, j, k)], s->x[b], q[NID(s, b, j, k)]);
    stencil_ab(j, s->ny, &a, &b);
    out[1] = ora_slope3(s->y[a], q[NID(s, i, a, k)], s->y[j], q[NID(s, i, j, k)], s->y[b], q[NID(s, i, b, k)]);
    out[2] = 0.0;
    if (s->dim == 3) {
        stencil_ab(k, s->nz, &a, &b);
        out[2] = ora_slope3(s->z[a], q[NID(s, i, j, a)], s->z[k], q[NID(s, i, j, k)], s->z[b], q[NID(s, i, j, b)]);
    }
}

void ora_set_macro_neq(ora_state *s, const double *rho, const double *u, const double *v,
                       const double *w, const double *T)
{
    ora_set_macro(s, rho, u, v, w, T);
    const double cf = 3.0 * s->tauf * s->dt;
    const double ct = (1.0 / s->sig_k) * s->dt;
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                const long id = NID(s, i, j, k);
                double gu[3], gv[3], gw[3] = {0.0, 0.0, 0.0}, gT[3];
                grad3(s, s->u, i, j, k, gu);
                grad3(s, s->v, i, j, k, gv);
                if (s->dim == 3) grad3(s, s->w, i, j, k, gw);
                grad3(s, s->temp, i, j, k, gT);
                const double div = (gu[0] + gv[1]) + gw[2];
                double *f = s->f + id * s->Q, *g = s->g + id * s->QT;
                for (int a = 0; a < s->Q; ++a) {
                    const double ex = s->ex[a], ey = s->ey[a], ez = s->ez[a];
                    double qq = (ex * ex) * gu[0] + (ex * ey) * (gv[0] + gu[1]) + (ey * ey) * gv[1];
                    if (s->dim == 3)
                        qq = ((qq + (ez * ez) * gw[2]) + (ex * ez) * (gw[0] + gu[2])) + (ey * ez) * (gw[1] + gv[2]);
                    qq = qq - div / 3.0;
                    f[a] = f[a] - ((cf * s->omega_U[a]) * s->rho[id]) * qq;
                }
                for (int a = 0; a < s->QT; ++a) {
                    const double en = (s->ex[a] * gT[0] + s->ey[a] * gT[1]) + s->ez[a] * gT[2];
                    g[a] = g[a] - (ct * s->omega_T[a]) * en;
                }
            }
}

void ora_destroy(ora_state *s)
{
    if (!s) return;
    free(s->x); free(s->y); free(s->z);
    free(s->inter_x); free(s->inter_y); free(s->inter_z);
    free(s->f); free(s->f_post); free(s->g); free(s->g_post);
    free(s->rho); free(s->u); free(s->v); free(s->w); free(s->temp); free(s->F);
    free(s->up); free(s->vp); free(s->wp); free(s->utemp);
    free(s);
}

/* ------------------------------------------------------------------------ */
/* collision_U: 2M:431-520 (2B:462-551)                                      */
/* ------------------------------------------------------------------------ */
static void collision_U_2d(ora_state *s)
{
    const double Snu = s->Snu, Sq = s->Sq, dt = s->dt, gbeta = s->gbeta;
    #pragma omp parallel for schedule(static)
    for (int j = 1; j <= s->ny; ++j)
        for (int i = 1; i <= s->nx; ++i) {
            long id = NID(s, i, j, 1);
            const double *f = s->f + id * 9;
            double *fp = s->f_post + id * 9;
            double m[9], meq[9], sv[9], fSource[9], m_post[9];
            double rho = s->rho[id], u = s->u[id], v = s->v[id];

            m[0] = f[0]+f[1]+f[2]+f[3]+f[4]+f[5]+f[6]+f[7]+f[8];
            m[1] = -4.0*f[0]-f[1]-f[2]-f[3]-f[4]+2.0*(f[5]+f[6]+f[7]+f[8]);
            m[2] = 4.0*f[0]-2.0*(f[1]+f[2]+f[3]+f[4])+f[5]+f[6]+f[7]+f[8];
            m[3] = f[1]-f[3]+f[5]-f[6]-f[7]+f[8];
            m[4] = -2.0*f[1]+2.0*f[3]+f[5]-f[6]-f[7]+f[8];
            m[5] = f[2]-f[4]+f[5]+f[6]-f[7]-f[8];
            m[6] = -2.0*f[2]+2.0*f[4]+f[5]+f[6]-f[7]-f[8];
            m[7] = f[1]-f[2]+f[3]-f[4];
            m[8] = f[5]-f[6]+f[7]-f[8];

            meq[0] = rho;
            meq[1] = rho*( -2.0+3.0*(u*u+v*v) );
            meq[2] = rho*( 1.0-3.0*(u*u+v*v) );
            meq[3] = rho*u;
            meq[4] = -rho*u;
            meq[5] = rho*v;
            meq[6] = -rho*v;
            meq[7] = rho*(u*u-v*v);
            meq[8] = rho*(u*v);

            sv[0] = 0.0; sv[1] = Snu; sv[2] = Snu; sv[3] = 0.0; sv[4] = Sq;
            sv[5] = 0.0; sv[6] = Sq; sv[7] = Snu; sv[8] = Snu;

            double Fx = 0.0;
            double Fy = gbeta*s->temp[id]*rho;
            s->F[id] = Fy;

            fSource[0] = 0.0;
            fSource[1] = (6.0-3.0*sv[1])*(u*Fx+v*Fy);
            fSource[2] = -(6.0-3.0*sv[2])*(u*Fx+v*Fy);
            fSource[3] = Fx;
            fSource[4] = -(1.0-0.5*sv[4])*Fx;
            fSource[5] = Fy;
            fSource[6] = -(1.0-0.5*sv[6])*Fy;
            fSource[7] = (2.0-sv[7])*(u*Fx-v*Fy);
            fSource[8] = (1-0.5*sv[8])*(v*Fx+u*Fy);

            for (int a = 0; a < 9; ++a)
                m_post[a] = m[a]-sv[a]*(m[a]-meq[a])+fSource[a]*dt;

            fp[0] = ( m_post[0]-m_post[1]+m_post[2] )/9.0;
            fp[1] = m_post[0]/9.0-m_post[1]/36.0-m_post[2]/18.0+m_post[3]/6.0-m_post[4]/6.0
                    +m_post[7]*0.25;
            fp[2] = m_post[0]/9.0-m_post[1]/36.0-m_post[2]/18.0
                    +m_post[5]/6.0-m_post[6]/6.0-m_post[7]*0.25;
            fp[3] = m_post[0]/9.0-m_post[1]/36.0-m_post[2]/18.0-m_post[3]/6.0+m_post[4]/6.0
                    +m_post[7]*0.25;
            fp[4] = m_post[0]/9.0-m_post[1]/36.0-m_post[2]/18.0
                    -m_post[5]/6.0+m_post[6]/6.0-m_post[7]*0.25;
            fp[5] = m_post[0]/9.0+m_post[1]/18.0+m_post[2]/36.0+m_post[3]/6.0+m_post[4]/12.0
                    +m_post[5]/6.0+m_post[6]/12.0+m_post[8]*0.25;
            fp[6] = m_post[0]/9.0+m_post[1]/18.0+m_post[2]/36.0-m_post[3]/6.0-m_post[4]/12.0
                    +m_post[5]/6.0+m_post[6]/12.0-m_post[8]*0.25;
            fp[7] = m_post[0]/9.0+m_post[1]/18.0+m_post[2]/36.0-m_post[3]/6.0-m_post[4]/12.0
                    -m_post[5]/6.0-m_post[6]/12.0+m_post[8]*0.25;
            fp[8] = m_post[0]/9.0+m_post[1]/18.0+m_post[2]/36.0+m_post[3]/6.0+m_post[4]/12.0
                    -m_post[5]/6.0-m_post[6]/12.0-m_post[8]*0.25;
        }
    /* f(0) = f_post(0): 2M:513-517 */
    for (long id = 0; id < s->nnode; ++id) s->f[id * 9] = s->f_post[id * 9];
}

/* collision_U 3D: 3M:445-669 (3B:524-748) */
static void collision_U_3d(ora_state *s)
{
    const double Snu = s->Snu, Sq = s->Sq, dt = s->dt, gbeta = s->gbeta;
    #pragma omp parallel for schedule(static)
    for (int k = 1; k <= s->nz; ++k)
    for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i) {
        long id = NID(s, i, j, k);
        const double *f = s->f + id * 19;
        double *fp = s->f_post + id * 19;
        double m[19], meq[19], sv[19], fSource[19], m_post[19];
        double rho = s->rho[id], u = s->u[id], v = s->v[id], w = s->w[id];
        double Vsquare = u*u+v*v+w*w;

        m[0]=f[0]+f[1]+f[2]+f[3]+f[4]+f[5]+f[6]+f[7]+f[8]+f[9]+f[10]+f[11]+f[12]+f[13]+f[14]+f[15]+f[16]+f[17]+f[18];
        m[1]=-30.0*f[0]-11.0*(f[1]+f[2]+f[3]+f[4]+f[5]+f[6])+8.0*(f[7]+f[8]+f[9]+f[10]+f[11]+f[12]+f[13]+f[14]+f[15]+f[16]+f[17]+f[18]);
        m[2]=12.0*f[0]-4.0*(f[1]+f[2]+f[3]+f[4]+f[5]+f[6])+(f[7]+f[8]+f[9]+f[10]+f[11]+f[12]+f[13]+f[14]+f[15]+f[16]+f[17]+f[18]);
        m[3]=f[1]-f[2]+f[7]-f[8]+f[9]-f[10]+f[11]-f[12]+f[13]-f[14];
        m[4]=4.0*(-f[1]+f[2])+f[7]-f[8]+f[9]-f[10]+f[11]-f[12]+f[13]-f[14];
        m[5]=f[3]-f[4]+f[7]+f[8]-f[9]-f[10]+f[15]-f[16]+f[17]-f[18];
        m[6]=-4.0*(f[3]-f[4])+f[7]+f[8]-f[9]-f[10]+f[15]-f[16]+f[17]-f[18];
        m[7]=f[5]-f[6]+f[11]+f[12]-f[13]-f[14]+f[15]+f[16]-f[17]-f[18];
        m[8]=-4.0*(f[5]-f[6])+f[11]+f[12]-f[13]-f[14]+f[15]+f[16]-f[17]-f[18];
        m[9]=2.0*(f[1]+f[2])-(f[3]+f[4]+f[5]+f[6])+f[7]+f[8]+f[9]+f[10]+f[11]+f[12]+f[13]+f[14]-2.0*(f[15]+f[16]+f[17]+f[18]);
        m[10]=-4.0*(f[1]+f[2])+2.0*(f[3]+f[4]+f[5]+f[6])+f[7]+f[8]+f[9]+f[10]+f[11]+f[12]+f[13]+f[14]-2.0*(f[15]+f[16]+f[17]+f[18]);
        m[11]=f[3]+f[4]-f[5]-f[6]+f[7]+f[8]+f[9]+f[10]-f[11]-f[12]-f[13]-f[14];
        m[12]=-2.0*(f[3]+f[4]-f[5]-f[6])+f[7]+f[8]+f[9]+f[10]-f[11]-f[12]-f[13]-f[14];
        m[13]=f[7]-f[8]-f[9]+f[10];
        m[14]=f[15]-f[16]-f[17]+f[18];
        m[15]=f[11]-f[12]-f[13]+f[14];
        m[16]=f[7]-f[8]+f[9]-f[10]-f[11]+f[12]-f[13]+f[14];
        m[17]=-f[7]-f[8]+f[9]+f[10]+f[15]-f[16]+f[17]-f[18];
        m[18]=f[11]+f[12]-f[13]-f[14]-f[15]-f[16]+f[17]+f[18];

        meq[0]=rho;
        meq[1]=-11.0*rho+19.0*rho*Vsquare;
        meq[2]=3.0*rho-5.5*rho*Vsquare;
        meq[3]=rho*u;
        meq[4]=-2.0*rho*u/3.0;
        meq[5]=rho*v;
        meq[6]=-2.0*rho*v/3.0;
        meq[7]=rho*w;
        meq[8]=-2.0*rho*w/3.0;
        meq[9]=3.0*rho*(u*u)-rho*Vsquare;
        meq[10]=-0.5*(3.0*rho*(u*u)-rho*Vsquare);
        meq[11]=rho*((v*v)-(w*w));
        meq[12]=-0.5*rho*((v*v)-(w*w));
        meq[13]=rho*u*v;
        meq[14]=rho*v*w;
        meq[15]=rho*u*w;
        meq[16]=0.0;
        meq[17]=0.0;
        meq[18]=0.0;

        sv[0]=0.0; sv[1]=Snu; sv[2]=Snu; sv[3]=0.0; sv[4]=Sq; sv[5]=0.0; sv[6]=Sq;
        sv[7]=0.0; sv[8]=Sq; sv[9]=Snu; sv[10]=Snu; sv[11]=Snu; sv[12]=Snu;
        sv[13]=Snu; sv[14]=Snu; sv[15]=Snu; sv[16]=Sq; sv[17]=Sq; sv[18]=Sq;

        double Fz = gbeta*s->temp[id]*rho;
        s->F[id] = Fz;

        fSource[0] = 0.0;
        fSource[1] = (38.0-19.0*sv[1])*w*Fz;
        fSource[2] = -(11.0-5.5*sv[2])*w*Fz;
        fSource[3] = 0.0;
        fSource[4] = 0.0;
        fSource[5] = 0.0;
        fSource[6] = 0.0;
        fSource[7] = (1.0-0.5*sv[7])*Fz;
        fSource[8] = -2.0*(1.0-0.5*sv[8])*Fz/3.0;
        fSource[9] = (-2.0+sv[9])*w*Fz;
        fSource[10] = (1.0-0.5*sv[10])*w*Fz;
        fSource[11] = -(2.0-sv[11])*w*Fz;
        fSource[12] = (1.0-0.5*sv[12])*w*Fz;
        fSource[13] = 0.0;
        fSource[14] = (1.0-0.5*sv[14])*v*Fz;
        fSource[15] = (1.0-0.5*sv[15])*u*Fz;
        fSource[16] = 0.0;
        fSource[17] = 0.0;
        fSource[18] = 0.0;

        for (int a = 0; a < 19; ++a)
            m_post[a] = m[a]-sv[a]*(m[a]-meq[a])+fSource[a]*dt;

        const double *mp = m_post;
        fp[0]=mp[0]/19.0-5.0*mp[1]/399.0+mp[2]/21.0;
        fp[1]=mp[0]/19.0-11.0*mp[1]/2394.0-mp[2]/63.0+mp[3]/10.0-mp[4]/10.0+mp[9]/18.0-mp[10]/18.0;
        fp[2]=mp[0]/19.0-11.0*mp[1]/2394.0-mp[2]/63.0-mp[3]/10.0+mp[4]/10.0+mp[9]/18.0-mp[10]/18.0;
        fp[3]=mp[0]/19.0-11.0*mp[1]/2394.0-mp[2]/63.0+mp[5]/10.0-mp[6]/10.0-mp[9]/36.0+mp[10]/36.0+mp[11]/12.0-mp[12]/12.0;
        fp[4]=mp[0]/19.0-11.0*mp[1]/2394.0-mp[2]/63.0-mp[5]/10.0+mp[6]/10.0-mp[9]/36.0+mp[10]/36.0+mp[11]/12.0-mp[12]/12.0;
        fp[5]=mp[0]/19.0-11.0*mp[1]/2394.0-mp[2]/63.0+mp[7]/10.0-mp[8]/10.0-mp[9]/36.0+mp[10]/36.0-mp[11]/12.0+mp[12]/12.0;
        fp[6]=mp[0]/19.0-11.0*mp[1]/2394.0-mp[2]/63.0-mp[7]/10.0+mp[8]/10.0-mp[9]/36.0+mp[10]/36.0-mp[11]/12.0+mp[12]/12.0;
        fp[7]=mp[0]/19.0+4.0*mp[1]/1197.0+mp[2]/252.0+mp[3]/10.0+mp[4]/40.0+mp[5]/10.0+mp[6]/40.0+mp[9]/36.0+mp[10]/72.0
              +mp[11]/12.0+mp[12]/24.0+mp[13]/4.0+mp[16]/8.0-mp[17]/8.0;
        fp[8]=mp[0]/19.0+4.0*mp[1]/1197.0+mp[2]/252.0-mp[3]/10.0-mp[4]/40.0+mp[5]/10.0+mp[6]/40.0+mp[9]/36.0+mp[10]/72.0
              +mp[11]/12.0+mp[12]/24.0-mp[13]/4.0-mp[16]/8.0-mp[17]/8.0;
        fp[9]=mp[0]/19.0+4.0*mp[1]/1197.0+mp[2]/252.0+mp[3]/10.0+mp[4]/40.0-mp[5]/10.0-mp[6]/40.0+mp[9]/36.0+mp[10]/72.0
              +mp[11]/12.0+mp[12]/24.0-mp[13]/4.0+mp[16]/8.0+mp[17]/8.0;
        fp[10]=mp[0]/19.0+4.0*mp[1]/1197.0+mp[2]/252.0-mp[3]/10.0-mp[4]/40.0-mp[5]/10.0-mp[6]/40.0+mp[9]/36.0+mp[10]/72.0
              +mp[11]/12.0+mp[12]/24.0+mp[13]/4.0-mp[16]/8.0+mp[17]/8.0;
        fp[11]=mp[0]/19.0+4.0*mp[1]/1197.0+mp[2]/252.0+mp[3]/10.0+mp[4]/40.0+mp[7]/10.0+mp[8]/40.0+mp[9]/36.0+mp[10]/72.0
              -mp[11]/12.0-mp[12]/24.0+mp[15]/4.0-mp[16]/8.0+mp[18]/8.0;
        fp[12]=mp[0]/19.0+4.0*mp[1]/1197.0+mp[2]/252.0-mp[3]/10.0-mp[4]/40.0+mp[7]/10.0+mp[8]/40.0+mp[9]/36.0+mp[10]/72.0
              -mp[11]/12.0-mp[12]/24.0-mp[15]/4.0+mp[16]/8.0+mp[18]/8.0;
        fp[13]=mp[0]/19.0+4.0*mp[1]/1197.0+mp[2]/252.0+mp[3]/10.0+mp[4]/40.0-mp[7]/10.0-mp[8]/40.0+mp[9]/36.0+mp[10]/72.0
              -mp[11]/12.0-mp[12]/24.0-mp[15]/4.0-mp[16]/8.0-mp[18]/8.0;
        fp[14]=mp[0]/19.0+4.0*mp[1]/1197.0+mp[2]/252.0-mp[3]/10.0-mp[4]/40.0-mp[7]/10.0-mp[8]/40.0+mp[9]/36.0+mp[10]/72.0
              -mp[11]/12.0-mp[12]/24.0+mp[15]/4.0+mp[16]/8.0-mp[18]/8.0;
        fp[15]=mp[0]/19.0+4.0*mp[1]/1197.0+mp[2]/252.0+mp[5]/10.0+mp[6]/40.0+mp[7]/10.0+mp[8]/40.0-mp[9]/18.0-mp[10]/36.0
              +mp[14]/4.0+mp[17]/8.0-mp[18]/8.0;
        fp[16]=mp[0]/19.0+4.0*mp[1]/1197.0+mp[2]/252.0-mp[5]/10.0-mp[6]/40.0+mp[7]/10.0+mp[8]/40.0-mp[9]/18.0-mp[10]/36.0
              -mp[14]/4.0-mp[17]/8.0-mp[18]/8.0;
        fp[17]=mp[0]/19.0+4.0*mp[1]/1197.0+mp[2]/252.0+mp[5]/10.0+mp[6]/40.0-mp[7]/10.0-mp[8]/40.0-mp[9]/18.0-mp[10]/36.0
              -mp[14]/4.0+mp[17]/8.0+mp[18]/8.0;
        fp[18]=mp[0]/19.0+4.0*mp[1]/1197.0+mp[2]/252.0-mp[5]/10.0-mp[6]/40.0-mp[7]/10.0-mp[8]/40.0-mp[9]/18.0-mp[10]/36.0
              +mp[14]/4.0-mp[17]/8.0+mp[18]/8.0;
    }
    /* f(0) = f_post(0): 3M:660-666 */
    for (long id = 0; id < s->nnode; ++id) s->f[id * 19] = s->f_post[id * 19];
}

/* ------------------------------------------------------------------------ */
/* collision_T: 2M:522-569, 3M:671-730                                       */
/* ------------------------------------------------------------------------ */
static void collision_T_2d(ora_state *s)
{
    const double sig_k = s->sig_k;
    #pragma omp parallel for schedule(static)
    for (int j = 1; j <= s->ny; ++j)
        for (int i = 1; i <= s->nx; ++i) {
            long id = NID(s, i, j, 1);
            const double *g = s->g + id * 5;
            double *gp = s->g_post + id * 5;
            double n[5], n_post[5], neq[5], Qr[5];
            double T = s->temp[id];
            n[0] = g[0]+g[1]+g[2]+g[3]+g[4];
            n[1] = g[1]-g[3];
            n[2] = g[2]-g[4];
            n[3] = g[1]+g[2]+g[3]+g[4];
            n[4] = g[1]-g[2]+g[3]-g[4];
            Qr[0] = 1.0; Qr[1] = sig_k; Qr[2] = sig_k; Qr[3] = 1.9; Qr[4] = 1.9;
            neq[0] = T;
            neq[1] = T*s->u[id];
            neq[2] = T*s->v[id];
            neq[3] = T*0.5;
            neq[4] = 0.0;
            for (int a = 0; a < 5; ++a) n_post[a] = n[a]-Qr[a]*(n[a]-neq[a]);
            gp[0] = n_post[0]-n_post[3];
            gp[1] = n_post[1]/2.0+n_post[3]/4.0+n_post[4]/4.0;
            gp[2] = n_post[2]/2.0+n_post[3]/4.0-n_post[4]/4.0;
            gp[3] = -n_post[1]/2.0+n_post[3]/4.0+n_post[4]/4.0;
            gp[4] = -n_post[2]/2.0+n_post[3]/4.0-n_post[4]/4.0;
        }
    for (long id = 0; id < s->nnode; ++id) s->g[id * 5] = s->g_post[id * 5];
}

static void collision_T_3d(ora_state *s)
{
    const double sig_k = s->sig_k;
    #pragma omp parallel for schedule(static)
    for (int k = 1; k <= s->nz; ++k)
    for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i) {
        long id = NID(s, i, j, k);
        const double *g = s->g + id * 7;
        double *gp = s->g_post + id * 7;
        double n[7], n_post[7], neq[7], Qr[7];
        double T = s->temp[id];
        n[0] = g[0]+g[1]+g[2]+g[3]+g[4]+g[5]+g[6];
        n[1] = g[1]-g[2];
        n[2] = g[3]-g[4];
        n[3] = g[5]-g[6];
        n[4] = g[1]+g[2]+g[3]+g[4]+g[5]+g[6];
        n[5] = g[1]+g[2]-g[3]-g[4];
        n[6] = g[1]+g[2]-g[5]-g[6];
        Qr[0] = 1.0; Qr[1] = sig_k; Qr[2] = sig_k; Qr[3] = sig_k; Qr[4] = 1.2; Qr[5] = 1.2; Qr[6] = 1.2;
        neq[0] = T;
        neq[1] = T*s->u[id];
        neq[2] = T*s->v[id];
        neq[3] = T*s->w[id];
        neq[4] = T*0.5;
        neq[5] = 0.0;
        neq[6] = 0.0;
        for (int a = 0; a < 7; ++a) n_post[a] = n[a]-Qr[a]*(n[a]-neq[a]);
        gp[0] = n_post[0]-n_post[4];
        gp[1] = n_post[1]/2.0+n_post[4]/6.0+n_post[5]/6.0+n_post[6]/6.0;
        gp[2] = -n_post[1]/2.0+n_post[4]/6.0+n_post[5]/6.0+n_post[6]/6.0;
        gp[3] = n_post[2]/2.0+n_post[4]/6.0-n_post[5]/3.0+n_post[6]/6.0;
        gp[4] = -n_post[2]/2.0+n_post[4]/6.0-n_post[5]/3.0+n_post[6]/6.0;
        gp[5] = n_post[3]/2.0+n_post[4]/6.0+n_post[5]/6.0-n_post[6]/3.0;
        gp[6] = -n_post[3]/2.0+n_post[4]/6.0+n_post[5]/6.0-n_post[6]/3.0;
    }
    for (long id = 0; id < s->nnode; ++id) s->g[id * 7] = s->g_post[id * 7];
}

/* ------------------------------------------------------------------------ */
/* interpolate (ISLBM streaming): 2M:591-660, 3M:751-876                     */
/* ------------------------------------------------------------------------ */

/* interpolateF: 2M:649-660 */
static inline double interpolateF(double x0, double x1, double x2, double x,
                                  double f0, double f1, double f2)
{
    return ((x - x1) * (x - x2)) / ((x0 - x1) * (x0 - x2)) * f0 +
           ((x - x0) * (x - x2)) / ((x1 - x0) * (x1 - x2)) * f1 +
           ((x - x0) * (x - x1)) / ((x2 - x0) * (x2 - x1)) * f2;
}

double ora_interpolateF(double x0, double x1, double x2, double x,
                        double f0, double f1, double f2)
{
    return interpolateF(x0, x1, x2, x, f0, f1, f2);
}

#define FP2(a, i, j) (s->f_post[NID(s, i, j, 1) * 9 + (a)])
#define GP2(a, i, j) (s->g_post[NID(s, i, j, 1) * 5 + (a)])

static void interpolate_2d(ora_state *s)
{
    const double dt = s->dt;
    const double *xG = s->x, *yG = s->y;
    #pragma omp parallel for schedule(static)
    for (int j = 1; j <= s->ny; ++j)
        for (int i = 1; i <= s->nx; ++i) {
            const int *ix = s->inter_x + i * 3, *iy = s->inter_y + j * 3;
            long id = NID(s, i, j, 1);
            for (int alpha = 1; alpha <= 8; ++alpha) {
                double delta_x = (double)s->ex[alpha] * dt;
                double delta_y = (double)s->ey[alpha] * dt;
                double f0 = interpolateF(yG[iy[0]] + delta_y, yG[iy[1]] + delta_y, yG[iy[2]] + delta_y,
                                         yG[iy[1]], FP2(alpha, ix[0], iy[0]), FP2(alpha, ix[0], iy[1]),
                                         FP2(alpha, ix[0], iy[2]));
                double f1 = interpolateF(yG[iy[0]] + delta_y, yG[iy[1]] + delta_y, yG[iy[2]] + delta_y,
                                         yG[iy[1]], FP2(alpha, ix[1], iy[0]), FP2(alpha, ix[1], iy[1]),
                                         FP2(alpha, ix[1], iy[2]));
                double f2 = interpolateF(yG[iy[0]] + delta_y, yG[iy[1]] + delta_y, yG[iy[2]] + delta_y,
                                         yG[iy[1]], FP2(alpha, ix[2], iy[0]), FP2(alpha, ix[2], iy[1]),
                                         FP2(alpha, ix[2], iy[2]));
                s->f[id * 9 + alpha] = interpolateF(xG[ix[0]] + delta_x, xG[ix[1]] + delta_x,
                                                    xG[ix[2]] + delta_x, xG[ix[1]], f0, f1, f2);
            }
            for (int alpha = 1; alpha <= 4; ++alpha) {
                double delta_x = (double)s->ex[alpha] * dt;
                double delta_y = (double)s->ey[alpha] * dt;
                double g0 = interpolateF(yG[iy[0]] + delta_y, yG[iy[1]] + delta_y, yG[iy[2]] + delta_y,
                                         yG[iy[1]], GP2(alpha, ix[0], iy[0]), GP2(alpha, ix[0], iy[1]),
                                         GP2(alpha, ix[0], iy[2]));
                double g1 = interpolateF(yG[iy[0]] + delta_y, yG[iy[1]] + delta_y, yG[iy[2]] + delta_y,
                                         yG[iy[1]], GP2(alpha, ix[1], iy[0]), GP2(alpha, ix[1], iy[1]),
                                         GP2(alpha, ix[1], iy[2]));
                double g2 = interpolateF(yG[iy[0]] + delta_y, yG[iy[1]] + delta_y, yG[iy[2]] + delta_y,
                                         yG[iy[1]], GP2(alpha, ix[2], iy[0]), GP2(alpha, ix[2], iy[1]),
                                         GP2(alpha, ix[2], iy[2]));
                s->g[id * 5 + alpha] = interpolateF(xG[ix[0]] + delta_x, xG[ix[1]] + delta_x,
                                                    xG[ix[2]] + delta_x, xG[ix[1]], g0, g1, g2);
            }
        }
}

#define FP3(a, i, j, k) (s->f_post[NID(s, i, j, k) * 19 + (a)])
#define GP3(a, i, j, k) (s->g_post[NID(s, i, j, k) * 7 + (a)])

static void interpolate_3d(ora_state *s)
{
    const double dt = s->dt;
    const double *xG = s->x, *yG = s->y, *zG = s->z;
    #pragma omp parallel for schedule(static)
    for (int k = 1; k <= s->nz; ++k)
    for (int j = 1; j <= s->ny; ++j)
    for (int i = 1; i <= s->nx; ++i) {
        const int *ix = s->inter_x + i * 3, *iy = s->inter_y + j * 3, *iz = s->inter_z + k * 3;
        long id = NID(s, i, j, k);
        for (int alpha = 1; alpha <= 18; ++alpha) {
            double delta_x = (double)s->ex[alpha] * dt;
            double delta_y = (double)s->ey[alpha] * dt;
            double delta_z = (double)s->ez[alpha] * dt;
            double f0, f1, f2, out;
            if (alpha == 5 || alpha == 6 || alpha == 15 || alpha == 16 || alpha == 17 || alpha == 18) {
                /* yoz plane: 3M:767-784 */
                f0 = interpolateF(zG[iz[0]] + delta_z, zG[iz[1]] + delta_z, zG[iz[2]] + delta_z, zG[iz[1]],
                                  FP3(alpha, ix[1], iy[0], iz[0]), FP3(alpha, ix[1], iy[0], iz[1]),
                                  FP3(alpha, ix[1], iy[0], iz[2]));
                f1 = interpolateF(zG[iz[0]] + delta_z, zG[iz[1]] + delta_z, zG[iz[2]] + delta_z, zG[iz[1]],
                                  FP3(alpha, ix[1], iy[1], iz[0]), FP3(alpha, ix[1], iy[1], iz[1]),
                                  FP3(alpha, ix[1], iy[1], iz[2]));
                f2 = interpolateF(zG[iz[0]] + delta_z, zG[iz[1]] + delta_z, zG[iz[2]] + delta_z, zG[iz[1]],
                                  FP3(alpha, ix[1], iy[2], iz[0]), FP3(alpha, ix[1], iy[2], iz[1]),
                                  FP3(alpha, ix[1], iy[2], iz[2]));
                out = interpolateF(yG[iy[0]] + delta_y, yG[iy[1]] + delta_y, yG[iy[2]] + delta_y, yG[iy[1]],
                                   f0, f1, f2);
            } else if (alpha == 1 || alpha == 2 || alpha == 11 || alpha == 12 || alpha == 13 || alpha == 14) {
                /* xoz plane: 3M:787-804 */
                f0 = interpolateF(zG[iz[0]] + delta_z, zG[iz[1]] + delta_z, zG[iz[2]] + delta_z, zG[iz[1]],
                                  FP3(alpha, ix[0], iy[1], iz[0]), FP3(alpha, ix[0], iy[1], iz[1]),
                                  FP3(alpha, ix[0], iy[1], iz[2]));
                f1 = interpolateF(zG[iz[0]] + delta_z, zG[iz[1]] + delta_z, zG[iz[2]] + delta_z, zG[iz[1]],
                                  FP3(alpha, ix[1], iy[1], iz[0]), FP3(alpha, ix[1], iy[1], iz[1]),
                                  FP3(alpha, ix[1], iy[1], iz[2]));
                f2 = interpolateF(zG[iz[0]] + delta_z, zG[iz[1]] + delta_z, zG[iz[2]] + delta_z, zG[iz[1]],
                                  FP3(alpha, ix[2], iy[1], iz[0]), FP3(alpha, ix[2], iy[1], iz[1]),
                                  FP3(alpha, ix[2], iy[1], iz[2]));
                out = interpolateF(xG[ix[0]] + delta_x, xG[ix[1]] + delta_x, xG[ix[2]] + delta_x, xG[ix[1]],
                                   f0, f1, f2);
            } else {
                /* xoy plane: 3M:807-824 */
                f0 = interpolateF(yG[iy[0]] + delta_y, yG[iy[1]] + delta_y, yG[iy[2]] + delta_y, yG[iy[1]],
                                  FP3(alpha, ix[0], iy[0], iz[1]), FP3(alpha, ix[0], iy[1], iz[1]),
                                  FP3(alpha, ix[0], iy[2], iz[1]));
                f1 = interpolateF(yG[iy[0]] + delta_y, yG[iy[1]] + delta_y, yG[iy[2]] + delta_y, yG[iy[1]],
                                  FP3(alpha, ix[1], iy[0], iz[1]), FP3(alpha, ix[1], iy[1], iz[1]),
                                  FP3(alpha, ix[1], iy[2], iz[1]));
                f2 = interpolateF(yG[iy[0]] + delta_y, yG[iy[1]] + delta_y, yG[iy[2]] + delta_y, yG[iy[1]],
                                  FP3(alpha, ix[2], iy[0], iz[1]), FP3(alpha, ix[2], iy[1], iz[1]),
                                  FP3(alpha, ix[2], iy[2], iz[1]));
                out = interpolateF(xG[ix[0]] + delta_x, xG[ix[1]] + delta_x, xG[ix[2]] + delta_x, xG[ix[1]],
                                   f0, f1, f2);
            }
            s->f[id * 19 + alpha] = out;
        }
        for (int alpha = 1; alpha <= 6; ++alpha) {
            double delta_x = (double)s->ex[alpha] * dt;
            double delta_y = (double)s->ey[alpha] * dt;
            double delta_z = (double)s->ez[alpha] * dt;
            double out;
            if (alpha == 3 || alpha == 4) {          /* 3M:838-842 */
                out = interpolateF(yG[iy[0]] + delta_y, yG[iy[1]] + delta_y, yG[iy[2]] + delta_y, yG[iy[1]],
                                   GP3(alpha, ix[1], iy[0], iz[1]), GP3(alpha, ix[1], iy[1], iz[1]),
                                   GP3(alpha, ix[1], iy[2], iz[1]));
            } else if (alpha == 5 || alpha == 6) {   /* 3M:844-848 */
                out = interpolateF(zG[iz[0]] + delta_z, zG[iz[1]] + delta_z, zG[iz[2]] + delta_z, zG[iz[1]],
                                   GP3(alpha, ix[1], iy[1], iz[0]), GP3(alpha, ix[1], iy[1], iz[1]),
                                   GP3(alpha, ix[1], iy[1], iz[2]));
            } else {                                 /* 3M:850-854 */
                out = interpolateF(xG[ix[0]] + delta_x, xG[ix[1]] + delta_x, xG[ix[2]] + delta_x, xG[ix[1]],
                                   GP3(alpha, ix[0], iy[1], iz[1]), GP3(alpha, ix[1], iy[1], iz[1]),
                                   GP3(alpha, ix[2], iy[1], iz[1]));
            }
            s->g[id * 7 + alpha] = out;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* bounceback_u / bounceback_T: 2B:731-801 (2M:662-724), 3B:1053-1197       */
/* ------------------------------------------------------------------------ */
#define F2(a, i, j) (s->f[NID(s, i, j, 1) * 9 + (a)])
#define G2(a, i, j) (s->g[NID(s, i, j, 1) * 5 + (a)])

static void bounceback_2d(ora_state *s)
{
    int nx = s->nx, ny = s->ny;
    for (int j = 1; j <= ny; ++j) {
        /* left, 2B:737-741 */
        F2(1, 1, j) = FP2(3, 1, j);
        F2(5, 1, j) = FP2(7, 1, j);
        F2(8, 1, j) = FP2(6, 1, j);
        /* right, 2B:745-749 */
        F2(3, nx, j) = FP2(1, nx, j);
        F2(6, nx, j) = FP2(8, nx, j);
        F2(7, nx, j) = FP2(5, nx, j);
    }
    for (int i = 1; i <= nx; ++i) {
        /* top, 2B:754-758 */
        F2(4, i, ny) = FP2(2, i, ny);
        F2(7, i, ny) = FP2(5, i, ny);
        F2(8, i, ny) = FP2(6, i, ny);
        /* bottom, 2B:761-765 */
        F2(2, i, 1) = FP2(4, i, 1);
        F2(5, i, 1) = FP2(7, i, 1);
        F2(6, i, 1) = FP2(8, i, 1);
    }
    /* thermal: anti-bounce-back (Dirichlet) left/right, bounce-back top/bottom: 2B:776-798 */
    for (int j = 1; j <= ny; ++j) {
        G2(1, 1, j) = -GP2(3, 1, j) + 2.0 * s->omega_T[1] * s->Thot;
        G2(3, nx, j) = -GP2(1, nx, j) + 2.0 * s->omega_T[3] * s->Tcold;
    }
    for (int i = 1; i <= nx; ++i) {
        G2(4, i, ny) = GP2(2, i, ny);
        G2(2, i, 1) = GP2(4, i, 1);
    }
}

#define F3(a, i, j, k) (s->f[NID(s, i, j, k) * 19 + (a)])
#define G3(a, i, j, k) (s->g[NID(s, i, j, k) * 7 + (a)])

static void bounceback_3d(ora_state *s)
{
    int nx = s->nx, ny = s->ny, nz = s->nz;
    /* y walls: 3B:1058-1081 */
    for (int k = 1; k <= nz; ++k)
        for (int i = 1; i <= nx; ++i) {
            F3(3, i, 1, k) = FP3(4, i, 1, k);
            F3(7, i, 1, k) = FP3(10, i, 1, k);
            F3(8, i, 1, k) = FP3(9, i, 1, k);
            F3(15, i, 1, k) = FP3(18, i, 1, k);
            F3(17, i, 1, k) = FP3(16, i, 1, k);
            F3(4, i, ny, k) = FP3(3, i, ny, k);
            F3(9, i, ny, k) = FP3(8, i, ny, k);
            F3(10, i, ny, k) = FP3(7, i, ny, k);
            F3(16, i, ny, k) = FP3(17, i, ny, k);
            F3(18, i, ny, k) = FP3(15, i, ny, k);
        }
    /* x walls: 3B:1084-1107 */
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j) {
            F3(1, 1, j, k) = FP3(2, 1, j, k);
            F3(9, 1, j, k) = FP3(8, 1, j, k);
            F3(7, 1, j, k) = FP3(10, 1, j, k);
            F3(13, 1, j, k) = FP3(12, 1, j, k);
            F3(11, 1, j, k) = FP3(14, 1, j, k);
            F3(2, nx, j, k) = FP3(1, nx, j, k);
            F3(8, nx, j, k) = FP3(9, nx, j, k);
            F3(10, nx, j, k) = FP3(7, nx, j, k);
            F3(12, nx, j, k) = FP3(13, nx, j, k);
            F3(14, nx, j, k) = FP3(11, nx, j, k);
        }
    /* z walls: 3B:1109-1133 */
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            F3(5, i, j, 1) = FP3(6, i, j, 1);
            F3(11, i, j, 1) = FP3(14, i, j, 1);
            F3(12, i, j, 1) = FP3(13, i, j, 1);
            F3(15, i, j, 1) = FP3(18, i, j, 1);
            F3(16, i, j, 1) = FP3(17, i, j, 1);
            F3(6, i, j, nz) = FP3(5, i, j, nz);
            F3(13, i, j, nz) = FP3(12, i, j, nz);
            F3(14, i, j, nz) = FP3(11, i, j, nz);
            F3(17, i, j, nz) = FP3(16, i, j, nz);
            F3(18, i, j, nz) = FP3(15, i, j, nz);
        }
    /* thermal: 3B:1143-1194 (isothermal y walls, adiabatic x and z walls) */
    for (int k = 1; k <= nz; ++k)
        for (int i = 1; i <= nx; ++i) {
            G3(3, i, 1, k) = -GP3(4, i, 1, k) + 2.0 * s->omega_T[3] * s->Thot;
            G3(4, i, ny, k) = -GP3(3, i, ny, k) + 2.0 * s->omega_T[4] * s->Tcold;
        }
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j) {
            G3(1, 1, j, k) = GP3(2, 1, j, k);
            G3(2, nx, j, k) = GP3(1, nx, j, k);
        }
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            G3(5, i, j, 1) = GP3(6, i, j, 1);
            G3(6, i, j, nz) = GP3(5, i, j, nz);
        }
}

/* ------------------------------------------------------------------------ */
/* macro_u / macro_t: 2M:726-753, 3M:988-1025                                */
/* ------------------------------------------------------------------------ */
static void macro_2d(ora_state *s)
{
    const double dt = s->dt;
    #pragma omp parallel for schedule(static)
    for (long id = 0; id < s->nnode; ++id) {
        const double *f = s->f + id * 9, *g = s->g + id * 5;
        double Fx = 0.0, Fy = s->F[id];
        double rho = f[0]+f[1]+f[2]+f[3]+f[4]+f[5]+f[6]+f[7]+f[8];
        s->rho[id] = rho;
        s->u[id] = ( f[1]-f[3]+f[5]-f[6]-f[7]+f[8]+0.5*dt*Fx)/rho;
        s->v[id] = ( f[2]-f[4]+f[5]+f[6]-f[7]-f[8]+0.5*dt*Fy)/rho;
        s->temp[id] = g[0]+g[1]+g[2]+g[3]+g[4];
    }
}

static void macro_3d(ora_state *s)
{
    const double dt = s->dt;
    #pragma omp parallel for schedule(static)
    for (long id = 0; id < s->nnode; ++id) {
        const double *f = s->f + id * 19, *g = s->g + id * 7;
        double rho = f[0]+f[1]+f[2]+f[3]+f[4]+f[5]+f[6]+f[7]+f[8]+f[9]+f[10]+f[11]+f[12]+f[13]+f[14]+f[15]+f[16]+f[17]+f[18];
        s->rho[id] = rho;
        s->u[id] = (f[1]-f[2]+f[7]-f[8]+f[9]-f[10]+f[11]-f[12]+f[13]-f[14])/rho;
        s->v[id] = (f[3]-f[4]+f[7]+f[8]-f[9]-f[10]+f[15]-f[16]+f[17]-f[18])/rho;
        s->w[id] = (f[5]-f[6]+f[11]+f[12]-f[13]-f[14]+f[15]+f[16]-f[17]-f[18]+0.5*dt*s->F[id])/rho;
        s->temp[id] = g[0]+g[1]+g[2]+g[3]+g[4]+g[5]+g[6];
    }
}

/* ------------------------------------------------------------------------ */
/* one loop iteration: 2M:307-330 (itc = itc+1; collision_U; collision_T;    */
/* update [no-op on one domain]; interpolate; bounceback_u; bounceback_T;    */
/* macro_u; macro_t)                                                         */
/* ------------------------------------------------------------------------ */
void ora_step(ora_state *s, int nsteps)
{
    for (int n = 0; n < nsteps; ++n) {
        s->itc += 1;
        if (s->dim == 2) {
            collision_U_2d(s);
            collision_T_2d(s);
            interpolate_2d(s);
            bounceback_2d(s);
            macro_2d(s);
        } else {
            collision_U_3d(s);
            collision_T_3d(s);
            interpolate_3d(s);
            bounceback_3d(s);
            macro_3d(s);
        }
    }
}

/* check: 2M:755-805 (2B:832-884), 3M:1027-1082.  Serial sums in (k, j, i)
 * order, the order of the single-rank loop; copies u -> up, T -> utemp. */
void ora_check(ora_state *s, double *errU, double *errT)
{
    double error1 = 0.0, error2 = 0.0, error3 = 0.0, error4 = 0.0;
    for (long id = 0; id < s->nnode; ++id) {
        double du = s->u[id] - s->up[id], dv = s->v[id] - s->vp[id];
        if (s->dim == 2) {
            error1 = error1 + du * du + dv * dv;
            error2 = error2 + s->u[id] * s->u[id] + s->v[id] * s->v[id];
        } else {
            double dw = s->w[id] - s->wp[id];
            error1 = error1 + du * du + dv * dv + dw * dw;
            error2 = error2 + s->u[id] * s->u[id] + s->v[id] * s->v[id] + s->w[id] * s->w[id];
        }
        s->up[id] = s->u[id];
        s->vp[id] = s->v[id];
        s->wp[id] = s->w[id];
    }
    *errU = sqrt(error1) / sqrt(error2);
    for (long id = 0; id < s->nnode; ++id) {
        double dT = s->temp[id] - s->utemp[id];
        error3 = error3 + dT * dT;
        error4 = error4 + s->temp[id] * s->temp[id];
        s->utemp[id] = s->temp[id];
    }
    *errT = sqrt(error3) / sqrt(error4);
}

/* ------------------------------------------------------------------------ */
/* Nusselt number and conservation sums.  The reference has no such         */
/* function; the definitions are shared, term for term, with the GPU path.  */
/*   walls: the halfway bounce-back wall lies dt/2 outside the first/last   */
/*     node: w_lo = c(1) - dt/2, w_hi = c(n) + dt/2;                         */
/*   cell widths: node 1 owns [w_lo, (c1+c2)/2], node n [(c(n-1)+c(n))/2,   */
/*     w_hi], others the midpoints either side;                              */
/*   local Nu = -(L_LB-1)/(Thot-Tcold) * dT/dn at the wall, dT/dn from the   */
/*     quadratic through (wall, T_wall), (node 1, T1), (node 2, T2) along the */
/*     heated axis (x in 2D, y in 3D), the wall temperature being Thot / Tcold;*/
/*   Nu_avg = sum(Nu * cell width [* cell depth]) / sum(widths [* depths]).  */
/* ------------------------------------------------------------------------ */
void ora_cell_widths(const double *c, int n, double dt, double *wd)
{
    double lo = c[1] - 0.5 * dt, hi = c[n] + 0.5 * dt;
    for (int i = 1; i <= n; ++i) {
        double a = (i == 1) ? lo : 0.5 * (c[i - 1] + c[i]);
        double b = (i == n) ? hi : 0.5 * (c[i] + c[i + 1]);
        wd[i - 1] = b - a;
    }
}

/* d/dx at xw of the quadratic through (xw,Tw), (x1,T1), (x2,T2) */
double ora_wall_gradient(double xw, double Tw, double x1, double T1, double x2, double T2)
{
    double d0 = ((xw - x1) + (xw - x2)) / ((xw - x1) * (xw - x2));
    double d1 = (xw - x2) / ((x1 - xw) * (x1 - x2));
    double d2 = (xw - x1) / ((x2 - xw) * (x2 - x1));
    return d0 * Tw + d1 * T1 + d2 * T2;
}

void ora_nusselt(ora_state *s, double *nu_hot, double *nu_cold)
{
    double scale = -(s->length_LB - 1.0) / (s->Thot - s->Tcold);
    double sh = 0.0, sc = 0.0, area = 0.0;
    if (s->dim == 2) {
        int nx = s->nx, ny = s->ny;
        double *wy = (double *)malloc(sizeof(double) * ny);
        ora_cell_widths(s->y, ny, s->dt, wy);
        double xlo = s->x[1] - 0.5 * s->dt, xhi = s->x[nx] + 0.5 * s->dt;
        for (int j = 1; j <= ny; ++j) {
            double gh = ora_wall_gradient(xlo, s->Thot, s->x[1], s->temp[NID(s, 1, j, 1)],
                                          s->x[2], s->temp[NID(s, 2, j, 1)]);
            double gc = ora_wall_gradient(xhi, s->Tcold, s->x[nx], s->temp[NID(s, nx, j, 1)],
                                          s->x[nx - 1], s->temp[NID(s, nx - 1, j, 1)]);
            sh += scale * gh * wy[j - 1];
            sc += scale * gc * wy[j - 1];
            area += wy[j - 1];
        }
        free(wy);
    } else {
        int nx = s->nx, ny = s->ny, nz = s->nz;
        double *wx = (double *)malloc(sizeof(double) * nx);
        double *wz = (double *)malloc(sizeof(double) * nz);
        ora_cell_widths(s->x, nx, s->dt, wx);
        ora_cell_widths(s->z, nz, s->dt, wz);
        double ylo = s->y[1] - 0.5 * s->dt, yhi = s->y[ny] + 0.5 * s->dt;
        for (int k = 1; k <= nz; ++k)
            for (int i = 1; i <= nx; ++i) {
                double gh = ora_wall_gradient(ylo, s->Thot, s->y[1], s->temp[NID(s, i, 1, k)],
                                              s->y[2], s->temp[NID(s, i, 2, k)]);
                double gc = ora_wall_gradient(yhi, s->Tcold, s->y[ny], s->temp[NID(s, i, ny, k)],
                                              s->y[ny - 1], s->temp[NID(s, i, ny - 1, k)]);
                double a = wx[i - 1] * wz[k - 1];
                sh += scale * gh * a;
                sc += scale * gc * a;
                area += a;
            }
        free(wx);
        free(wz);
    }
    *nu_hot = sh / area;
    *nu_cold = sc / area;
}

/* mass = sum(rho * cell volume), energy = sum(T * cell volume) */
void ora_sums(ora_state *s, double *mass, double *energy)
{
    int nx = s->nx, ny = s->ny, nz = s->nz;
    double *wx = (double *)malloc(sizeof(double) * nx);
    double *wy = (double *)malloc(sizeof(double) * ny);
    double *wz = (double *)malloc(sizeof(double) * nz);
    ora_cell_widths(s->x, nx, s->dt, wx);
    ora_cell_widths(s->y, ny, s->dt, wy);
    if (s->dim == 3) ora_cell_widths(s->z, nz, s->dt, wz); else wz[0] = 1.0;
    double m = 0.0, e = 0.0;
    for (int k = 1; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                long id = NID(s, i, j, k);
                double vol = wx[i - 1] * wy[j - 1] * wz[k - 1];
                m += s->rho[id] * vol;
                e += s->temp[id] * vol;
            }
    free(wx); free(wy); free(wz);
    *mass = m;
    *energy = e;
}

/* ------------------------------------------------------------------------ */
/* accessors for the ctypes wrapper                                          */
/* ------------------------------------------------------------------------ */
double *ora_ptr(ora_state *s, int which)
{
    switch (which) {
    case 0: return s->f;
    case 1: return s->f_post;
    case 2: return s->g;
    case 3: return s->g_post;
    case 4: return s->rho;
    case 5: return s->u;
    case 6: return s->v;
    case 7: return s->w;
    case 8: return s->temp;
    case 9: return s->F;
    case 10: return s->x;
    case 11: return s->y;
    case 12: return s->z;
    default: return 0;
    }
}

/* params: 0 viscosity_LB, 1 kappa, 2 gbeta, 3 tauf, 4 Snu, 5 Sq, 6 sig_k, 7 dt, 8 length_LB */
void ora_params(ora_state *s, double *out)
{
    out[0] = s->viscosity_LB; out[1] = s->kappa; out[2] = s->gbeta; out[3] = s->tauf;
    out[4] = s->Snu; out[5] = s->Sq; out[6] = s->sig_k; out[7] = s->dt; out[8] = s->length_LB;
}

long ora_itc(ora_state *s) { return s->itc; }

void ora_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int ora_get_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
