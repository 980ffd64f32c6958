/*
 * pictor_oracle.c -- CPU restatement (FP64) of PICTOR's Cartesian PIC step.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never part of it.
 * Parity against the reference itself is UNPINNED (the reference is Fortran,
 * has no tests or golden vectors, and cannot be compiled here); the
 * restatement is pinned to hand-derived known-answer vectors instead.
 *
 * Every routine follows the reference loop for loop and keeps its order of
 * floating-point operations (Fortran evaluates a+b+c as (a+b)+c and a*b*c as
 * (a*b)*c), so that with -ffp-contract=off the results are those of the
 * reference CPU build compiled without FMA contraction.  File:line citations
 * are relative to the reference project root.
 */
#include "pictor_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* 1-based (i,j,k) -> 0-based column-major offset. */
#define ID(g, i, j, k) ((int64_t)((i) - 1) + (int64_t)(g)->mx * ((int64_t)((j) - 1) + (int64_t)(g)->my * (int64_t)((k) - 1)))

static const double PI_PSN = 3.14159265358979323846264; /* vars.F90:224 */

void orc_grid_init(orc_grid *g)
{
    g->mx = g->nx + 5;
    g->my = g->ny + 5;
    g->mz = (g->dims == 2) ? 1 : g->nz + 5;
}

/* ------------------------------------------------------------------------- */
/* Field solver: em_update.F90 (Yee) and em_update_lehe.F90 (Lehe)            */
/* ------------------------------------------------------------------------- */

/* em_update_lehe.F90:8-25 (Fortran parameters; grid_dx=dy=dz=1). */
void orc_lehe_coefficients(const orc_grid *g, double o[12])
{
    const double c = g->c;
    const double cinv = 1.0 / c;                         /* vars.F90:222 */
    const double beta_xy = 0.125 * (1.0 * 1.0);
    const double beta_xz = 0.125 * (1.0 * 1.0);
    const double beta_yx = 0.125, beta_yz = 0.0, beta_zx = 0.125, beta_zy = 0.0;
    const double s = sin((0.5 * PI_PSN) * c);
    const double delta_x = 0.25 * (1.0 - (cinv * cinv) * (s * s));
    const double delta_y = 0.0, delta_z = 0.0;
    double ax, ay, az;
    if (g->dims == 3) {
        ax = ((1.0 - 2.0 * beta_xy) - 2.0 * beta_xz) - 3.0 * delta_x;
        ay = ((1.0 - 2.0 * beta_yx) - 2.0 * beta_yz) - 3.0 * delta_y;
        az = ((1.0 - 2.0 * beta_zx) - 2.0 * beta_zy) - 3.0 * delta_z;
    } else {
        ax = (1.0 - 2.0 * beta_xy) - 3.0 * delta_x;
        ay = (1.0 - 2.0 * beta_yx) - 3.0 * delta_y;
        az = 1.0;
    }
    o[0] = ax; o[1] = ay; o[2] = az;
    o[3] = beta_xy; o[4] = beta_xz; o[5] = beta_yx; o[6] = beta_yz; o[7] = beta_zx; o[8] = beta_zy;
    o[9] = delta_x; o[10] = delta_y; o[11] = delta_z;
}

/* em_update_lehe.F90:223-258 (inv_d = 1). */
static double gradX(const orc_grid *g, const double *L, const double *F, int i, int j, int k)
{
    double r = L[0] * (F[ID(g, i + 1, j, k)] - F[ID(g, i, j, k)]);
    r = r + L[3] * (F[ID(g, i + 1, j + 1, k)] - F[ID(g, i, j + 1, k)]);
    r = r + L[3] * (F[ID(g, i + 1, j - 1, k)] - F[ID(g, i, j - 1, k)]);
    if (g->dims == 3) {
        r = r + L[4] * (F[ID(g, i + 1, j, k + 1)] - F[ID(g, i, j, k + 1)]);
        r = r + L[4] * (F[ID(g, i + 1, j, k - 1)] - F[ID(g, i, j, k - 1)]);
    }
    r = r + L[9] * (F[ID(g, i + 2, j, k)] - F[ID(g, i - 1, j, k)]);
    return r;
}

static double gradY(const orc_grid *g, const double *L, const double *F, int i, int j, int k)
{
    double r = L[1] * (F[ID(g, i, j + 1, k)] - F[ID(g, i, j, k)]);
    r = r + L[5] * (F[ID(g, i + 1, j + 1, k)] - F[ID(g, i + 1, j, k)]);
    r = r + L[5] * (F[ID(g, i - 1, j + 1, k)] - F[ID(g, i - 1, j, k)]);
    if (g->dims == 3) {
        r = r + L[6] * (F[ID(g, i, j + 1, k + 1)] - F[ID(g, i, j, k + 1)]);
        r = r + L[6] * (F[ID(g, i, j + 1, k - 1)] - F[ID(g, i, j, k - 1)]);
    }
    r = r + L[10] * (F[ID(g, i, j + 2, k)] - F[ID(g, i, j - 1, k)]);
    return r;
}

static double gradZ(const orc_grid *g, const double *L, const double *F, int i, int j, int k)
{
    double r = L[2] * (F[ID(g, i, j, k + 1)] - F[ID(g, i, j, k)]);
    r = r + L[7] * (F[ID(g, i + 1, j, k + 1)] - F[ID(g, i + 1, j, k)]);
    r = r + L[7] * (F[ID(g, i - 1, j, k + 1)] - F[ID(g, i - 1, j, k)]);
    r = r + L[8] * (F[ID(g, i, j + 1, k + 1)] - F[ID(g, i, j + 1, k)]);
    r = r + L[8] * (F[ID(g, i, j - 1, k + 1)] - F[ID(g, i, j - 1, k)]);
    r = r + L[11] * (F[ID(g, i, j, k + 2)] - F[ID(g, i, j, k - 1)]);
    return r;
}

/* em_update.F90:41-77 (Yee) / em_update_lehe.F90:191-221 (Lehe). */
void orc_update_b_half(const orc_grid *g, orc_fields *f)
{
    const double h = (g->c * 0.5) * 1.0; /* fld_halfc, vars.F90:221 */
    const double *Ex = f->Ex, *Ey = f->Ey, *Ez = f->Ez;
    double *Bx = f->Bx, *By = f->By, *Bz = f->Bz;
    if (g->fdtd == 0) {
        const int k1 = g->dims == 3 ? 2 : 1, k2 = g->dims == 3 ? g->mz - 1 : 1;
        for (int k = k1; k <= k2; k++)
            for (int j = 2; j <= g->my - 1; j++)
                for (int i = 2; i <= g->mx - 1; i++) {
                    const int64_t c0 = ID(g, i, j, k);
                    if (g->dims == 3) {
                        Bx[c0] = (Bx[c0] - h * (Ez[ID(g, i, j + 1, k)] - Ez[c0])) + h * (Ey[ID(g, i, j, k + 1)] - Ey[c0]);
                        By[c0] = (By[c0] - h * (Ex[ID(g, i, j, k + 1)] - Ex[c0])) + h * (Ez[ID(g, i + 1, j, k)] - Ez[c0]);
                        Bz[c0] = (Bz[c0] - h * (Ey[ID(g, i + 1, j, k)] - Ey[c0])) + h * (Ex[ID(g, i, j + 1, k)] - Ex[c0]);
                    } else {
                        Bx[c0] = Bx[c0] - h * (Ez[ID(g, i, j + 1, k)] - Ez[c0]);
                        By[c0] = By[c0] + h * (Ez[ID(g, i + 1, j, k)] - Ez[c0]);
                        Bz[c0] = (Bz[c0] - h * (Ey[ID(g, i + 1, j, k)] - Ey[c0])) + h * (Ex[ID(g, i, j + 1, k)] - Ex[c0]);
                    }
                }
    } else {
        double L[12];
        orc_lehe_coefficients(g, L);
        const int k1 = g->dims == 3 ? 3 : 1, k2 = g->dims == 3 ? g->mz - 3 : 1;
        for (int k = k1; k <= k2; k++)
            for (int j = 3; j <= g->my - 3; j++)
                for (int i = 3; i <= g->mx - 3; i++) {
                    const int64_t c0 = ID(g, i, j, k);
                    if (g->dims == 3) {
                        Bx[c0] = (Bx[c0] - h * gradY(g, L, Ez, i, j, k)) + h * gradZ(g, L, Ey, i, j, k);
                        By[c0] = (By[c0] - h * gradZ(g, L, Ex, i, j, k)) + h * gradX(g, L, Ez, i, j, k);
                        Bz[c0] = (Bz[c0] - h * gradX(g, L, Ey, i, j, k)) + h * gradY(g, L, Ex, i, j, k);
                    } else {
                        Bx[c0] = Bx[c0] - h * gradY(g, L, Ez, i, j, k);
                        By[c0] = By[c0] + h * gradX(g, L, Ez, i, j, k);
                        Bz[c0] = (Bz[c0] - h * gradX(g, L, Ey, i, j, k)) + h * gradY(g, L, Ex, i, j, k);
                    }
                }
    }
}

/* em_update.F90:9-39 (Yee loops 2..m-1) / em_update_lehe.F90:146-187 (3..m-3). */
void orc_update_e(const orc_grid *g, orc_fields *f)
{
    const double fc = g->c * 1.0; /* fldc, vars.F90:220 */
    double *Ex = f->Ex, *Ey = f->Ey, *Ez = f->Ez;
    const double *Bx = f->Bx, *By = f->By, *Bz = f->Bz;
    const int lo = g->fdtd == 0 ? 2 : 3;
    const int k1 = g->dims == 3 ? lo : 1, k2 = g->dims == 3 ? (g->fdtd == 0 ? g->mz - 1 : g->mz - 3) : 1;
    const int jhi = g->fdtd == 0 ? g->my - 1 : g->my - 3, ihi = g->fdtd == 0 ? g->mx - 1 : g->mx - 3;
    for (int k = k1; k <= k2; k++)
        for (int j = lo; j <= jhi; j++)
            for (int i = lo; i <= ihi; i++) {
                const int64_t c0 = ID(g, i, j, k);
                if (g->dims == 3) {
                    Ex[c0] = (Ex[c0] + fc * (Bz[c0] - Bz[ID(g, i, j - 1, k)])) - fc * (By[c0] - By[ID(g, i, j, k - 1)]);
                    Ey[c0] = (Ey[c0] + fc * (Bx[c0] - Bx[ID(g, i, j, k - 1)])) - fc * (Bz[c0] - Bz[ID(g, i - 1, j, k)]);
                    Ez[c0] = (Ez[c0] + fc * (By[c0] - By[ID(g, i - 1, j, k)])) - fc * (Bx[c0] - Bx[ID(g, i, j - 1, k)]);
                } else {
                    Ex[c0] = Ex[c0] + fc * (Bz[c0] - Bz[ID(g, i, j - 1, k)]);
                    Ey[c0] = Ey[c0] - fc * (Bz[c0] - Bz[ID(g, i - 1, j, k)]);
                    Ez[c0] = (Ez[c0] + fc * (By[c0] - By[ID(g, i - 1, j, k)])) - fc * (Bx[c0] - Bx[ID(g, i, j - 1, k)]);
                }
            }
}

/* em_update.F90:79-102 (identical in em_update_lehe.F90:264-287). */
void orc_add_current(const orc_grid *g, orc_fields *f)
{
    const int k1 = g->dims == 3 ? 3 : 1, k2 = g->dims == 3 ? g->mz - 3 : 1;
    for (int k = k1; k <= k2; k++)
        for (int j = 3; j <= g->my - 3; j++)
            for (int i = 3; i <= g->mx - 3; i++) {
                const int64_t c0 = ID(g, i, j, k);
                f->Ex[c0] = f->Ex[c0] - (f->Jx[c0] * 1.0) * 1.0;
                f->Ey[c0] = f->Ey[c0] - (f->Jy[c0] * 1.0) * 1.0;
                f->Ez[c0] = f->Ez[c0] - (f->Jz[c0] * 1.0) * 1.0;
            }
}

void orc_reset_current(const orc_grid *g, orc_fields *f)
{
    const size_t n = (size_t)g->mx * g->my * g->mz;
    memset(f->Jx, 0, n * sizeof(double));
    memset(f->Jy, 0, n * sizeof(double));
    memset(f->Jz, 0, n * sizeof(double));
}

/* ------------------------------------------------------------------------- */
/* Periodic single-rank halo copy and current fold (comm_fld.F90)            */
/* ------------------------------------------------------------------------- */

/* Copy along one axis: high ghosts m-2..m <- 3..5, low ghosts 1..2 <- m-4..m-3
   (layer map of subdomains.F90:592-612 with the neighbour being this rank).
   lo/hi give the index ranges of the two other axes. */
static void halo_axis(const orc_grid *g, double *F, int axis, const int lo[3], const int hi[3])
{
    const int m = axis == 0 ? g->mx : axis == 1 ? g->my : g->mz;
    for (int k = lo[2]; k <= hi[2]; k++)
        for (int j = lo[1]; j <= hi[1]; j++)
            for (int i = lo[0]; i <= hi[0]; i++) {
                int idx[3] = {i, j, k};
                if (idx[axis] != 1) continue; /* iterate the layer axis below */
                for (int l = 0; l < 3; l++) {
                    int d[3] = {i, j, k}, s[3] = {i, j, k};
                    d[axis] = m - 2 + l; s[axis] = 3 + l;
                    F[ID(g, d[0], d[1], d[2])] = F[ID(g, s[0], s[1], s[2])];
                }
                for (int l = 0; l < 2; l++) {
                    int d[3] = {i, j, k}, s[3] = {i, j, k};
                    d[axis] = 1 + l; s[axis] = m - 4 + l;
                    F[ID(g, d[0], d[1], d[2])] = F[ID(g, s[0], s[1], s[2])];
                }
            }
}

/* comm_fld.F90:75-130: y faces (x range 3..mx-3), then z faces (3D), then x
   faces over the full y,z range. */
void orc_send_recv_flds(const orc_grid *g, double *Fx, double *Fy, double *Fz)
{
    double *F[3] = {Fx, Fy, Fz};
    for (int c = 0; c < 3; c++) {
        int lo[3] = {3, 1, 1}, hi[3] = {g->mx - 3, 1, g->mz};
        halo_axis(g, F[c], 1, lo, hi);
        if (g->dims == 3) {
            int lo2[3] = {3, 1, 1}, hi2[3] = {g->mx - 3, g->my, 1};
            halo_axis(g, F[c], 2, lo2, hi2);
        }
        int lo3[3] = {1, 1, 1}, hi3[3] = {1, g->my, g->mz};
        halo_axis(g, F[c], 0, lo3, hi3);
    }
}

/* Fold along one axis: 3..5 += m-2..m and m-4..m-3 += 1..2 (AddBuffToFld,
   comm_fld.F90:288-307, with the neighbour being this rank). */
static void fold_axis(const orc_grid *g, double *F, int axis, const int lo[3], const int hi[3])
{
    const int m = axis == 0 ? g->mx : axis == 1 ? g->my : g->mz;
    for (int k = lo[2]; k <= hi[2]; k++)
        for (int j = lo[1]; j <= hi[1]; j++)
            for (int i = lo[0]; i <= hi[0]; i++) {
                double buf_hi[3], buf_lo[2];
                for (int l = 0; l < 3; l++) {
                    int s[3] = {i, j, k};
                    s[axis] = m - 2 + l;
                    buf_hi[l] = F[ID(g, s[0], s[1], s[2])];
                }
                for (int l = 0; l < 2; l++) {
                    int s[3] = {i, j, k};
                    s[axis] = 1 + l;
                    buf_lo[l] = F[ID(g, s[0], s[1], s[2])];
                }
                for (int l = 0; l < 3; l++) {
                    int d[3] = {i, j, k};
                    d[axis] = 3 + l;
                    F[ID(g, d[0], d[1], d[2])] = F[ID(g, d[0], d[1], d[2])] + buf_hi[l];
                }
                for (int l = 0; l < 2; l++) {
                    int d[3] = {i, j, k};
                    d[axis] = m - 4 + l;
                    F[ID(g, d[0], d[1], d[2])] = F[ID(g, d[0], d[1], d[2])] + buf_lo[l];
                }
            }
}

/* comm_fld.F90:15-33: x faces (full y,z), then y faces (x 3..mx-3), then z. */
void orc_update_current_all_faces(const orc_grid *g, double *Jx, double *Jy, double *Jz)
{
    double *F[3] = {Jx, Jy, Jz};
    for (int c = 0; c < 3; c++) {
        int lo[3] = {1, 1, 1}, hi[3] = {1, g->my, g->mz};
        fold_axis(g, F[c], 0, lo, hi);
    }
    for (int c = 0; c < 3; c++) {
        int lo[3] = {3, 1, 1}, hi[3] = {g->mx - 3, 1, g->mz};
        fold_axis(g, F[c], 1, lo, hi);
    }
    if (g->dims == 3)
        for (int c = 0; c < 3; c++) {
            int lo[3] = {3, 1, 1}, hi[3] = {g->mx - 3, g->my, 1};
            fold_axis(g, F[c], 2, lo, hi);
        }
}

/* current.F90:55-163 MovingAverageFilter on one periodic rank: before each
   axis pass the halo of that axis is refreshed (SendRecvFldsYZ / ZX / XY),
   then F = wtm1*F(-1) + wt0*F + wtp1*F(+1) over 2..m-2 (2D k = 1). */
static void moving_average_axis(const orc_grid *g, double *F, int axis)
{
    const size_t n = (size_t)g->mx * g->my * g->mz;
    double *tmp = (double *)malloc(n * sizeof(double));
    memcpy(tmp, F, n * sizeof(double));
    const int k1 = g->dims == 3 ? 2 : 1, k2 = g->dims == 3 ? g->mz - 2 : 1;
    for (int k = k1; k <= k2; k++)
        for (int j = 2; j <= g->my - 2; j++)
            for (int i = 2; i <= g->mx - 2; i++) {
                int lo[3] = {i, j, k}, hi[3] = {i, j, k};
                lo[axis] -= 1;
                hi[axis] += 1;
                tmp[ID(g, i, j, k)] = (0.25 * F[ID(g, lo[0], lo[1], lo[2])] + 0.5 * F[ID(g, i, j, k)]) +
                                      0.25 * F[ID(g, hi[0], hi[1], hi[2])];
            }
    for (int k = k1; k <= k2; k++)
        for (int j = 2; j <= g->my - 2; j++)
            for (int i = 2; i <= g->mx - 2; i++) F[ID(g, i, j, k)] = tmp[ID(g, i, j, k)];
    free(tmp);
}

void orc_filter_current(const orc_grid *g, double *Jx, double *Jy, double *Jz, int passes)
{
    double *F[3] = {Jx, Jy, Jz};
    for (int ps = 0; ps < passes; ps++) {                        /* smoothen_current, current.F90:19-30 */
        for (int c = 0; c < 3; c++) {
            int lo[3] = {1, 1, 1}, hi[3] = {1, g->my, g->mz};
            halo_axis(g, F[c], 0, lo, hi);                       /* SendRecvFldsYZ */
        }
        for (int c = 0; c < 3; c++) moving_average_axis(g, F[c], 0);
        for (int c = 0; c < 3; c++) {
            int lo[3] = {3, 1, 1}, hi[3] = {g->mx - 3, 1, g->mz};
            halo_axis(g, F[c], 1, lo, hi);                       /* SendRecvFldsZX */
        }
        for (int c = 0; c < 3; c++) moving_average_axis(g, F[c], 1);
        if (g->dims == 3) {
            for (int c = 0; c < 3; c++) {
                int lo[3] = {3, 1, 1}, hi[3] = {g->mx - 3, g->my, 1};
                halo_axis(g, F[c], 2, lo, hi);                   /* SendRecvFldsXY */
            }
            for (int c = 0; c < 3; c++) moving_average_axis(g, F[c], 2);
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Mover + deposit: movdep.F90:12-258, movdep_routines.F90:6-311             */
/* ------------------------------------------------------------------------- */

/* GatherVecEfld / GatherVecBfld, movdep_routines.F90:6-223: node values of a
   component at the 4 (2D) or 8 (3D) corners of cell (i,j,k), corner order
   nn = (0,0,0),(1,0,0),(0,1,0),(1,1,0),(0,0,1),... */
static void node_values(const orc_grid *g, const orc_fields *f, int i, int j, int k, double V[6][8])
{
    const int nc = g->dims == 3 ? 8 : 4;
    for (int nn = 0; nn < nc; nn++) {
        const int a = i + (nn & 1), b = j + ((nn >> 1) & 1), c = k + ((nn >> 2) & 1);
        V[0][nn] = (f->Ex[ID(g, a - 1, b, c)] + f->Ex[ID(g, a, b, c)]) * 0.5;
        V[1][nn] = (f->Ey[ID(g, a, b - 1, c)] + f->Ey[ID(g, a, b, c)]) * 0.5;
        if (g->dims == 3) {
            V[2][nn] = (f->Ez[ID(g, a, b, c - 1)] + f->Ez[ID(g, a, b, c)]) * 0.5;
            V[3][nn] = (((f->Bx[ID(g, a, b - 1, c - 1)] + f->Bx[ID(g, a, b, c - 1)]) + f->Bx[ID(g, a, b - 1, c)]) + f->Bx[ID(g, a, b, c)]) * 0.25 + g->bext[0];
            V[4][nn] = (((f->By[ID(g, a - 1, b, c - 1)] + f->By[ID(g, a - 1, b, c)]) + f->By[ID(g, a, b, c - 1)]) + f->By[ID(g, a, b, c)]) * 0.25 + g->bext[1];
        } else {
            V[2][nn] = f->Ez[ID(g, a, b, c)];
            V[3][nn] = (f->Bx[ID(g, a, b - 1, c)] + f->Bx[ID(g, a, b, c)]) * 0.5 + g->bext[0];
            V[4][nn] = (f->By[ID(g, a - 1, b, c)] + f->By[ID(g, a, b, c)]) * 0.5 + g->bext[1];
        }
        V[5][nn] = (((f->Bz[ID(g, a - 1, b - 1, c)] + f->Bz[ID(g, a - 1, b, c)]) + f->Bz[ID(g, a, b - 1, c)]) + f->Bz[ID(g, a, b, c)]) * 0.25 + g->bext[2];
    }
}

typedef struct {
    int64_t cell;  /* VecJ column (1-based short_arr_ind)                */
    double val[12];
} vecj_contrib;

/* The 8 (2D) or 12 (3D) VecJ entries of one zigzag segment, with the
   wtF/Jwt tables of vars.F90:328-355 expanded.  Products are left to right
   as in movdep.F90:209,233. */
static void segment_values(int dims, double Fx, double Fy, double Fz, double Wx, double Wy, double Wz, double out[12])
{
    if (dims == 2) {
        out[0] = ((Fx * 1.0) * (1.0 - Wy)) * 1.0;
        out[1] = ((Fx * 1.0) * Wy) * 1.0;
        out[2] = ((Fy * (1.0 - Wx)) * 1.0) * 1.0;
        out[3] = ((Fy * Wx) * 1.0) * 1.0;
        out[4] = ((Fz * (1.0 - Wx)) * (1.0 - Wy)) * 1.0;
        out[5] = ((Fz * Wx) * (1.0 - Wy)) * 1.0;
        out[6] = ((Fz * (1.0 - Wx)) * Wy) * 1.0;
        out[7] = ((Fz * Wx) * Wy) * 1.0;
    } else {
        out[0] = ((Fx * 1.0) * (1.0 - Wy)) * (1.0 - Wz);
        out[1] = ((Fx * 1.0) * Wy) * (1.0 - Wz);
        out[2] = ((Fx * 1.0) * (1.0 - Wy)) * Wz;
        out[3] = ((Fx * 1.0) * Wy) * Wz;
        out[4] = ((Fy * (1.0 - Wx)) * 1.0) * (1.0 - Wz);
        out[5] = ((Fy * Wx) * 1.0) * (1.0 - Wz);
        out[6] = ((Fy * (1.0 - Wx)) * 1.0) * Wz;
        out[7] = ((Fy * Wx) * 1.0) * Wz;
        out[8] = ((Fz * (1.0 - Wx)) * (1.0 - Wy)) * 1.0;
        out[9] = ((Fz * Wx) * (1.0 - Wy)) * 1.0;
        out[10] = ((Fz * (1.0 - Wx)) * Wy) * 1.0;
        out[11] = ((Fz * Wx) * Wy) * 1.0;
    }
}

/* Per-particle body of movdep.F90:68-249.  Appends the two deposit segments
   to VecJ (thread slice vj), or, with rec != NULL, stores them as the two
   records rec[0], rec[1] (cell and values) for a later ordered sum. */
static void move_one(const orc_grid *g, orc_particles *p, const orc_fields *f, int64_t n, double *vj,
                     vecj_contrib *rec)
{
    const int nc = g->dims == 3 ? 8 : 4, nj = g->dims == 3 ? 12 : 8;
    const double c = g->c, sqc = c * c, cinv = 1.0 / c;
    const double x0 = p->x[n], y0 = p->y[n], z0 = p->z[n];
    const double qm = p->flv[n] == 0 ? 0.0 : g->flvrqm[p->flv[n]] * 0.5;     /* :74-80 */
    const int ip0 = (int)x0, jp0 = (int)y0, kp0 = (int)z0;                     /* :89-91 */
    const double dx = x0 - ip0, dy = y0 - jp0;
    double wt[8];
    if (g->dims == 3) {
        const double dz = z0 - kp0;
        for (int nn = 0; nn < 8; nn++) {
            const double wx = (nn & 1) ? (0.0 + 1.0 * dx) : (1.0 + -1.0 * dx);
            const double wy = (nn & 2) ? (0.0 + 1.0 * dy) : (1.0 + -1.0 * dy);
            const double wz = (nn & 4) ? (0.0 + 1.0 * dz) : (1.0 + -1.0 * dz);
            wt[nn] = (wx * wy) * wz;
        }
    } else {
        for (int nn = 0; nn < 4; nn++) {
            const double wx = (nn & 1) ? (0.0 + 1.0 * dx) : (1.0 + -1.0 * dx);
            const double wy = (nn & 2) ? (0.0 + 1.0 * dy) : (1.0 + -1.0 * dy);
            wt[nn] = wx * wy;
        }
    }
    double V[6][8];
    node_values(g, f, ip0, jp0, g->dims == 3 ? kp0 : 1, V);
    double pE[3] = {0, 0, 0}, pB[3] = {0, 0, 0};
    for (int nn = 0; nn < nc; nn++) {                                          /* :116-129 */
        pE[0] = pE[0] + wt[nn] * V[0][nn];
        pE[1] = pE[1] + wt[nn] * V[1][nn];
        pE[2] = pE[2] + wt[nn] * V[2][nn];
        pB[0] = pB[0] + wt[nn] * V[3][nn];
        pB[1] = pB[1] + wt[nn] * V[4][nn];
        pB[2] = pB[2] + wt[nn] * V[5][nn];
    }
    for (int d = 0; d < 3; d++) { pE[d] = pE[d] * qm; pB[d] = pB[d] * qm; } /* :134-139 */

    /* Boris push, movdep.F90:143-173 */
    double u0 = c * p->u[n] + pE[0];
    double v0 = c * p->v[n] + pE[1];
    double w0 = c * p->w[n] + pE[2];
    double gg = 1.0 / sqrt(((sqc + u0 * u0) + v0 * v0) + w0 * w0);
    const double bx = gg * pB[0], by = gg * pB[1], bz = gg * pB[2];
    const double ff = 2.0 / (((1.0 + bx * bx) + by * by) + bz * bz);
    const double u1 = ((u0 + v0 * bz) - w0 * by) * ff;
    const double v1 = ((v0 + w0 * bx) - u0 * bz) * ff;
    const double w1 = ((w0 + u0 * by) - v0 * bx) * ff;
    u0 = ((u0 + v1 * bz) - w1 * by) + pE[0];
    v0 = ((v0 + w1 * bx) - u1 * bz) + pE[1];
    w0 = ((w0 + u1 * by) - v1 * bx) + pE[2];
    p->u[n] = u0 * cinv;
    p->v[n] = v0 * cinv;
    p->w[n] = w0 * cinv;
    gg = sqc / sqrt(((sqc + u0 * u0) + v0 * v0) + w0 * w0);
    const double x1 = p->x[n] + (p->u[n] * gg) * 1.0;
    const double y1 = p->y[n] + (p->v[n] * gg) * 1.0;
    const double z1 = p->z[n] + (p->w[n] * gg) * 1.0;
    p->x[n] = x1; p->y[n] = y1; p->z[n] = z1;

    /* zigzag deposit, movdep.F90:177-237 */
    const int ip = (int)x1, jp = (int)y1, kp = (int)z1;
    const double xr = fmin((double)((ip0 < ip ? ip0 : ip) + 1), fmax((double)(ip0 > ip ? ip0 : ip), 0.5 * (x0 + x1)));
    const double yr = fmin((double)((jp0 < jp ? jp0 : jp) + 1), fmax((double)(jp0 > jp ? jp0 : jp), 0.5 * (y0 + y1)));
    const double zr = fmin((double)((kp0 < kp ? kp0 : kp) + 1), fmax((double)(kp0 > kp ? kp0 : kp), 0.5 * (z0 + z1)));
    const double qthis = p->q[n] * g->qi;
    double seg[12];
    {
        const double Fx1 = qthis * (xr - x0), Fy1 = qthis * (yr - y0), Fz1 = qthis * (zr - z0);
        const double Wx1 = 0.5 * (x0 + xr) - ip0, Wy1 = 0.5 * (y0 + yr) - jp0;
        const double Wz1 = g->dims == 3 ? 0.5 * (z0 + zr) - kp0 : 0.0;
        const int64_t cell = g->dims == 3 ? ID(g, ip0, jp0, kp0) : ID(g, ip0, jp0, 1);
        segment_values(g->dims, Fx1, Fy1, Fz1, Wx1, Wy1, Wz1, seg);
        if (rec) {
            rec[0].cell = cell;
            memcpy(rec[0].val, seg, sizeof(seg));
        } else {
            for (int nn = 0; nn < nj; nn++) vj[cell * nj + nn] = vj[cell * nj + nn] + seg[nn];
        }
    }
    {
        const double Fx2 = qthis * (x1 - xr), Fy2 = qthis * (y1 - yr), Fz2 = qthis * (z1 - zr);
        const double Wx2 = 0.5 * (x1 + xr) - ip, Wy2 = 0.5 * (y1 + yr) - jp;
        const double Wz2 = g->dims == 3 ? 0.5 * (z1 + zr) - kp : 0.0;
        const int64_t cell = g->dims == 3 ? ID(g, ip, jp, kp) : ID(g, ip, jp, 1);
        segment_values(g->dims, Fx2, Fy2, Fz2, Wx2, Wy2, Wz2, seg);
        if (rec) {
            rec[1].cell = cell;
            memcpy(rec[1].val, seg, sizeof(seg));
        } else {
            for (int nn = 0; nn < nj; nn++) vj[cell * nj + nn] = vj[cell * nj + nn] + seg[nn];
        }
    }
    /* 2D periodic z, movdep.F90:241-249 (zmin=1, zmax=2, zlen=1) */
    if (g->dims == 2) {
        if (p->z[n] > 2.0) p->z[n] = p->z[n] - 1.0;
        else if (p->z[n] < 1.0) p->z[n] = 1.0 + p->z[n];
    }
}

/* ReduceCurrentMatrix scatter, movdep_routines.F90:262-308 (thread slices
   already summed into vj). */
static void reduce_current_matrix(const orc_grid *g, const double *vj, orc_fields *f)
{
    double *Jx = f->Jx, *Jy = f->Jy, *Jz = f->Jz;
    if (g->dims == 3) {
        for (int k = 1; k <= g->mz - 1; k++)
            for (int j = 1; j <= g->my - 1; j++)
                for (int i = 1; i <= g->mx - 1; i++) {
                    const double *v = vj + ID(g, i, j, k) * 12;
                    Jx[ID(g, i, j, k)] += v[0];
                    Jx[ID(g, i, j + 1, k)] += v[1];
                    Jx[ID(g, i, j, k + 1)] += v[2];
                    Jx[ID(g, i, j + 1, k + 1)] += v[3];
                    Jy[ID(g, i, j, k)] += v[4];
                    Jy[ID(g, i + 1, j, k)] += v[5];
                    Jy[ID(g, i, j, k + 1)] += v[6];
                    Jy[ID(g, i + 1, j, k + 1)] += v[7];
                    Jz[ID(g, i, j, k)] += v[8];
                    Jz[ID(g, i + 1, j, k)] += v[9];
                    Jz[ID(g, i, j + 1, k)] += v[10];
                    Jz[ID(g, i + 1, j + 1, k)] += v[11];
                }
    } else {
        for (int j = 1; j <= g->my - 1; j++)
            for (int i = 1; i <= g->mx - 1; i++) {
                const double *v = vj + ID(g, i, j, 1) * 8;
                Jx[ID(g, i, j, 1)] += v[0];
                Jx[ID(g, i, j + 1, 1)] += v[1];
                Jy[ID(g, i, j, 1)] += v[2];
                Jy[ID(g, i + 1, j, 1)] += v[3];
                Jz[ID(g, i, j, 1)] += v[4];
                Jz[ID(g, i + 1, j, 1)] += v[5];
                Jz[ID(g, i, j + 1, 1)] += v[6];
                Jz[ID(g, i + 1, j + 1, 1)] += v[7];
            }
    }
}

/* With OpenMP: 0 = the reference's OPEN_MP structure (thread-private VecJ
   slices summed in thread order, movdep.F90:57-66 and
   movdep_routines.F90:251-255), whose rounding depends on the thread count;
   1 = each cell's VecJ entries summed in particle order, as the serial build
   does, so that the result equals the serial build bit for bit at any thread
   count (the particles are moved in parallel into per-particle records,
   which a stable counting sort by cell groups for the per-cell sums). */
static int g_exact_order = 0;
void orc_set_exact_order(int on) { g_exact_order = on != 0; }

void orc_move_deposit(const orc_grid *g, orc_particles *p, orc_fields *f)
{
    const int nj = g->dims == 3 ? 12 : 8;
    const size_t ncell = (size_t)g->mx * g->my * g->mz;
    double *vj = (double *)calloc(ncell * nj, sizeof(double));
    orc_reset_current(g, f); /* J is zero whenever the deposit starts (current.F90:13-17) */
#ifdef _OPENMP
    int nthreads = omp_get_max_threads();
#else
    int nthreads = 1;
#endif
    if (nthreads <= 1 || p->used < 4096) {
        for (int64_t n = 0; n < p->used; n++) move_one(g, p, f, n, vj, NULL);
    } else if (g_exact_order) {
#ifdef _OPENMP
        const int64_t nrec = 2 * p->used;
        vecj_contrib *rec = (vecj_contrib *)malloc((size_t)nrec * sizeof(vecj_contrib));
        int64_t *start = (int64_t *)calloc(ncell + 1, sizeof(int64_t));
        int64_t *order = (int64_t *)malloc((size_t)nrec * sizeof(int64_t));
#pragma omp parallel for schedule(static)
        for (int64_t n = 0; n < p->used; n++) move_one(g, p, f, n, NULL, rec + 2 * n);
        for (int64_t r = 0; r < nrec; r++) start[rec[r].cell + 1]++;
        for (size_t c = 0; c < ncell; c++) start[c + 1] += start[c];
        {
            int64_t *fill = (int64_t *)malloc(ncell * sizeof(int64_t));
            memcpy(fill, start, ncell * sizeof(int64_t));
            for (int64_t r = 0; r < nrec; r++) order[fill[rec[r].cell]++] = r;
            free(fill);
        }
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < (int64_t)ncell; c++)
            for (int64_t t = start[c]; t < start[c + 1]; t++)
                for (int nn = 0; nn < nj; nn++) vj[c * nj + nn] = vj[c * nj + nn] + rec[order[t]].val[nn];
        free(order);
        free(start);
        free(rec);
#endif
    } else {
#ifdef _OPENMP
        /* OPEN_MP path of movdep.F90:57-66: blocks of 32 particles, one private
           VecJ per thread, summed in thread order (movdep_routines.F90:251-255). */
        double *priv = (double *)calloc((size_t)nthreads * ncell * nj, sizeof(double));
        const int64_t nblocks = (p->used + 31) / 32;
#pragma omp parallel
        {
            double *mine = priv + (size_t)omp_get_thread_num() * ncell * nj;
#pragma omp for schedule(static)
            for (int64_t b = 0; b < nblocks; b++) {
                const int64_t e = (b + 1) * 32 < p->used ? (b + 1) * 32 : p->used;
                for (int64_t n = b * 32; n < e; n++) move_one(g, p, f, n, mine, NULL);
            }
#pragma omp for schedule(static)
            for (int64_t cidx = 0; cidx < (int64_t)ncell; cidx++)
                for (int t = 0; t < nthreads; t++)
                    for (int nn = 0; nn < nj; nn++) vj[cidx * nj + nn] += priv[((size_t)t * ncell + cidx) * nj + nn];
        }
        free(priv);
#endif
    }
    reduce_current_matrix(g, vj, f);
    free(vj);
}

/* ------------------------------------------------------------------------- */
/* Particle wrap: loadprtlout.F90:13-106, comm_prtl.F90:11-66                */
/* ------------------------------------------------------------------------- */

/* RemovePrtl, loadprtlout.F90:164-181 */
static void remove_prtl(const orc_grid *g, orc_particles *p, int64_t n)
{
    p->q[n] = 0; p->flv[n] = 0; p->u[n] = 0; p->v[n] = 0; p->w[n] = 0;
    p->x[n] = 3.8; p->y[n] = 3.8; p->z[n] = g->dims == 3 ? 3.8 : 1.5;
}

int orc_exchange_particles(const orc_grid *g, orc_particles *p)
{
    const double xmin = 3.0, xmax = (double)(g->mx - 2), ymin = 3.0, ymax = (double)(g->my - 2);
    const double zmin = g->dims == 3 ? 3.0 : 1.0, zmax = g->dims == 3 ? (double)(g->mz - 2) : 2.0;
    const double len[3] = {xmax - xmin, ymax - ymin, zmax - zmin};
    const int nfaces = g->dims == 3 ? 6 : 4;
    int64_t *lists[6];
    int64_t cnt[6] = {0, 0, 0, 0, 0, 0};
    double (*saved)[8] = NULL; /* q,x,y,z,u,v,w,flv of each leaver */
    int64_t nsaved = 0;
    for (int fc = 0; fc < 6; fc++) lists[fc] = NULL;
    /* count pass is folded into the scan: grow arrays as needed */
    int64_t cap_saved = 1024;
    saved = (double (*)[8])malloc((size_t)cap_saved * sizeof(*saved));
    for (int fc = 0; fc < nfaces; fc++) lists[fc] = (int64_t *)malloc((size_t)cap_saved * sizeof(int64_t));
    int64_t cap_list[6] = {cap_saved, cap_saved, cap_saved, cap_saved, cap_saved, cap_saved};

    for (int64_t i = 0; i < p->used; i++) {
        if (p->flv[i] == 0) continue;
        double x = p->x[i], y = p->y[i], z = p->z[i];
#define SEND(fc)                                                                              \
    do {                                                                                      \
        if (nsaved == cap_saved) {                                                            \
            cap_saved *= 2;                                                                   \
            saved = (double (*)[8])realloc(saved, (size_t)cap_saved * sizeof(*saved));        \
        }                                                                                     \
        saved[nsaved][0] = p->q[i]; saved[nsaved][1] = p->x[i]; saved[nsaved][2] = p->y[i];   \
        saved[nsaved][3] = p->z[i]; saved[nsaved][4] = p->u[i]; saved[nsaved][5] = p->v[i];   \
        saved[nsaved][6] = p->w[i]; saved[nsaved][7] = (double)p->flv[i];                    \
        if (cnt[fc] == cap_list[fc]) {                                                        \
            cap_list[fc] *= 2;                                                                \
            lists[fc] = (int64_t *)realloc(lists[fc], (size_t)cap_list[fc] * sizeof(int64_t)); \
        }                                                                                     \
        lists[fc][cnt[fc]++] = nsaved++;                                                      \
        remove_prtl(g, p, i);                                                                 \
        x = p->x[i]; y = p->y[i]; z = p->z[i];                                                \
    } while (0)
        if (x < xmin) {                                                       /* :31-41 */
            if ((y <= (ymax + xmin) - x) && (y >= (ymin - xmin) + x)) {
                if (g->dims == 2 || ((z <= (zmax + xmin) - x) && (z >= (zmin - xmin) + x))) SEND(0);
            }
        } else if (x > xmax) {                                                /* :42-53 */
            if ((y <= (ymax - xmax) + x) && (y >= (ymin + xmax) - x)) {
                if (g->dims == 2 || ((z <= (zmax - xmax) + x) && (z >= (zmin + xmax) - x))) SEND(1);
            }
        }
        if (y < ymin) {                                                       /* :54-64 */
            if ((y < (ymin - xmin) + x) && (y < (ymin + xmax) - x)) {
                if (g->dims == 2 || ((z >= (zmin - ymin) + y) && (z <= (zmax + ymin) - y))) SEND(2);
            }
        } else if (y > ymax) {                                                /* :65-76 */
            if ((y > (ymax + xmin) - x) && (y > (ymax - xmax) + x)) {
                if (g->dims == 2 || ((z >= (zmin + ymax) - y) && (z <= (zmax - ymax) + y))) SEND(3);
            }
        }
        if (g->dims == 3) {
            if (z < zmin) {                                                   /* :79-86 */
                if ((z < (zmin - xmin) + x) && (z < (zmin + xmax) - x))
                    if ((z < (zmin - ymin) + y) && (z < (zmin + ymax) - y)) SEND(4);
            } else if (z > zmax) {                                            /* :87-95 */
                if ((z > (zmax + xmin) - x) && (z > (zmax - xmax) + x))
                    if ((z > (zmax + ymin) - y) && (z > (zmax - ymax) + y)) SEND(5);
            }
        }
#undef SEND
    }
    int64_t total = 0;
    for (int fc = 0; fc < nfaces; fc++) total += cnt[fc];
    int rc = 0;
    if (p->used + total > p->capacity) {
        rc = -1;
    } else {
        /* AppendParticles order: recv(1)..recv(n) hold send(2),send(1),send(4),... */
        static const int order[6] = {1, 0, 3, 2, 5, 4};
        for (int o = 0; o < nfaces; o++) {
            const int fc = order[o];
            const int axis = fc / 2;
            for (int64_t m = 0; m < cnt[fc]; m++) {
                const double *s = saved[lists[fc][m]];
                double pos[3] = {s[1], s[2], s[3]};
                /* CopyTransferPrtl subtracts the send list shift (len on high
                   faces), InsertPrtls adds the recv list shift (len on the
                   receiving high list): low faces end up +len, high faces -len. */
                if (fc % 2 == 0) pos[axis] = (pos[axis] - 0.0) + len[axis];
                else pos[axis] = (pos[axis] - len[axis]) + 0.0;
                const int64_t d = p->used++;
                p->q[d] = s[0]; p->x[d] = pos[0]; p->y[d] = pos[1]; p->z[d] = pos[2];
                p->u[d] = s[4]; p->v[d] = s[5]; p->w[d] = s[6]; p->flv[d] = (int32_t)s[7];
            }
        }
    }
    for (int fc = 0; fc < nfaces; fc++) free(lists[fc]);
    free(saved);
    return rc;
}

/* ------------------------------------------------------------------------- */
/* ReorderPrtlArr, mem_prtl.F90:166-301 (serial: stable)                     */
/* ------------------------------------------------------------------------- */
void orc_reorder(const orc_grid *g, orc_particles *p, int64_t *perm)
{
    const size_t ncell = (size_t)g->mx * g->my * g->mz;
    int64_t *pcount = (int64_t *)calloc(ncell, sizeof(int64_t));
    int64_t np = 0;
    for (int64_t n = 0; n < p->used; n++)                                         /* :178-190 */
        if (p->flv[n] != 0) {
            const int i = (int)floor(p->x[n]), j = (int)floor(p->y[n]);
            const int k = g->dims == 3 ? (int)floor(p->z[n]) : 1;
            pcount[ID(g, i, j, k)]++;
            np++;
        }
    int64_t offset = 0;                                                           /* :199-214 */
    for (size_t cidx = 0; cidx < ncell; cidx++) {
        const int64_t t = pcount[cidx];
        pcount[cidx] = offset;
        offset += t;
    }
    double *tmp = (double *)malloc((size_t)(np > 0 ? np : 1) * sizeof(double));
    int32_t *tmpi = (int32_t *)malloc((size_t)(np > 0 ? np : 1) * sizeof(int32_t));
    int64_t *dest = (int64_t *)malloc((size_t)(p->used > 0 ? p->used : 1) * sizeof(int64_t));
    for (int64_t n = 0; n < p->used; n++) {                                       /* :238-272 */
        dest[n] = -1;
        if (p->flv[n] != 0) {
            const int i = (int)floor(p->x[n]), j = (int)floor(p->y[n]);
            const int k = g->dims == 3 ? (int)floor(p->z[n]) : 1;
            dest[n] = pcount[ID(g, i, j, k)]++;
        }
    }
    double *arrs[7] = {p->q, p->x, p->y, p->z, p->u, p->v, p->w};
    for (int a = 0; a < 7; a++) {
        for (int64_t n = 0; n < p->used; n++)
            if (dest[n] >= 0) tmp[dest[n]] = arrs[a][n];
        memcpy(arrs[a], tmp, (size_t)np * sizeof(double));
    }
    for (int64_t n = 0; n < p->used; n++)
        if (dest[n] >= 0) {
            tmpi[dest[n]] = p->flv[n];
            if (perm) perm[dest[n]] = n;
        }
    memcpy(p->flv, tmpi, (size_t)np * sizeof(int32_t));
    for (int64_t n = np; n < p->used; n++) { p->q[n] = 0; p->flv[n] = 0; }      /* :274-277 */
    p->used = np;
    free(pcount); free(tmp); free(tmpi); free(dest);
}

/* ------------------------------------------------------------------------- */
/* Walls along x on one rank (xborders(procxind) = 0): src/bc/bc_reflect.F90  */
/* ------------------------------------------------------------------------- */
/* Add (sign +1) or subtract (-1) the x layer `from` onto the layer `to` of F
   over every (j, k), then zero `from` (whole planes, ghosts included). */
static void fold_x_layer(const orc_grid *g, double *F, int to, int from, double sign)
{
    for (int k = 1; k <= g->mz; k++)
        for (int j = 1; j <= g->my; j++) {
            if (sign > 0) F[ID(g, to, j, k)] = F[ID(g, to, j, k)] + F[ID(g, from, j, k)];
            else F[ID(g, to, j, k)] = F[ID(g, to, j, k)] - F[ID(g, from, j, k)];
        }
    for (int k = 1; k <= g->mz; k++)
        for (int j = 1; j <= g->my; j++) F[ID(g, from, j, k)] = 0.0;
}

/* RefBC_Prtl_Left (bc_reflect.F90:146-155), RefPrtlLeft (:164-176),
   ReflCurrentLeft (:195-213). */
void orc_refl_prtl_left(const orc_grid *g, orc_particles *p, orc_fields *f, double pos)
{
    const double xmin = pos - 0.0 + 3;
    if (xmin > 1)
        for (int64_t n = 0; n < p->used; n++)
            if (p->flv[n] != 0 && p->x[n] < xmin) {
                p->u[n] = -p->u[n];
                p->x[n] = 2.0 * xmin - p->x[n];
            }
    int ind = (int)ceil(pos - 0.0 + 3);
    if (ind >= 2 && ind <= g->mx) {
        fold_x_layer(g, f->Jy, ind, ind - 1, 1.0);
        fold_x_layer(g, f->Jz, ind, ind - 1, 1.0);
    }
    ind = (int)ceil(pos - 0.5 - 0.0 + 3);
    if (ind >= 2 && ind <= g->mx) fold_x_layer(g, f->Jx, ind, ind - 1, -1.0);
}

/* RefBC_Prtl_Right (bc_reflect.F90:135-144), RefPrtlRight (:178-190),
   ReflCurrentRight (:215-237); the wall of bc_face(2) is `pos` itself. */
void orc_refl_prtl_right(const orc_grid *g, orc_particles *p, orc_fields *f, double pos)
{
    const double xmax = pos - 0.0 + 3;
    if (xmax < g->mx - 1)
        for (int64_t n = 0; n < p->used; n++)
            if (p->flv[n] != 0 && p->x[n] > xmax) {
                p->u[n] = -p->u[n];
                p->x[n] = 2.0 * xmax - p->x[n];
            }
    int ind = (int)floor(pos - 0.0 + 3);
    if (ind >= 1 && ind <= g->mx - 1) {
        fold_x_layer(g, f->Jy, ind, ind + 1, 1.0);
        fold_x_layer(g, f->Jz, ind, ind + 1, 1.0);
    }
    ind = (int)floor(pos - 0.5 - 0.0 + 3);
    if (ind >= 1 && ind <= g->mx - 1) fold_x_layer(g, f->Jx, ind, ind + 1, -1.0);
}

/* CondBC_Fld_Left (bc_reflect.F90:58-72): Ey, Ez = 0 on x layers 1..floor(pos+3). */
void orc_cond_fld_left(const orc_grid *g, orc_fields *f, double pos)
{
    int xl = (int)floor(pos - 0.0 + 3);
    if (xl < 1) return;
    if (xl > g->mx) xl = g->mx;
    for (int k = 1; k <= g->mz; k++)
        for (int j = 1; j <= g->my; j++)
            for (int i = 1; i <= xl; i++) {
                f->Ey[ID(g, i, j, k)] = 0.0;
                f->Ez[ID(g, i, j, k)] = 0.0;
            }
}

/* CondBC_Fld_Right (bc_reflect.F90:43-56): Ey, Ez = 0 on x layers ceiling(pos+3)..mx. */
void orc_cond_fld_right(const orc_grid *g, orc_fields *f, double pos)
{
    int xr = (int)ceil(pos - 0.0 + 3);
    if (xr > g->mx) return;
    if (xr < 1) xr = 1;
    for (int k = 1; k <= g->mz; k++)
        for (int j = 1; j <= g->my; j++)
            for (int i = xr; i <= g->mx; i++) {
                f->Ey[ID(g, i, j, k)] = 0.0;
                f->Ez[ID(g, i, j, k)] = 0.0;
            }
}

/* y layer version of fold_x_layer: F(:,to,:) +-= F(:,from,:); F(:,from,:) = 0. */
static void fold_y_layer(const orc_grid *g, double *F, int to, int from, double sign)
{
    for (int k = 1; k <= g->mz; k++)
        for (int i = 1; i <= g->mx; i++) {
            if (sign > 0) F[ID(g, i, to, k)] = F[ID(g, i, to, k)] + F[ID(g, i, from, k)];
            else F[ID(g, i, to, k)] = F[ID(g, i, to, k)] - F[ID(g, i, from, k)];
        }
    for (int k = 1; k <= g->mz; k++)
        for (int i = 1; i <= g->mx; i++) F[ID(g, i, from, k)] = 0.0;
}

/* RefBC_Prtl_Bottom (bc_reflect.F90:106-128): y mirrored below ymin = pos + 3,
   the current of layer W - 1 (W = int(ymin)) folded onto W. */
void orc_refl_prtl_bottom(const orc_grid *g, orc_particles *p, orc_fields *f, double pos)
{
    const double ymin = pos - 0.0 + 3;
    const int W = (int)ymin;
    if (ymin > 1)
        for (int64_t n = 0; n < p->used; n++)
            if (p->flv[n] != 0 && p->y[n] < ymin) {
                p->v[n] = -p->v[n];
                p->y[n] = 2.0 * ymin - p->y[n];
            }
    if (W >= 3 && W <= g->my - 2) {
        fold_y_layer(g, f->Jx, W, W - 1, 1.0);
        fold_y_layer(g, f->Jy, W, W - 1, -1.0);
        fold_y_layer(g, f->Jz, W, W - 1, 1.0);
    }
}

/* RefBC_Prtl_Top (bc_reflect.F90:79-104): y mirrored above ymax = pos + 3,
   Jx, Jz of layer W + 1 folded onto W and Jy of W onto W - 1 (W = int(ymax)). */
void orc_refl_prtl_top(const orc_grid *g, orc_particles *p, orc_fields *f, double pos)
{
    const double ymax = pos - 0.0 + 3;
    const int W = (int)ymax;
    if (ymax < g->my - 1)
        for (int64_t n = 0; n < p->used; n++)
            if (p->flv[n] != 0 && p->y[n] > ymax) {
                p->v[n] = -p->v[n];
                p->y[n] = 2.0 * ymax - p->y[n];
            }
    if (W >= 2 && W <= g->my - 2) {
        for (int k = 1; k <= g->mz; k++)
            for (int i = 1; i <= g->mx; i++) {
                f->Jx[ID(g, i, W, k)] = f->Jx[ID(g, i, W, k)] + f->Jx[ID(g, i, W + 1, k)];
                f->Jy[ID(g, i, W - 1, k)] = f->Jy[ID(g, i, W - 1, k)] - f->Jy[ID(g, i, W, k)];
                f->Jz[ID(g, i, W, k)] = f->Jz[ID(g, i, W, k)] + f->Jz[ID(g, i, W + 1, k)];
            }
        for (int k = 1; k <= g->mz; k++)
            for (int i = 1; i <= g->mx; i++) {
                f->Jx[ID(g, i, W + 1, k)] = 0.0;
                f->Jy[ID(g, i, W, k)] = 0.0;
                f->Jz[ID(g, i, W + 1, k)] = 0.0;
            }
    }
}

/* CondBC_Fld_Bottom (bc_reflect.F90:27-41): Ex, Ez = 0 on y layers 1..floor(pos+3). */
void orc_cond_fld_bottom(const orc_grid *g, orc_fields *f, double pos)
{
    int yl = (int)floor(pos - 0.0 + 3);
    if (yl < 1) return;
    if (yl > g->my) yl = g->my;
    for (int k = 1; k <= g->mz; k++)
        for (int j = 1; j <= yl; j++)
            for (int i = 1; i <= g->mx; i++) {
                f->Ex[ID(g, i, j, k)] = 0.0;
                f->Ez[ID(g, i, j, k)] = 0.0;
            }
}

/* CondBC_Fld_Top (bc_reflect.F90:11-25): Ex, Ez = 0 on y layers ceiling(pos+3)..my. */
void orc_cond_fld_top(const orc_grid *g, orc_fields *f, double pos)
{
    int yl = (int)ceil(pos - 0.0 + 3);
    if (yl > g->my) return;
    if (yl < 1) yl = 1;
    for (int k = 1; k <= g->mz; k++)
        for (int j = yl; j <= g->my; j++)
            for (int i = 1; i <= g->mx; i++) {
                f->Ex[ID(g, i, j, k)] = 0.0;
                f->Ez[ID(g, i, j, k)] = 0.0;
            }
}

/* RemovePrtl_Left / Right (bc_open.F90:8-62): the coordinate of the face's
   axis compared with the wall, the removed particle holed as RemovePrtl
   does (x = y = 3.8, z = 3.8 in 3D, 1.5 in 2D; the y and z faces pass
   their axis as the routine's x, which changes nothing in those values). */
void orc_remove_prtl(const orc_grid *g, orc_particles *p, int face, double pos)
{
    const double wall = pos - 0.0 + 3;   /* bc_pos_local with the borders at 0 */
    const int axis = (face - 1) / 2, low = (face % 2) == 1;
    for (int64_t n = 0; n < p->used; n++) {
        if (p->flv[n] == 0) continue;
        const double c = axis == 0 ? p->x[n] : axis == 1 ? p->y[n] : p->z[n];
        if (low ? c < wall : c > wall) {
            p->q[n] = 0;
            p->flv[n] = 0;
            p->u[n] = 0;
            p->v[n] = 0;
            p->w[n] = 0;
            p->x[n] = 3.8;
            p->y[n] = 3.8;
            p->z[n] = g->dims == 3 ? 3.8 : 1.5;
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Field faces of EnforceBC_Final (bc.F90:292-340) on one rank: x0 = y0 =    */
/* z0 = -3 (z0 = 0 in 2D)                                                    */
/* ------------------------------------------------------------------------- */
static double cube(double t) { return t * t * t; }   /* t**3 */

/* AttenFactorVacuum (bc_attenuate.F90:222-290). */
static double atten_factor_vacuum(const double *p, const double *sc, int three_d, double x, double y, double z)
{
    double af = 0.0;
    if (x < p[0]) {
        if ((y <= (p[3] + p[0] - x)) && (y >= (p[2] - p[0] + x)))
            if (z <= (p[5] + p[0] - x) && (z >= (p[4] - p[0] + x))) af = cube(fabs(x - p[0]) / sc[0]);
    } else if (x > p[1]) {
        if ((y <= (p[3] - p[1] + x)) && (y >= (p[2] + p[1] - x)))
            if ((z <= (p[5] - p[1] + x)) && (z >= (p[4] + p[1] - x))) af = cube(fabs(x - p[1]) / sc[1]);
    }
    if (y < p[2]) {
        if ((y < (p[2] - p[0] + x)) && (y < (p[2] + p[1] - x)))
            if ((z >= (p[4] - p[2] + y)) && (z <= (p[5] + p[2] - y))) af = cube(fabs(y - p[2]) / sc[2]);
    } else if (y > p[3]) {
        if ((y > (p[3] + p[0] - x)) && (y > (p[3] - p[1] + x)))
            if ((z >= (p[4] + p[3] - y)) && (z <= (p[5] - p[3] + y))) af = cube(fabs(y - p[3]) / sc[3]);
    }
    if (three_d) {
        if (z < p[4]) {
            if ((z < (p[4] - p[0] + x)) && (z < (p[4] + p[1] - x)))
                if ((z < (p[4] - p[2] + y)) && (z < (p[4] + p[3] - y))) af = cube(fabs(z - p[4]) / sc[4]);
        } else if (z > p[5]) {
            if (z > (p[5] + p[0] - x) && (z > (p[5] - p[1] + x)))
                if ((z > (p[5] + p[2] - y)) && (z > (p[5] - p[3] + y))) af = cube(fabs(z - p[5]) / sc[5]);
        }
    }
    af = af < 1.0 ? af : 1.0;   /* min(1.0, af) */
    af = af > 0.0 ? af : 0.0;   /* max(0.0, af) */
    return 1.0 - af;
}

/* Attenuate_EM_Vacuum (bc_attenuate.F90:151-220): bit n-1 of `faces` marks
   bc_face(n) as 'attn' at pos[n-1] with attn_scale scale[n-1]; the other
   faces keep attn_vac_pos = -+huge(1) and attn_vac_pos_ind = -+huge(1). */
void orc_attn_vacuum(const orc_grid *g, orc_fields *f, int faces, const double *pos, const double *scale)
{
    double p[6], sc[6];
    long long ind[6];
    for (int n = 0; n < 6; n++) {
        const int on = (faces >> n) & 1, upper = (n & 1) != 0;
        p[n] = on ? pos[n] : (upper ? 2147483647.0 : -2147483647.0);
        sc[n] = on ? scale[n] : 1.0;
        ind[n] = on ? (upper ? (long long)ceil(p[n]) + 1 : (long long)floor(p[n]) - 1) : (upper ? 2147483647 : -2147483647);
    }
    const int three_d = g->dims == 3;
    int inside = 1 - 3 > ind[0] && g->mx - 3 < ind[1] && 1 - 3 > ind[2] && g->my - 3 < ind[3] &&
                 (!three_d || (1 - 3 > ind[4] && g->mz - 3 < ind[5]));
    if (inside) return;
    const double x0 = -3, y0 = -3, z0 = three_d ? -3 : 0;
    for (int k = 1; k <= g->mz; k++)
        for (int j = 1; j <= g->my; j++)
            for (int i = 1; i <= g->mx; i++) {
                inside = i - 3 > ind[0] && i - 3 < ind[1] && j - 3 > ind[2] && j - 3 < ind[3] &&
                         (!three_d || (k - 3 > ind[4] && k - 3 < ind[5]));
                if (inside) continue;
                const int64_t c = ID(g, i, j, k);
                f->Ex[c] = f->Ex[c] * atten_factor_vacuum(p, sc, three_d, i + 0.5 + x0, j + y0, k + z0);
                f->Ey[c] = f->Ey[c] * atten_factor_vacuum(p, sc, three_d, i + x0, j + 0.5 + y0, k + z0);
                f->Ez[c] = f->Ez[c] * atten_factor_vacuum(p, sc, three_d, i + x0, j + y0, k + 0.5 + z0);
                f->Bx[c] = f->Bx[c] * atten_factor_vacuum(p, sc, three_d, i + x0, j + 0.5 + y0, k + 0.5 + z0);
                f->By[c] = f->By[c] * atten_factor_vacuum(p, sc, three_d, i + 0.5 + x0, j + y0, k + 0.5 + z0);
                f->Bz[c] = f->Bz[c] * atten_factor_vacuum(p, sc, three_d, i + 0.5 + x0, j + 0.5 + y0, k + z0);
            }
}

/* atnn_domain (bc_attenuate.F90:117-131) and AttenFactor (:102-115). */
static int atnn_domain(double xg, double yg, double pos, int side, double dl)
{
    switch (side) {
        case 1: return xg >= pos && xg <= pos + dl;
        case 2: return xg <= pos && xg >= pos - dl;
        case 3: return yg >= pos && yg <= pos + dl;
        case 4: return yg <= pos && yg >= pos - dl;
    }
    return 0;
}
static double atten_factor(double x, double y, double pos, int side, double dl)
{
    double af = 0.0;
    if (side == 1 || side == 2) af = cube(fabs(x - pos) / dl);
    else af = cube(fabs(y - pos) / dl);
    af = af < 1.0 ? af : 1.0;
    af = af > 0.0 ? af : 0.0;
    return 1.0 - af;
}

/* Attenuate_EM_Flow (bc_attenuate.F90:16-98) on face `side` 1..4 for a flow
   with the uniform MagFld b[3] and Drift v[3]. */
void orc_attn_flow(const orc_grid *g, orc_fields *f, int side, double pos, double dl, double scale, const double *b,
                   const double *v)
{
    const double x0 = -3, y0 = -3;
    if (dl == 0) return;
    if ((side == 1 || side == 3) && (side == 1 ? (pos + dl) - x0 < 1 : (pos + dl) - y0 < 1)) return;
    if ((side == 2 || side == 4) && (side == 2 ? (pos - dl) - x0 > g->mx : (pos - dl) - y0 > g->my)) return;
    for (int k = 1; k <= g->mz; k++)
        for (int j = 1; j <= g->my; j++)
            for (int i = 1; i <= g->mx; i++) {
                const int64_t c = ID(g, i, j, k);
                double xg, yg, f0;
                xg = i + 0.5 + x0; yg = j + y0;
                if (atnn_domain(xg, yg, pos, side, dl)) {
                    f0 = v[2] * b[1] - v[1] * b[2];
                    f->Ex[c] = (f->Ex[c] - f0) * atten_factor(xg, yg, pos, side, scale) + f0;
                }
                xg = i + x0; yg = j + 0.5 + y0;
                if (atnn_domain(xg, yg, pos, side, dl)) {
                    f0 = v[0] * b[2] - v[2] * b[0];
                    f->Ey[c] = (f->Ey[c] - f0) * atten_factor(xg, yg, pos, side, scale) + f0;
                }
                xg = i + x0; yg = j + y0;
                if (atnn_domain(xg, yg, pos, side, dl)) {
                    f0 = v[1] * b[0] - v[0] * b[1];
                    f->Ez[c] = (f->Ez[c] - f0) * atten_factor(xg, yg, pos, side, scale) + f0;
                }
                xg = i + x0; yg = j + 0.5 + y0;
                if (atnn_domain(xg, yg, pos, side, dl))
                    f->Bx[c] = (f->Bx[c] - b[0]) * atten_factor(xg, yg, pos, side, scale) + b[0];
                xg = i + 0.5 + x0; yg = j + y0;
                if (atnn_domain(xg, yg, pos, side, dl))
                    f->By[c] = (f->By[c] - b[1]) * atten_factor(xg, yg, pos, side, scale) + b[1];
                xg = i + 0.5 + x0; yg = j + 0.5 + y0;
                if (atnn_domain(xg, yg, pos, side, dl))
                    f->Bz[c] = (f->Bz[c] - b[2]) * atten_factor(xg, yg, pos, side, scale) + b[2];
            }
}

/* OpenBC_Fld_Right (bc.F90:411-440). */
void orc_open_fld_right(const orc_grid *g, orc_fields *f, double pos)
{
    const int xl = (int)ceil(pos - 0.0 + 3);
    if (!(xl >= 1 && xl <= g->mx - 1)) return;
    for (int i = xl + 1; i <= g->mx; i++)
        for (int k = 1; k <= g->mz; k++)
            for (int j = 1; j <= g->my; j++) {
                f->Ey[ID(g, i, j, k)] = 0.5 * f->Ey[ID(g, i, j, k)];
                f->Ez[ID(g, i, j, k)] = 0.5 * f->Ez[ID(g, i, j, k)];
                f->Bx[ID(g, i, j, k)] = f->Bx[ID(g, xl, j, k)];
            }
    for (int i = xl; i <= g->mx; i++)
        for (int k = 1; k <= g->mz; k++)
            for (int j = 1; j <= g->my; j++) {
                f->Ex[ID(g, i, j, k)] = 0.5 * f->Ex[ID(g, i, j, k)];
                f->By[ID(g, i, j, k)] = 0.5 * f->By[ID(g, i, j, k)];
                f->Bz[ID(g, i, j, k)] = 0.5 * f->Bz[ID(g, i, j, k)];
            }
}

/* OpenBC_Fld_Left (bc.F90:442-469). */
void orc_open_fld_left(const orc_grid *g, orc_fields *f, double pos)
{
    const int xl = (int)ceil(pos - 0.0 + 3);
    if (!(xl >= 2 && xl <= g->mx)) return;
    for (int i = 1; i <= xl - 1; i++)
        for (int k = 1; k <= g->mz; k++)
            for (int j = 1; j <= g->my; j++) {
                f->Ey[ID(g, i, j, k)] = 0.5 * f->Ey[ID(g, i, j, k)];
                f->Ez[ID(g, i, j, k)] = 0.5 * f->Ez[ID(g, i, j, k)];
                f->Bx[ID(g, i, j, k)] = f->Bx[ID(g, xl, j, k)];
                f->Ex[ID(g, i, j, k)] = 0.5 * f->Ex[ID(g, i, j, k)];
                f->By[ID(g, i, j, k)] = 0.5 * f->By[ID(g, i, j, k)];
                f->Bz[ID(g, i, j, k)] = 0.5 * f->Bz[ID(g, i, j, k)];
            }
}

/* OpenBC_Prtl_Right (bc.F90:478-538) / OpenBC_Prtl_Left (:540-600) with the
   column means of OpenBC_MeanPrtlSpeed (:603-621), DeletePrtl
   (mem_prtl.F90:7-22) and InsertNewPrtl (:120-133); side 1 right, 0 left.
   Returns -1 (nothing appended past the capacity) when the copies do not
   fit. */
int orc_open_prtl(const orc_grid *g, orc_particles *p, int side, double pos, double dx)
{
    const double wall = pos - 0.0 + 3;
    if (side == 1 ? !(wall < g->mx - 1) : !(wall > 1)) return 0;
    for (int64_t n = 0; n < p->used; n++)
        if (p->q[n] != 0 && (side == 1 ? p->x[n] > wall : p->x[n] < wall)) {
            p->q[n] = 0.0;
            p->x[n] = 3.8;
            p->y[n] = 3.8;
            p->z[n] = g->dims == 3 ? 3.8 : 1.5;
            p->u[n] = 0.0;
            p->v[n] = 0.0;
            p->w[n] = 0.0;
            p->flv[n] = 0;
        }
    const int ncol = g->my * g->mz;
    double *den = malloc(sizeof(double) * (size_t)ncol), *vel = malloc(sizeof(double) * (size_t)ncol);
    for (int c = 0; c < ncol; c++) { den[c] = 1.0; vel[c] = 0.0; }
#define IN_LAYER(n) (p->q[n] != 0 && (side == 1 ? (p->x[n] > wall - dx && p->x[n] < wall) \
                                              : (p->x[n] < wall + dx && p->x[n] > wall)))
    for (int64_t n = 0; n < p->used; n++)
        if (IN_LAYER(n) && p->flv[n] <= 2) {
            const int j = (int)p->y[n], k = g->dims == 3 ? (int)p->z[n] : 1;
            const double invg = 1.0 / sqrt(1.0 + p->u[n] * p->u[n] + p->v[n] * p->v[n] + p->w[n] * p->w[n]);
            const double vx = p->u[n] * invg;
            den[(j - 1) + g->my * (k - 1)] = den[(j - 1) + g->my * (k - 1)] + 1.0;
            vel[(j - 1) + g->my * (k - 1)] = vel[(j - 1) + g->my * (k - 1)] + vx;
        }
    for (int c = 0; c < ncol; c++) vel[c] = vel[c] / den[c];
    const int64_t used0 = p->used;
    int64_t m = 0;
    for (int64_t n = 0; n < used0; n++) if (IN_LAYER(n)) m++;
    if (used0 + m > p->capacity) { free(den); free(vel); return -1; }
    for (int64_t n = 0; n < used0; n++)
        if (IN_LAYER(n)) {
            const int j = (int)p->y[n], k = g->dims == 3 ? (int)p->z[n] : 1;
            double v0 = vel[(j - 1) + g->my * (k - 1)];
            if (side == 1 ? v0 > 0 : v0 < 0) v0 = 0.0;
            const double gamma = sqrt(1.0 + p->u[n] * p->u[n] + p->v[n] * p->v[n] + p->w[n] * p->w[n]);
            const int64_t d = p->used;
            p->x[d] = 2 * wall - p->x[n];
            p->y[d] = p->y[n];
            p->z[d] = p->z[n];
            p->u[d] = p->u[n] - gamma * v0;
            p->v[d] = p->v[n];
            p->w[d] = p->w[n];
            p->q[d] = p->q[n];
            p->flv[d] = p->flv[n];
            p->used = d + 1;
        }
#undef IN_LAYER
    free(den);
    free(vel);
    return 0;
}

/* DepositCurrentPIC (deposit.F90:11-103): the zigzag current of a move from
   (x0, y0, z0) to (x, y, z) added straight into J. */
static void deposit_current_pic(const orc_grid *g, orc_fields *f, double x0, double y0, double z0, double x,
                                double y, double z, double q)
{
    const double qthis = q * g->qi;
    const int i1 = (int)floor(x0), i2 = (int)floor(x), j1 = (int)floor(y0), j2 = (int)floor(y);
    int k1 = (int)floor(z0), k2 = (int)floor(z);
    const double xr = fmin((double)((i1 < i2 ? i1 : i2) + 1), fmax((double)(i1 > i2 ? i1 : i2), 0.5 * (x0 + x)));
    const double yr = fmin((double)((j1 < j2 ? j1 : j2) + 1), fmax((double)(j1 > j2 ? j1 : j2), 0.5 * (y0 + y)));
    const double zr = fmin((double)((k1 < k2 ? k1 : k2) + 1), fmax((double)(k1 > k2 ? k1 : k2), 0.5 * (z0 + z)));
    const double Fx1 = qthis * (xr - x0), Fy1 = qthis * (yr - y0), Fz1 = qthis * (zr - z0);
    const double Wx1 = 0.5 * (x0 + xr) - i1, Wy1 = 0.5 * (y0 + yr) - j1;
    const double Wx2 = 0.5 * (x + xr) - i2, Wy2 = 0.5 * (y + yr) - j2;
    double Wz1, Wz2;
    const int three = g->dims == 3;
    if (!three) { k1 = 1; k2 = 1; Wz1 = 0.0; Wz2 = 0.0; }
    else { Wz1 = 0.5 * (z0 + zr) - k1; Wz2 = 0.5 * (z + zr) - k2; }
    const double Fx2 = qthis * (x - xr), Fy2 = qthis * (y - yr), Fz2 = qthis * (z - zr);
    double *Jx = f->Jx, *Jy = f->Jy, *Jz = f->Jz;
    Jx[ID(g, i1, j1, k1)] += Fx1 * (1.0 - Wy1) * (1.0 - Wz1);
    Jx[ID(g, i1, j1 + 1, k1)] += Fx1 * Wy1 * (1.0 - Wz1);
    if (three) {
        Jx[ID(g, i1, j1, k1 + 1)] += Fx1 * (1.0 - Wy1) * Wz1;
        Jx[ID(g, i1, j1 + 1, k1 + 1)] += Fx1 * Wy1 * Wz1;
    }
    Jx[ID(g, i2, j2, k2)] += Fx2 * (1.0 - Wy2) * (1.0 - Wz2);
    Jx[ID(g, i2, j2 + 1, k2)] += Fx2 * Wy2 * (1.0 - Wz2);
    if (three) {
        Jx[ID(g, i2, j2, k2 + 1)] += Fx2 * (1.0 - Wy2) * Wz2;
        Jx[ID(g, i2, j2 + 1, k2 + 1)] += Fx2 * Wy2 * Wz2;
    }
    Jy[ID(g, i1, j1, k1)] += Fy1 * (1.0 - Wx1) * (1.0 - Wz1);
    Jy[ID(g, i1 + 1, j1, k1)] += Fy1 * Wx1 * (1.0 - Wz1);
    if (three) {
        Jy[ID(g, i1, j1, k1 + 1)] += Fy1 * (1.0 - Wx1) * Wz1;
        Jy[ID(g, i1 + 1, j1, k1 + 1)] += Fy1 * Wx1 * Wz1;
    }
    Jy[ID(g, i2, j2, k2)] += Fy2 * (1.0 - Wx2) * (1.0 - Wz2);
    Jy[ID(g, i2 + 1, j2, k2)] += Fy2 * Wx2 * (1.0 - Wz2);
    if (three) {
        Jy[ID(g, i2, j2, k2 + 1)] += Fy2 * (1.0 - Wx2) * Wz2;
        Jy[ID(g, i2 + 1, j2, k2 + 1)] += Fy2 * Wx2 * Wz2;
    }
    Jz[ID(g, i1, j1, k1)] += Fz1 * (1.0 - Wx1) * (1.0 - Wy1);
    Jz[ID(g, i1 + 1, j1, k1)] += Fz1 * Wx1 * (1.0 - Wy1);
    Jz[ID(g, i1, j1 + 1, k1)] += Fz1 * (1.0 - Wx1) * Wy1;
    Jz[ID(g, i1 + 1, j1 + 1, k1)] += Fz1 * Wx1 * Wy1;
    Jz[ID(g, i2, j2, k2)] += Fz2 * (1.0 - Wx2) * (1.0 - Wy2);
    Jz[ID(g, i2 + 1, j2, k2)] += Fz2 * Wx2 * (1.0 - Wy2);
    Jz[ID(g, i2, j2 + 1, k2)] += Fz2 * (1.0 - Wx2) * Wy2;
    Jz[ID(g, i2 + 1, j2 + 1, k2)] += Fz2 * Wx2 * Wy2;
}

/* RefPrtlFluidFrameRight (bc_inflow.F90:62-97) with ReflectPrtlMovingFrameX
   (:100-121) for a uniform drift vx, on one rank. */
void orc_refl_fluid_right(const orc_grid *g, orc_particles *p, orc_fields *f, double pos, double vx)
{
    const double xinj = pos - 0.0 + 3;
    if (xinj > g->mx - 1) return;
    const double x1 = xinj + vx * g->c;
    for (int64_t n = 0; n < p->used; n++) {
        if (!(p->q[n] != 0 && p->x[n] > x1)) continue;
        double db, dg;
        if (fabs(vx) < 1.0) { db = vx; dg = 1.0 / sqrt((1.0 - vx) * (1.0 + vx)); }
        else { dg = fabs(vx); db = sqrt((vx - 1.0) * (vx + 1.0)) / vx; }
        double u = p->u[n];
        const double v = p->v[n], w = p->w[n];
        double gamma = sqrt(1.0 + u * u + v * v + w * w);
        db = -db;
        u = dg * u + dg * db * gamma;
        u = -u;
        gamma = sqrt(1.0 + u * u + v * v + w * w);
        db = -db;
        u = dg * u + dg * db * gamma;
        p->u[n] = u;
        const double x0 = p->x[n], y0 = p->y[n], z0 = p->z[n];
        p->x[n] = 2.0 * x1 - x0;
        deposit_current_pic(g, f, x0, y0, z0, p->x[n], p->y[n], p->z[n], p->q[n]);
    }
}

/* ------------------------------------------------------------------------- */
/* One time step, src/MAIN.F90:42-284                                        */
/* ------------------------------------------------------------------------- */
int orc_step_filtered(const orc_grid *g, orc_particles *p, orc_fields *f, int t, int reorder_period, int curr_filter)
{
    orc_update_b_half(g, f);
    orc_send_recv_flds(g, f->Bx, f->By, f->Bz);
    orc_move_deposit(g, p, f);
    int rc = orc_exchange_particles(g, p);
    orc_update_b_half(g, f);
    orc_send_recv_flds(g, f->Bx, f->By, f->Bz);
    orc_update_e(g, f);
    orc_send_recv_flds(g, f->Ex, f->Ey, f->Ez);
    orc_update_current_all_faces(g, f->Jx, f->Jy, f->Jz);
    orc_filter_current(g, f->Jx, f->Jy, f->Jz, curr_filter);  /* MAIN.F90:156-165 */
    orc_add_current(g, f);
    orc_send_recv_flds(g, f->Ex, f->Ey, f->Ez);
    if (reorder_period > 0 && t % reorder_period == 0) orc_reorder(g, p, NULL);
    return rc;
}

int orc_step(const orc_grid *g, orc_particles *p, orc_fields *f, int t, int reorder_period)
{
    orc_update_b_half(g, f);                                   /* :49-56 */
    orc_send_recv_flds(g, f->Bx, f->By, f->Bz);                /* :58 */
    orc_move_deposit(g, p, f);                                 /* :63-71 */
    int rc = orc_exchange_particles(g, p);                     /* :86-94 + :145-150 */
    orc_update_b_half(g, f);                                   /* :101-111 */
    orc_send_recv_flds(g, f->Bx, f->By, f->Bz);
    orc_update_e(g, f);
    orc_send_recv_flds(g, f->Ex, f->Ey, f->Ez);
    orc_update_current_all_faces(g, f->Jx, f->Jy, f->Jz);      /* :124 */
    orc_add_current(g, f);                                     /* :170-172 */
    orc_send_recv_flds(g, f->Ex, f->Ey, f->Ez);                /* :184 */
    if (reorder_period > 0 && t % reorder_period == 0) orc_reorder(g, p, NULL); /* :259-265 */
    return rc;
}

/* ------------------------------------------------------------------------- */
/* Diagnostics: savedata_routines.F90:265-348                                */
/* ------------------------------------------------------------------------- */
void orc_field_energy(const orc_grid *g, const orc_fields *f, double out[2])
{
    double eb = 0, ee = 0;
    const int k1 = g->dims == 3 ? 3 : 1, k2 = g->dims == 3 ? g->mz - 3 : 1;
    for (int k = k1; k <= k2; k++)
        for (int j = 3; j <= g->my - 3; j++)
            for (int i = 3; i <= g->mx - 3; i++) {
                const int64_t c0 = ID(g, i, j, k);
                eb = eb + ((f->Bx[c0] * f->Bx[c0] + f->By[c0] * f->By[c0]) + f->Bz[c0] * f->Bz[c0]);
                ee = ee + ((f->Ex[c0] * f->Ex[c0] + f->Ey[c0] * f->Ey[c0]) + f->Ez[c0] * f->Ez[c0]);
            }
    out[0] = eb;
    out[1] = ee;
}

void orc_particle_energy(const orc_grid *g, const orc_particles *p, double masse, double massi, double *energy)
{
    const double c = g->c;
    const double mec2 = (masse * c) * c;
    (void)massi;
    for (int64_t n = 0; n < p->used; n++) {
        if (p->flv[n] == 0) continue;
        const double gm = sqrt(((1.0 + p->u[n] * p->u[n]) + p->v[n] * p->v[n]) + p->w[n] * p->w[n]);
        const int fl = p->flv[n];
        /* weight wtp = |q| for the loaders here (charge = weight * FlvrCharge) */
        const double wt = fabs(p->q[n]);
        if (p->q[n] > 0) energy[fl - 1] += (((gm - 1.0) * wt) * (p->q[n] * g->qi / g->flvrqm[fl])) * c * c;
        if (p->q[n] < 0) energy[fl - 1] += ((gm - 1.0) * wt) * mec2;
    }
}

static int wrap_node(int idx, int n)
{
    int r = (idx - 3) % n;
    if (r < 0) r += n;
    return 3 + r;
}

double orc_gauss_residual(const orc_grid *g, const orc_fields *f, const orc_particles *p, double *rho_max)
{
    const size_t ncell = (size_t)g->mx * g->my * g->mz;
    double *rho = (double *)calloc(ncell, sizeof(double));
    double *rho_pos = (double *)calloc(ncell, sizeof(double));
    for (int64_t n = 0; n < p->used; n++) {
        if (p->flv[n] == 0) continue;
        const double q = p->q[n] * g->qi;
        const int i = (int)floor(p->x[n]), j = (int)floor(p->y[n]);
        const double dx = p->x[n] - i, dy = p->y[n] - j;
        const int k = g->dims == 3 ? (int)floor(p->z[n]) : 1;
        const double dz = g->dims == 3 ? p->z[n] - k : 0.0;
        const int nc = g->dims == 3 ? 8 : 4;
        for (int nn = 0; nn < nc; nn++) {
            const double w = ((nn & 1) ? dx : 1.0 - dx) * ((nn & 2) ? dy : 1.0 - dy) * ((nn & 4) ? dz : 1.0 - dz);
            const int a = wrap_node(i + (nn & 1), g->nx), b = wrap_node(j + ((nn >> 1) & 1), g->ny);
            const int cc = g->dims == 3 ? wrap_node(k + ((nn >> 2) & 1), g->nz) : 1;
            rho[ID(g, a, b, cc)] += q * w;
            if (q > 0) rho_pos[ID(g, a, b, cc)] += q * w;
        }
    }
    double res = 0, rmax = 0;
    const int k1 = g->dims == 3 ? 3 : 1, k2 = g->dims == 3 ? g->mz - 3 : 1;
    for (int k = k1; k <= k2; k++)
        for (int j = 3; j <= g->my - 3; j++)
            for (int i = 3; i <= g->mx - 3; i++) {
                double div = (f->Ex[ID(g, i, j, k)] - f->Ex[ID(g, i - 1, j, k)]) + (f->Ey[ID(g, i, j, k)] - f->Ey[ID(g, i, j - 1, k)]);
                if (g->dims == 3) div = div + (f->Ez[ID(g, i, j, k)] - f->Ez[ID(g, i, j, k - 1)]);
                const double r = fabs(div - rho[ID(g, i, j, k)]);
                if (r > res) res = r;
                if (fabs(rho_pos[ID(g, i, j, k)]) > rmax) rmax = fabs(rho_pos[ID(g, i, j, k)]);
            }
    free(rho);
    free(rho_pos);
    if (rho_max) *rho_max = rmax;
    return res;
}

/* ------------------------------------------------------------------------- */
/* Synthetic inputs: Philox-4x32-10 in place of gfortran random_number       */
/* ------------------------------------------------------------------------- */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

double orc_u01(uint32_t hi, uint32_t lo)
{
    const uint64_t b = (((uint64_t)hi << 32) | lo) >> 11;
    return (double)b * (1.0 / 9007199254740992.0);
}

/* prob_dist.F90:34-54 */
void orc_maxbolt_table(int n, double *X, double *P)
{
    const double dX = (15.0 - 0.0) / (double)(n - 1);
    for (int i = 1; i <= n; i++) X[i - 1] = dX * (double)(i - 1);
    double s = 0;
    P[0] = 0;
    for (int i = 2; i <= n; i++) {
        s = s + sqrt(X[i - 1]) * exp(-X[i - 1]);
        P[i - 1] = s;
    }
    for (int i = 0; i < n; i++) P[i] = P[i] / s;
}

/* prob_dist.F90:85-105 (1-based result) */
static int binary_search(int n, const double *A, double val)
{
    int imin = 1, imax = n, imid = (imin + imax) / 2, search = 1;
    while (search) {
        const int prev = imid;
        if (A[imid - 1] >= val) imax = imid;
        if (A[imid - 1] <= val) imin = imid;
        imid = (imin + imax) / 2;
        if (imin + 1 >= imax) search = 0;
        if (imid == prev) search = 0;
    }
    return imin;
}

/* prob_dist.F90:72-83 */
static double inv_pdf(const double *X, const double *P, double pdf, int idx)
{
    if (P[idx] == P[idx - 1]) return X[idx - 1];
    return X[idx - 1] + (X[idx] - X[idx - 1]) * ((pdf - P[idx - 1]) / (P[idx] - P[idx - 1]));
}

/* prob_dist.F90:223-254 */
static void add_drift_vel(double *u, double *v, double *w, double vx, double vy, double vz)
{
    const double drift = sqrt((vx * vx + vy * vy) + vz * vz);
    double beta, gamma;
    if (fabs(drift) < 1.0) {
        beta = drift;
        gamma = 1.0 / sqrt((1.0 - drift) * (1.0 + drift));
    } else {
        gamma = fabs(drift);
        beta = sqrt((drift - 1.0) * (drift + 1.0)) / drift;
    }
    double d[3] = {vx, vy, vz};
    const double mag = sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
    if (mag == 0) d[0] = d[1] = d[2] = 0;
    else { d[0] = d[0] / mag; d[1] = d[1] / mag; d[2] = d[2] / mag; }
    const double gm = sqrt(((1.0 + *u * *u) + *v * *v) + *w * *w);
    const double projn = (*u * d[0] + *v * d[1]) + *w * d[2];
    *u = (*u + ((gamma - 1.0) * projn) * d[0]) + ((gamma * beta) * gm) * d[0];
    *v = (*v + ((gamma - 1.0) * projn) * d[1]) + ((gamma * beta) * gm) * d[1];
    *w = (*w + ((gamma - 1.0) * projn) * d[2]) + ((gamma * beta) * gm) * d[2];
}

int64_t orc_load_weibel(const orc_weibel *wb, orc_particles *p)
{
    enum { NT = 10000 };
    static double X[NT], P[NT];
    orc_maxbolt_table(NT, X, P);
    const uint32_t key[2] = {wb->seed, 0x50494354u};
    const double x1 = 0, x2 = wb->nx, y1 = 0, y2 = wb->ny, z1 = 0, z2 = wb->dims == 3 ? wb->nz : 1;
    const double zmin = wb->dims == 3 ? 3.0 : 1.0;
    /* init_prtl.F90:190 */
    const int64_t ntrial = (int64_t)(wb->epc * fmax(0.0, x2 - x1) * fmax(0.0, y2 - y1) * fmax(0.0, z2 - z1));
    p->used = 0;
    for (uint32_t call = 0; call < 2; call++) {
        for (int64_t n = 0; n < ntrial; n++) {
            uint32_t r[4], ctr[4] = {(uint32_t)n, call, 0, 0};
            orc_philox4x32_10(ctr, key, r);
            const double r1 = orc_u01(r[0], r[1]), r2 = orc_u01(r[2], r[3]);
            ctr[2] = 1;
            orc_philox4x32_10(ctr, key, r);
            const double r3 = orc_u01(r[0], r[1]), racpt = orc_u01(r[2], r[3]);
            const double xg = x1 + r1 * (x2 - x1), yg = y1 + r2 * (y2 - y1), zg = z1 + r3 * (z2 - z1);
            if (!(racpt <= wb->density)) continue;                         /* :209 */
            const double xl = (xg - 0.0) + 3.0, yl = (yg - 0.0) + 3.0, zl = (zg - 0.0) + zmin;
            for (int s = 0; s < 2; s++) {                                  /* InsertPrtl_PSP */
                const double temp = s == 0 ? wb->temp_ion : wb->temp_elc;
                ctr[2] = 2 + s;
                orc_philox4x32_10(ctr, key, r);
                const double rmb = orc_u01(r[0], r[1]), riso2 = orc_u01(r[2], r[3]);
                ctr[2] = 4 + s;
                orc_philox4x32_10(ctr, key, r);
                const double riso3 = orc_u01(r[0], r[1]);
                /* GetVelGamma_MaxBolt, prob_dist.F90:13-30 */
                const int idx = binary_search(NT, P, rmb);
                double beta = inv_pdf(X, P, rmb, idx);
                beta = sqrt(beta * temp);
                if (beta >= 1.0) beta = 0.0;
                const double gamma = 1.0 / sqrt((1.0 + beta) * (1.0 - beta));
                /* iso3vel, prob_dist.F90:56-70 */
                const double ct = 2.0 * riso2 - 1.0;
                const double st = sqrt(1.0 - ct * ct);
                const double phi = (2.0 * PI_PSN) * riso3;
                double u = (gamma * beta) * ct;
                double v = ((gamma * beta) * st) * cos(phi);
                double w = ((gamma * beta) * st) * sin(phi);
                /* setup_weibel.F90:23-24: call 0 drifts flavour 1 left and
                   flavour 2 right, call 1 the reverse. */
                const double sgn = ((call == 0) == (s == 0)) ? -1.0 : 1.0;
                add_drift_vel(&u, &v, &w, sgn * wb->drift, 0.0, 0.0);
                if (p->used >= p->capacity) return -1;
                const int64_t d = p->used++;
                p->x[d] = xl; p->y[d] = yl; p->z[d] = zl;
                p->u[d] = u; p->v[d] = v; p->w[d] = w;
                p->q[d] = (1.0 * (s == 0 ? 1.0 : -1.0)) * 1.0;             /* :161 */
                p->flv[d] = s + 1;
            }
        }
    }
    return p->used;
}

/* InjectNewPrtl (bc_inflow.F90:134-189) with SetInjDomain (:191-235),
   GetIntPoissonDist (prob_dist.F90:194-216), GetNewPrtlPos
   (bc_inflow.F90:237-256) and InsertPrtl_PSP (init_prtl.F90:138-169) on one
   rank, for a uniform density and drift; the draws are Philox-4x32-10
   (counter trial, call, stream; key seed, "INJC"; the Poisson draw at trial
   0xFFFFFFFF).  Returns the particles appended, or -1 (none appended) past
   the capacity. */
int64_t orc_inject(const orc_grid *g, orc_particles *p, const orc_inflow *f)
{
    enum { NT = 10000 };
    static double X[NT], P[NT];
    orc_maxbolt_table(NT, X, P);
    const uint32_t key[2] = {f->seed, 0x494E4A43u};
    double x1 = 3.0, x2 = g->mx - 2, y1 = 3.0, y2 = g->my - 2;
    double z1 = g->dims == 3 ? 3.0 : 1.0, z2 = g->dims == 3 ? g->mz - 2 : 2.0;
    const double pos = f->pos, vc = f->vmax * g->c, shift = f->speed * g->c;
    const int side = f->face;
    if (side == 1) { x1 = fmax(pos - shift, 0.0) - 0.0 + 3; x2 = fmin(pos + vc, (double)g->nx) - 0.0 + 3; }
    if (side == 2) { x1 = fmax(pos - vc, 0.0) - 0.0 + 3; x2 = fmin(pos + shift, (double)g->nx) - 0.0 + 3; }
    if (side == 3) { y1 = fmax(pos - shift, 0.0) - 0.0 + 3; y2 = fmin(pos + vc, (double)g->ny) - 0.0 + 3; }
    if (side == 4) { y1 = fmax(pos - vc, 0.0) - 0.0 + 3; y2 = fmin(pos + shift, (double)g->ny) - 0.0 + 3; }
    if (side == 5) { z1 = fmax(pos - shift, 0.0) - 0.0 + 3; z2 = fmin(pos + vc, (double)g->nz) - 0.0 + 3; }
    if (side == 6) { z1 = fmax(pos - vc, 0.0) - 0.0 + 3; z2 = fmin(pos + shift, (double)g->nz) - 0.0 + 3; }
    int64_t n = (int64_t)(f->epc * fmax(0.0, x2 - x1) * fmax(0.0, y2 - y1) * fmax(0.0, z2 - z1));
    if (n <= 0) return 0;
    if (n < 1000) {
        uint32_t r[4], ctr[4] = {0xFFFFFFFFu, f->call, 0, 0};
        orc_philox4x32_10(ctr, key, r);
        const double r1 = orc_u01(r[0], r[1]);
        const double mean = (double)n;
        double sum = exp(-mean), sum_logn = 0;
        const double log_mean = log(mean);
        int64_t k = 0;
        while (sum < r1) {
            k = k + 1;
            sum_logn = sum_logn + log((double)k);
            sum = sum + exp(-mean + (double)k * log_mean - sum_logn);
            if (k > 10000) break;
        }
        n = k;
    }
    const int64_t used0 = p->used;
    for (int64_t t = 0; t < n; t++) {
        uint32_t r[4], ctr[4] = {(uint32_t)t, f->call, 0, 0};
        orc_philox4x32_10(ctr, key, r);
        const double r1 = orc_u01(r[0], r[1]), r2 = orc_u01(r[2], r[3]);
        ctr[2] = 1;
        orc_philox4x32_10(ctr, key, r);
        const double r3 = orc_u01(r[0], r[1]), racpt = orc_u01(r[2], r[3]);
        const double xl = x1 + r1 * (x2 - x1), yl = y1 + r2 * (y2 - y1), zl = z1 + r3 * (z2 - z1);
        const double xg = xl + (0.0 - 3.0), yg = yl + (0.0 - 3.0), zg = g->dims == 3 ? zl + (0.0 - 3.0) : zl;
        int acpt = racpt <= f->density;
        if (side == 1 && xg > pos + f->drift[0] * g->c) acpt = 0;
        if (side == 2 && xg < pos + f->drift[0] * g->c) acpt = 0;
        if (side == 3 && yg > pos + f->drift[1] * g->c) acpt = 0;
        if (side == 4 && yg < pos + f->drift[1] * g->c) acpt = 0;
        if (side == 5 && zg > pos + f->drift[2] * g->c) acpt = 0;
        if (side == 6 && zg < pos + f->drift[2] * g->c) acpt = 0;
        if (!acpt) continue;
        for (int sp = 0; sp < f->nspecies; sp++) {
            ctr[2] = 2 + 2 * sp;
            orc_philox4x32_10(ctr, key, r);
            const double rmb = orc_u01(r[0], r[1]), riso2 = orc_u01(r[2], r[3]);
            ctr[2] = 3 + 2 * sp;
            orc_philox4x32_10(ctr, key, r);
            const double riso3 = orc_u01(r[0], r[1]);
            const int idx = binary_search(NT, P, rmb);
            double beta = inv_pdf(X, P, rmb, idx);
            beta = sqrt(beta * f->temp[sp]);
            if (beta >= 1.0) beta = 0.0;
            const double gamma = 1.0 / sqrt((1.0 + beta) * (1.0 - beta));
            const double ct = 2.0 * riso2 - 1.0;
            const double st = sqrt(1.0 - ct * ct);
            const double phi = (2.0 * PI_PSN) * riso3;
            double u = (gamma * beta) * ct;
            double v = ((gamma * beta) * st) * cos(phi);
            double w = ((gamma * beta) * st) * sin(phi);
            add_drift_vel(&u, &v, &w, f->drift[0], f->drift[1], f->drift[2]);
            if (p->used >= p->capacity) { p->used = used0; return -1; }
            const int64_t d = p->used++;
            p->x[d] = xl; p->y[d] = yl; p->z[d] = zl;
            p->u[d] = u; p->v[d] = v; p->w[d] = w;
            p->q[d] = f->charge[sp];
            p->flv[d] = f->flv[sp];
        }
    }
    return p->used - used0;
}

/* ---- convolutional PML, bc_pml.F90 ------------------------------------- */

/* The profile of every face: pml_pos / pml_pos_ind of Update_PML_Position
   (bc_pml.F90:56-71) and pml_params_arr as SetPMLParameters (:42-53) sets a
   'pml' face; the other faces keep the type's defaults (:6-12) and the
   +-huge(1) positions.  alpha_max is the default-kind literal 9.0e-4. */
typedef struct {
    double pos[6], ind[6], L[6], kmax[6], smax[6], amax[6];
    int n[6];
} pml_profile;

static void pml_profile_init(const orc_pml *p, pml_profile *q)
{
    const double huge = 2147483647.0;   /* huge(1) */
    for (int f = 0; f < 6; f++) {
        const int upper = f & 1;        /* bc_face 2, 4, 6 */
        q->n[f] = 4;
        q->kmax[f] = 1.0;
        if ((p->faces >> f) & 1) {
            q->L[f] = p->thickness[f];
            q->smax[f] = 1.0;
            q->amax[f] = (double)9.0e-4f;
            q->pos[f] = p->pos[f];
            q->ind[f] = upper ? ceil(p->pos[f]) + 1.0 : floor(p->pos[f]) - 1.0;
        } else {
            q->L[f] = 10.0;
            q->smax[f] = 0.0;
            q->amax[f] = 1.0;
            q->pos[f] = upper ? huge : -huge;
            q->ind[f] = upper ? huge : -huge;
        }
    }
}

/* x**n for an integer n >= 0 by squaring, as gfortran evaluates a real to a
   variable integer power. */
static double ipow(double x, int n)
{
    double y = (n & 1) ? x : 1.0;
    while (n >>= 1) {
        x = x * x;
        if (n & 1) y = y * x;
    }
    return y;
}

static double pml_kappa(const pml_profile *q, double d, int f)   /* :330-335 */
{
    const double k = 1.0 + ipow(d / q->L[f], q->n[f]) * (q->kmax[f] - 1.0);
    return q->kmax[f] < k ? q->kmax[f] : k;
}
static double pml_sigma(const pml_profile *q, double d, int f)   /* :337-341 */
{
    const double s = q->smax[f] * ipow(d / q->L[f], q->n[f]);
    return q->smax[f] < s ? q->smax[f] : s;
}

/* pml_c (:271-288) */
static double pml_c(const pml_profile *q, double fc, double x, int axis)
{
    double c = 0.0;
    const int lo = 2 * axis, hi = 2 * axis + 1;
    if (x > q->pos[hi]) c = fc * (1.0 / pml_kappa(q, x - q->pos[hi], hi) - 1.0);
    if (x < q->pos[lo]) c = fc * (1.0 / pml_kappa(q, q->pos[lo] - x, lo) - 1.0);
    return c;
}

/* pml_ab (:290-316) */
static void pml_ab(const pml_profile *q, double x, int axis, double *a, double *b)
{
    const int lo = 2 * axis, hi = 2 * axis + 1;
    *a = 0.0;
    *b = 0.0;
    for (int side = 0; side < 2; side++) {
        const int f = side == 0 ? hi : lo;
        if (side == 0 ? !(x > q->pos[hi]) : !(x < q->pos[lo])) continue;
        const double d = side == 0 ? x - q->pos[hi] : q->pos[lo] - x;
        const double alpha = q->amax[f], sigma = pml_sigma(q, d, f), kappa = pml_kappa(q, d, f);
        *a = exp(-(sigma / kappa) - alpha);
        *b = (sigma / (sigma * kappa + alpha * (kappa * kappa))) * (*a - 1.0);
    }
}

/* no_pml_this_domain (:67-69) with xborders = yborders = zborders = 0 */
static int pml_outside_grid(const orc_grid *g, const pml_profile *q)
{
    return 1 - 3 > q->ind[0] && g->mx - 3 < q->ind[1] && 1 - 3 > q->ind[2] && g->my - 3 < q->ind[3] &&
           1 - 3 > q->ind[4] && g->mz - 3 < q->ind[5];
}

/* beyond the layer of the faces of one axis: x < pos(lo) - L(lo) or x > pos(hi) + L(hi) */
static int pml_beyond(const pml_profile *q, double x, int axis)
{
    return x < q->pos[2 * axis] - q->L[2 * axis] || x > q->pos[2 * axis + 1] + q->L[2 * axis + 1];
}

/* UpdateElcFld_PML (bc_pml.F90:83-144): E = E + the convolution terms at the
   cells outside the interior box; E beyond the layers zeroed. */
void orc_pml_e(const orc_grid *g, orc_fields *f, orc_pml *p)
{
    pml_profile q;
    pml_profile_init(p, &q);
    if (pml_outside_grid(g, &q)) return;
    const int three_d = g->dims == 3;
    const double fc = g->c;
    double *p1x = p->psiE[0], *p1y = p->psiE[1], *p1z = p->psiE[2];
    double *p2x = p->psiE[3], *p2y = p->psiE[4], *p2z = p->psiE[5];
    const int k0 = three_d ? 2 : 1, k1 = three_d ? g->mz - 1 : 1;
    for (int k = k0; k <= k1; k++)
        for (int j = 2; j <= g->my - 1; j++)
            for (int i = 2; i <= g->mx - 1; i++) {
                const double xg = i - 3, yg = j - 3, zg = k - 3;
                const int inside = xg > q.ind[0] && xg < q.ind[1] && yg > q.ind[2] && yg < q.ind[3] &&
                                   zg > q.ind[4] && zg < q.ind[5];
                if (inside) continue;
                double ax, bx, ay, by, az, bz;
                pml_ab(&q, xg, 0, &ax, &bx);
                pml_ab(&q, yg, 1, &ay, &by);
                pml_ab(&q, zg, 2, &az, &bz);
                const double cx = pml_c(&q, fc, xg, 0), cy = pml_c(&q, fc, yg, 1), cz = pml_c(&q, fc, zg, 2);
                const int64_t c = ID(g, i, j, k), cxm = ID(g, i - 1, j, k), cym = ID(g, i, j - 1, k);
                const int64_t czm = three_d ? ID(g, i, j, k - 1) : c;
                p1x[c] = ay * p1x[c] + (by * fc) * (f->Bz[c] - f->Bz[cym]);
                p1z[c] = ax * p1z[c] + (bx * fc) * (f->By[c] - f->By[cxm]);
                if (three_d) {
                    p1y[c] = az * p1y[c] + (bz * fc) * (f->Bx[c] - f->Bx[czm]);
                    p2x[c] = az * p2x[c] + (bz * fc) * (f->By[c] - f->By[czm]);
                }
                p2y[c] = ax * p2y[c] + (bx * fc) * (f->Bz[c] - f->Bz[cxm]);
                p2z[c] = ay * p2z[c] + (by * fc) * (f->Bx[c] - f->Bx[cym]);
                if (three_d) {
                    f->Ex[c] = ((f->Ex[c] + cy * (f->Bz[c] - f->Bz[cym])) - cz * (f->By[c] - f->By[czm])) + p1x[c] - p2x[c];
                    f->Ey[c] = ((f->Ey[c] + cz * (f->Bx[c] - f->Bx[czm])) - cx * (f->Bz[c] - f->Bz[cxm])) + p1y[c] - p2y[c];
                } else {
                    f->Ex[c] = (f->Ex[c] + cy * (f->Bz[c] - f->Bz[cym])) + p1x[c];
                    f->Ey[c] = (f->Ey[c] - cx * (f->Bz[c] - f->Bz[cxm])) - p2y[c];
                }
                f->Ez[c] = ((f->Ez[c] + cx * (f->By[c] - f->By[cxm])) - cy * (f->Bx[c] - f->Bx[cym])) + p1z[c] - p2z[c];
                if (pml_beyond(&q, xg + 0.5, 0) || pml_beyond(&q, yg, 1) || pml_beyond(&q, zg, 2)) f->Ex[c] = 0.0;
                if (pml_beyond(&q, xg, 0) || pml_beyond(&q, yg + 0.5, 1) || pml_beyond(&q, zg, 2)) f->Ey[c] = 0.0;
                if (pml_beyond(&q, xg, 0) || pml_beyond(&q, yg, 1) || pml_beyond(&q, zg + 0.5, 2)) f->Ez[c] = 0.0;
            }
}

/* UpdateMagFld_PML (bc_pml.F90:146-264): the same for B at the half-cell
   positions; the interior test on the integer ones. */
void orc_pml_b(const orc_grid *g, orc_fields *f, orc_pml *p)
{
    pml_profile q;
    pml_profile_init(p, &q);
    if (pml_outside_grid(g, &q)) return;
    const int three_d = g->dims == 3;
    const double fc = g->c;
    double *p1x = p->psiB[0], *p1y = p->psiB[1], *p1z = p->psiB[2];
    double *p2x = p->psiB[3], *p2y = p->psiB[4], *p2z = p->psiB[5];
    const int k0 = three_d ? 2 : 1, k1 = three_d ? g->mz - 1 : 1;
    for (int k = k0; k <= k1; k++)
        for (int j = 2; j <= g->my - 1; j++)
            for (int i = 2; i <= g->mx - 1; i++) {
                const int inside = i - 3 > q.ind[0] && i - 3 < q.ind[1] && j - 3 > q.ind[2] && j - 3 < q.ind[3] &&
                                   k - 3 > q.ind[4] && k - 3 < q.ind[5];
                if (inside) continue;
                const double xg = (i - 3) + 0.5, yg = (j - 3) + 0.5, zg = (k - 3) + 0.5;
                double ax, bx, ay, by, az, bz;
                pml_ab(&q, xg, 0, &ax, &bx);
                pml_ab(&q, yg, 1, &ay, &by);
                pml_ab(&q, zg, 2, &az, &bz);
                const double cx = pml_c(&q, fc, xg, 0), cy = pml_c(&q, fc, yg, 1), cz = pml_c(&q, fc, zg, 2);
                const int64_t c = ID(g, i, j, k), cxp = ID(g, i + 1, j, k), cyp = ID(g, i, j + 1, k);
                const int64_t czp = three_d ? ID(g, i, j, k + 1) : c;
                p1x[c] = ay * p1x[c] + (by * fc) * (f->Ez[cyp] - f->Ez[c]);
                p1z[c] = ax * p1z[c] + (bx * fc) * (f->Ey[cxp] - f->Ey[c]);
                if (three_d) {
                    p1y[c] = az * p1y[c] + (bz * fc) * (f->Ex[czp] - f->Ex[c]);
                    p2x[c] = az * p2x[c] + (bz * fc) * (f->Ey[czp] - f->Ey[c]);
                }
                p2y[c] = ax * p2y[c] + (bx * fc) * (f->Ez[cxp] - f->Ez[c]);
                p2z[c] = ay * p2z[c] + (by * fc) * (f->Ex[cyp] - f->Ex[c]);
                if (three_d) {
                    f->Bx[c] = ((f->Bx[c] - cy * (f->Ez[cyp] - f->Ez[c])) + cz * (f->Ey[czp] - f->Ey[c])) - p1x[c] + p2x[c];
                    f->By[c] = ((f->By[c] - cz * (f->Ex[czp] - f->Ex[c])) + cx * (f->Ez[cxp] - f->Ez[c])) - p1y[c] + p2y[c];
                } else {
                    f->Bx[c] = (f->Bx[c] - cy * (f->Ez[cyp] - f->Ez[c])) - p1x[c];
                    f->By[c] = (f->By[c] + cx * (f->Ez[cxp] - f->Ez[c])) + p2y[c];
                }
                f->Bz[c] = ((f->Bz[c] - cx * (f->Ey[cxp] - f->Ey[c])) + cy * (f->Ex[cyp] - f->Ex[c])) - p1z[c] + p2z[c];
                if (pml_beyond(&q, xg - 0.5, 0) || pml_beyond(&q, yg, 1) || pml_beyond(&q, zg, 2)) f->Bx[c] = 0.0;
                if (pml_beyond(&q, xg, 0) || pml_beyond(&q, yg - 0.5, 1) || pml_beyond(&q, zg, 2)) f->By[c] = 0.0;
                if (pml_beyond(&q, xg, 0) || pml_beyond(&q, yg, 1) || pml_beyond(&q, zg - 0.5, 2)) f->Bz[c] = 0.0;
            }
}
