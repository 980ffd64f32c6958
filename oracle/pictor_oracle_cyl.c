/*
 * pictor_oracle_cyl.c -- CPU restatement (FP64) of PICTOR's cylindrical
 * (r, theta, z) step: src/cyl/cyl_common.F90, cyl_em_update.F90 (Yee),
 * cyl_em_update_lehe.F90 (Lehe, restated with its syntax errors fixed),
 * cyl_movdep_strang.F90 (Strang-split mover, near-axis sub-stepping,
 * AxisCurrentBC) and src/movdep/deposit.F90 (the scalar deposit the
 * sub-stepper uses).
 *
 * TEST INFRASTRUCTURE ONLY (see pictor_oracle.h); parity against the
 * reference itself is unpinned.
 *
 * Set-up restated: one rank holding the axis (inc_axis, procxind = 0,
 * xborders(0) = 0), 3D grid x = r, y = theta, z; the theta and z faces are
 * periodic, the r faces are not (PeriodicX_Off, subdomains.F90:493-501, as
 * SetBC_* does for a cylinder): no halo copy or current fold across them, and
 * particles leaving through r = r_max are dropped (LoadPrtlOutliers sends
 * them to MPI_PROC_NULL).  InitParam_cyl sets indepLBaxis = 2 when the axis
 * is included (cyl_common.F90:26), which changes the order and the ranges of
 * the halo and fold exchanges; both are restated.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "pictor_oracle.h"

#define ID(g, i, j, k) ((int64_t)((i) - 1) + (int64_t)(g)->mx * ((int64_t)((j) - 1) + (int64_t)(g)->my * (int64_t)((k) - 1)))

static const double PI_PSN = 3.14159265358979323846264;

/* InitParam_cyl, cyl_common.F90:19-32 */
void orc_cyl_params(const orc_grid *g, double out[4])
{
    const double dtheta = 2.0 * PI_PSN / g->ny;
    out[0] = dtheta;
    out[1] = 4.0 / g->ny;          /* ax_perm_area */
    out[2] = 1.0 / dtheta;         /* inv_dtheta   */
    out[3] = -0.5;                 /* rshift       */
}

/* --- halo and fold (comm_fld.F90 with indepLBaxis = 2, x faces closed) --- */
static void copy_layers(const orc_grid *g, double *F, int axis, int ilo, int ihi, int jlo, int jhi, int klo, int khi)
{
    const int m = axis == 1 ? g->my : g->mz;
    for (int k = klo; k <= khi; k++)
        for (int j = jlo; j <= jhi; j++)
            for (int i = ilo; i <= ihi; i++) {
                const int a = axis == 1 ? j : k;
                if (a != 1) continue;
                for (int l = 0; l < 3; l++) {
                    int dj = j, dk = k, sj = j, sk = k;
                    if (axis == 1) { dj = m - 2 + l; sj = 3 + l; } else { dk = m - 2 + l; sk = 3 + l; }
                    F[ID(g, i, dj, dk)] = F[ID(g, i, sj, sk)];
                }
                for (int l = 0; l < 2; l++) {
                    int dj = j, dk = k, sj = j, sk = k;
                    if (axis == 1) { dj = 1 + l; sj = m - 4 + l; } else { dk = 1 + l; sk = m - 4 + l; }
                    F[ID(g, i, dj, dk)] = F[ID(g, i, sj, sk)];
                }
            }
}

/* SendRecvFlds: x faces closed, y faces (x 1..mx, z 3..mz-3), then z faces
   (full x, y): comm_fld.F90:75-91 with the ranges of SetCommFldDomain. */
void orc_cyl_send_recv_flds(const orc_grid *g, double *Fx, double *Fy, double *Fz)
{
    double *F[3] = {Fx, Fy, Fz};
    for (int c = 0; c < 3; c++) copy_layers(g, F[c], 1, 1, g->mx, 1, 1, 3, g->mz - 3);
    for (int c = 0; c < 3; c++) copy_layers(g, F[c], 2, 1, g->mx, 1, g->my, 1, 1);
}

static void fold_layers(const orc_grid *g, double *F, int axis, int ilo, int ihi, int jlo, int jhi, int klo, int khi)
{
    const int m = axis == 1 ? g->my : g->mz;
    for (int k = klo; k <= khi; k++)
        for (int j = jlo; j <= jhi; j++)
            for (int i = ilo; i <= ihi; i++) {
                double hi3[3], lo2[2];
                for (int l = 0; l < 3; l++) hi3[l] = axis == 1 ? F[ID(g, i, m - 2 + l, k)] : F[ID(g, i, j, m - 2 + l)];
                for (int l = 0; l < 2; l++) lo2[l] = axis == 1 ? F[ID(g, i, 1 + l, k)] : F[ID(g, i, j, 1 + l)];
                for (int l = 0; l < 3; l++) {
                    const int64_t d = axis == 1 ? ID(g, i, 3 + l, k) : ID(g, i, j, 3 + l);
                    F[d] = F[d] + hi3[l];
                }
                for (int l = 0; l < 2; l++) {
                    const int64_t d = axis == 1 ? ID(g, i, m - 4 + l, k) : ID(g, i, j, m - 4 + l);
                    F[d] = F[d] + lo2[l];
                }
            }
}

/* UpdateCurrentAllFaces, comm_fld.F90:15-33 with indepLBaxis = 2: z faces
   (full x, y) first, then y faces (x 1..mx, z 3..mz-3). */
void orc_cyl_fold(const orc_grid *g, double *Jx, double *Jy, double *Jz)
{
    double *F[3] = {Jx, Jy, Jz};
    for (int c = 0; c < 3; c++) fold_layers(g, F[c], 2, 1, g->mx, 1, g->my, 1, 1);
    for (int c = 0; c < 3; c++) fold_layers(g, F[c], 1, 1, g->mx, 1, 1, 3, g->mz - 3);
}

/* --- field solver --------------------------------------------------------- */

static void axis_partner(const orc_grid *g, int j, int *jpp)
{
    const int ny = g->ny;
    int p = j + ny / 2;
    if (p > g->my - 3) p = p - ny;
    *jpp = p;
}

/* UpdateEFldAxis, cyl_em_update.F90:143-185 */
static void e_axis(const orc_grid *g, orc_fields *f)
{
    for (int k = 1; k <= g->mz; k++)
        for (int j = 1; j <= g->my; j++) {
            int jpp;
            axis_partner(g, j, &jpp);
            f->Ex[ID(g, 3, j, k)] = 0.5 * (f->Ex[ID(g, 4, j, k)] - f->Ex[ID(g, 4, jpp, k)]);
            f->Ex[ID(g, 2, j, k)] = -f->Ex[ID(g, 4, jpp, k)];
            f->Ey[ID(g, 3, j, k)] = -f->Ey[ID(g, 4, jpp, k)];
            f->Ez[ID(g, 3, j, k)] = f->Ez[ID(g, 4, jpp, k)];
        }
}

/* UpdateBFldAxis, cyl_em_update.F90:187-227 */
static void b_axis(const orc_grid *g, orc_fields *f)
{
    for (int k = 1; k <= g->mz; k++)
        for (int j = 1; j <= g->my; j++) {
            int jpp;
            axis_partner(g, j, &jpp);
            f->By[ID(g, 3, j, k)] = 0.5 * (f->By[ID(g, 4, j, k)] - f->By[ID(g, 4, jpp, k)]);
            f->By[ID(g, 2, j, k)] = -f->By[ID(g, 4, jpp, k)];
            f->Bx[ID(g, 3, j, k)] = -f->Bx[ID(g, 4, jpp, k)];
            f->Bz[ID(g, 2, j, k)] = f->Bz[ID(g, 4, jpp, k)];
        }
}

/* Lehe (cyl_em_update_lehe.F90:6-17, 255-289, trailing "+ &" removed) */
static void cyl_lehe(const orc_grid *g, double dtheta, double L[12])
{
    const double c = g->c, cinv = 1.0 / c;
    L[3] = 0.0;                                            /* beta_xy */
    L[4] = 0.125;                                          /* beta_xz */
    L[5] = 0.0;                                            /* beta_yx */
    L[6] = 0.125;                                          /* beta_yz */
    L[7] = 0.125 * ((1.0 / 1.0) * (1.0 / 1.0));            /* beta_zx = 0.125*(dz/dx)^2 */
    L[8] = 0.125 * ((1.0 / (1.0 * dtheta)) * (1.0 / (1.0 * dtheta))); /* beta_zy */
    L[9] = 0.0; L[10] = 0.0;
    const double s = sin((0.5 * PI_PSN) * c);
    L[11] = 0.25 * (1.0 - (cinv * cinv) * (s * s));       /* delta_z */
    L[0] = ((1.0 - 2.0 * L[3]) - 2.0 * L[4]) - 3.0 * L[9];
    L[1] = ((1.0 - 2.0 * L[5]) - 2.0 * L[6]) - 3.0 * L[10];
    L[2] = ((1.0 - 2.0 * L[7]) - 2.0 * L[8]) - 3.0 * L[11];
}

static double lgx(const orc_grid *g, const double *L, const double *F, int i, int j, int k)
{
    double r = L[0] * (F[ID(g, i + 1, j, k)] - F[ID(g, i, j, k)]);
    r = r + L[4] * (F[ID(g, i + 1, j, k + 1)] - F[ID(g, i, j, k + 1)]);
    r = r + L[4] * (F[ID(g, i + 1, j, k - 1)] - F[ID(g, i, j, k - 1)]);
    return r;
}

static double lgx1(const orc_grid *g, const double *L, const double *F, int i, int j, int k, double rp, double rr)
{
    double r = L[0] * (rp * F[ID(g, i + 1, j, k)] - rr * F[ID(g, i, j, k)]);
    r = r + L[4] * (rp * F[ID(g, i + 1, j, k + 1)] - rr * F[ID(g, i, j, k + 1)]);
    r = r + L[4] * (rp * F[ID(g, i + 1, j, k - 1)] - rr * F[ID(g, i, j, k - 1)]);
    return r;
}

static double lgy(const orc_grid *g, const double *L, const double *F, int i, int j, int k)
{
    double r = (L[1] * 1.0) * (F[ID(g, i, j + 1, k)] - F[ID(g, i, j, k)]);
    r = r + (L[6] * 1.0) * (F[ID(g, i, j + 1, k + 1)] - F[ID(g, i, j, k + 1)]);
    r = r + (L[6] * 1.0) * (F[ID(g, i, j + 1, k - 1)] - F[ID(g, i, j, k - 1)]);
    return r;
}

static double lgz(const orc_grid *g, const double *L, const double *F, int i, int j, int k)
{
    double r = L[2] * (F[ID(g, i, j, k + 1)] - F[ID(g, i, j, k)]);
    r = r + L[7] * (F[ID(g, i + 1, j, k + 1)] - F[ID(g, i + 1, j, k)]);
    r = r + L[7] * (F[ID(g, i - 1, j, k + 1)] - F[ID(g, i - 1, j, k)]);
    r = r + L[8] * (F[ID(g, i, j + 1, k + 1)] - F[ID(g, i, j + 1, k)]);
    r = r + L[8] * (F[ID(g, i, j - 1, k + 1)] - F[ID(g, i, j - 1, k)]);
    r = r + L[11] * (F[ID(g, i, j, k + 2)] - F[ID(g, i, j, k - 1)]);
    return r;
}

/* UpdateBfieldHalf, cyl_em_update.F90:49-110 / cyl_em_update_lehe.F90:62-118.
   The Lehe loop keeps k in 2..mz-2 so that the delta_z stencil (k-1, k+2)
   stays inside the array; the shipped file indexes k = 0 and mz+1 at the loop
   ends, which are ghost layers the z halo overwrites anyway. */
void orc_cyl_update_b_half(const orc_grid *g, orc_fields *f)
{
    double P[4];
    orc_cyl_params(g, P);
    const double dtheta = P[0], ax = P[1], rmin = 0.0 + P[3];
    const double h = (g->c * 0.5) * 1.0;
    double L[12];
    if (g->fdtd == 1) cyl_lehe(g, dtheta, L);
    const int k1 = g->fdtd == 1 ? 2 : 1, k2 = g->fdtd == 1 ? g->mz - 2 : g->mz - 1;
    for (int k = k1; k <= k2; k++)
        for (int j = 1; j <= g->my - 1; j++)
            for (int i = 4; i <= g->mx - 1; i++) {
                const double r = (((double)i - 3.0) + rmin) * 1.0;
                const double rp_half = r + 0.5 * 1.0, rp = r + 1.0;
                const int64_t c0 = ID(g, i, j, k);
                if (g->fdtd == 0) {
                    f->Bx[c0] = (f->Bx[c0] - (h * (f->Ez[ID(g, i, j + 1, k)] - f->Ez[c0])) / (r * dtheta)) +
                                (h * 1.0) * (f->Ey[ID(g, i, j, k + 1)] - f->Ey[c0]);
                    f->By[c0] = (f->By[c0] - (h * 1.0) * (f->Ex[ID(g, i, j, k + 1)] - f->Ex[c0])) +
                                (h * 1.0) * (f->Ez[ID(g, i + 1, j, k)] - f->Ez[c0]);
                    f->Bz[c0] = f->Bz[c0] - (h * ((1.0 * (rp * f->Ey[ID(g, i + 1, j, k)] - r * f->Ey[c0])) -
                                                  (f->Ex[ID(g, i, j + 1, k)] - f->Ex[c0]) / dtheta)) / rp_half;
                } else {
                    f->Bx[c0] = (f->Bx[c0] - (h * lgy(g, L, f->Ez, i, j, k)) / (r * dtheta)) +
                                (h * 1.0) * lgz(g, L, f->Ey, i, j, k);
                    f->By[c0] = (f->By[c0] - (h * 1.0) * lgz(g, L, f->Ex, i, j, k)) + (h * 1.0) * lgx(g, L, f->Ez, i, j, k);
                    f->Bz[c0] = f->Bz[c0] - (h * ((1.0 * lgx1(g, L, f->Ey, i, j, k, rp, r)) -
                                                  lgy(g, L, f->Ex, i, j, k) / dtheta)) / rp_half;
                }
            }
    /* UpdateBzAxis (cyl_em_update.F90:231-246) then Bz(3,j,k) = Bz_ax(k) */
    double *bzax = (double *)calloc((size_t)g->mz + 1, sizeof(double));
    for (int k = 1; k <= g->mz - 1; k++) {
        double s = 0.0;
        for (int j = 3; j <= g->my - 3; j++) s = s - (h * ax) * f->Ey[ID(g, 4, j, k)];
        bzax[k] = f->Bz[ID(g, 3, 3, k)] + s;
    }
    for (int k = 1; k <= g->mz - 1; k++)
        for (int j = 1; j <= g->my - 1; j++) f->Bz[ID(g, 3, j, k)] = bzax[k];
    free(bzax);
    b_axis(g, f);
}

/* UpdateEfield, cyl_em_update.F90:7-46 (Yee E in both schemes) */
void orc_cyl_update_e(const orc_grid *g, orc_fields *f)
{
    double P[4];
    orc_cyl_params(g, P);
    const double dtheta = P[0], rmin = 0.0 + P[3];
    const double fc = g->c * 1.0;
    for (int k = 3; k <= g->mz - 3; k++)
        for (int j = 3; j <= g->my - 3; j++)
            for (int i = 4; i <= g->mx - 3; i++) {
                const double r = (((double)i - 3.0) + rmin) * 1.0;
                const double rp_half = r + 0.5 * 1.0, rm_half = r - 0.5 * 1.0;
                const int64_t c0 = ID(g, i, j, k);
                f->Ex[c0] = (f->Ex[c0] + (fc * (f->Bz[c0] - f->Bz[ID(g, i, j - 1, k)])) / (rp_half * dtheta)) -
                            (fc * 1.0) * (f->By[c0] - f->By[ID(g, i, j, k - 1)]);
                f->Ey[c0] = (f->Ey[c0] + (fc * 1.0) * (f->Bx[c0] - f->Bx[ID(g, i, j, k - 1)])) -
                            (fc * 1.0) * (f->Bz[c0] - f->Bz[ID(g, i - 1, j, k)]);
                f->Ez[c0] = (f->Ez[c0] + ((fc * 1.0) * (rp_half * f->By[c0] - rm_half * f->By[ID(g, i - 1, j, k)])) / r) -
                            (fc * (f->Bx[c0] - f->Bx[ID(g, i, j - 1, k)])) / (r * dtheta);
            }
    e_axis(g, f);
}

/* AddCurrent, cyl_em_update.F90:114-140 (RZtwoD off) */
void orc_cyl_add_current(const orc_grid *g, orc_fields *f)
{
    double P[4];
    orc_cyl_params(g, P);
    const double dtheta = P[0], rmin = 0.0 + P[3];
    for (int k = 3; k <= g->mz - 3; k++)
        for (int j = 3; j <= g->my - 3; j++)
            for (int i = 4; i <= g->mx - 3; i++) {
                const double r = (((double)i - 3.0) + rmin) * 1.0;
                const double rp_half = r + 0.5 * 1.0;
                const int64_t c0 = ID(g, i, j, k);
                f->Ex[c0] = f->Ex[c0] - (f->Jx[c0] * 1.0) / (rp_half * dtheta);
                f->Ey[c0] = f->Ey[c0] - (f->Jy[c0] * 1.0) * 1.0;
                f->Ez[c0] = f->Ez[c0] - (f->Jz[c0] * 1.0) / (r * dtheta);
            }
    e_axis(g, f);
}

/* --- mover ----------------------------------------------------------------- */

/* Interp_VecEM_GridPoints (interpolation.F90:434-490) over the node values of
   GatherVecEfld/GatherVecBfld (3D). */
static void interp(const orc_grid *g, const orc_fields *f, double x, double y, double z, double pE[3], double pB[3])
{
    const int ip = (int)x, jp = (int)y, kp = (int)z;
    const double dx = x - ip, dy = y - jp, dz = z - kp;
    double wt[8];
    for (int nn = 0; nn < 8; nn++) {
        const double wx = (nn & 1) ? (0.0 + 1.0 * dx) : (1.0 + -1.0 * dx);
        const double wy = (nn & 2) ? (0.0 + 1.0 * dy) : (1.0 + -1.0 * dy);
        const double wz = (nn & 4) ? (0.0 + 1.0 * dz) : (1.0 + -1.0 * dz);
        wt[nn] = (wx * wy) * wz;
    }
    pE[0] = pE[1] = pE[2] = pB[0] = pB[1] = pB[2] = 0.0;
    for (int nn = 0; nn < 8; nn++) {
        const int a = ip + (nn & 1), b = jp + ((nn >> 1) & 1), c = kp + ((nn >> 2) & 1);
        const double vex = (f->Ex[ID(g, a - 1, b, c)] + f->Ex[ID(g, a, b, c)]) * 0.5;
        const double vey = (f->Ey[ID(g, a, b - 1, c)] + f->Ey[ID(g, a, b, c)]) * 0.5;
        const double vez = (f->Ez[ID(g, a, b, c - 1)] + f->Ez[ID(g, a, b, c)]) * 0.5;
        const double vbx = (((f->Bx[ID(g, a, b - 1, c - 1)] + f->Bx[ID(g, a, b, c - 1)]) + f->Bx[ID(g, a, b - 1, c)]) + f->Bx[ID(g, a, b, c)]) * 0.25 + g->bext[0];
        const double vby = (((f->By[ID(g, a - 1, b, c - 1)] + f->By[ID(g, a - 1, b, c)]) + f->By[ID(g, a, b, c - 1)]) + f->By[ID(g, a, b, c)]) * 0.25 + g->bext[1];
        const double vbz = (((f->Bz[ID(g, a - 1, b - 1, c)] + f->Bz[ID(g, a - 1, b, c)]) + f->Bz[ID(g, a, b - 1, c)]) + f->Bz[ID(g, a, b, c)]) * 0.25 + g->bext[2];
        pE[0] = pE[0] + wt[nn] * vex;
        pE[1] = pE[1] + wt[nn] * vey;
        pE[2] = pE[2] + wt[nn] * vez;
        pB[0] = pB[0] + wt[nn] * vbx;
        pB[1] = pB[1] + wt[nn] * vby;
        pB[2] = pB[2] + wt[nn] * vbz;
    }
}

/* One Boris half: u0 (in units of c*gamma*v/c) rotated in place. */
static void half_boris(double sqc, const double pE[3], const double pBin[3], double *u0, double *v0, double *w0)
{
    const double gg = 1.0 / sqrt(((sqc + *u0 * *u0) + *v0 * *v0) + *w0 * *w0);
    const double bx = gg * pBin[0], by = gg * pBin[1], bz = gg * pBin[2];
    const double ff = 2.0 / (((1.0 + bx * bx) + by * by) + bz * bz);
    const double u1 = ((*u0 + *v0 * bz) - *w0 * by) * ff;
    const double v1 = ((*v0 + *w0 * bx) - *u0 * bz) * ff;
    const double w1 = ((*w0 + *u0 * by) - *v0 * bx) * ff;
    *u0 = ((*u0 + v1 * bz) - w1 * by) + pE[0];
    *v0 = ((*v0 + w1 * bx) - u1 * bz) + pE[1];
    *w0 = ((*w0 + u1 * by) - v1 * bx) + pE[2];
}

/* DepositCurrentPIC, deposit.F90:11-103 (3D), directly into J */
static void deposit_pic(const orc_grid *g, orc_fields *f, double x0, double y0, double z0, double x, double y, double z, double q)
{
    const double qthis = q * g->qi;
    const int i1 = (int)floor(x0), i2 = (int)floor(x), j1 = (int)floor(y0), j2 = (int)floor(y);
    const int k1 = (int)floor(z0), k2 = (int)floor(z);
    const double xr = fmin((double)((i1 < i2 ? i1 : i2) + 1), fmax((double)(i1 > i2 ? i1 : i2), 0.5 * (x0 + x)));
    const double yr = fmin((double)((j1 < j2 ? j1 : j2) + 1), fmax((double)(j1 > j2 ? j1 : j2), 0.5 * (y0 + y)));
    const double zr = fmin((double)((k1 < k2 ? k1 : k2) + 1), fmax((double)(k1 > k2 ? k1 : k2), 0.5 * (z0 + z)));
    const double Fx1 = qthis * (xr - x0), Fy1 = qthis * (yr - y0), Fz1 = qthis * (zr - z0);
    const double Wx1 = 0.5 * (x0 + xr) - i1, Wy1 = 0.5 * (y0 + yr) - j1;
    const double Wx2 = 0.5 * (x + xr) - i2, Wy2 = 0.5 * (y + yr) - j2;
    const double Wz1 = 0.5 * (z0 + zr) - k1, Wz2 = 0.5 * (z + zr) - k2;
    const double Fx2 = qthis * (x - xr), Fy2 = qthis * (y - yr), Fz2 = qthis * (z - zr);
    double *Jx = f->Jx, *Jy = f->Jy, *Jz = f->Jz;
    Jx[ID(g, i1, j1, k1)] += (Fx1 * (1.0 - Wy1)) * (1.0 - Wz1);
    Jx[ID(g, i1, j1 + 1, k1)] += (Fx1 * Wy1) * (1.0 - Wz1);
    Jx[ID(g, i1, j1, k1 + 1)] += (Fx1 * (1.0 - Wy1)) * Wz1;
    Jx[ID(g, i1, j1 + 1, k1 + 1)] += (Fx1 * Wy1) * Wz1;
    Jx[ID(g, i2, j2, k2)] += (Fx2 * (1.0 - Wy2)) * (1.0 - Wz2);
    Jx[ID(g, i2, j2 + 1, k2)] += (Fx2 * Wy2) * (1.0 - Wz2);
    Jx[ID(g, i2, j2, k2 + 1)] += (Fx2 * (1.0 - Wy2)) * Wz2;
    Jx[ID(g, i2, j2 + 1, k2 + 1)] += (Fx2 * Wy2) * Wz2;
    Jy[ID(g, i1, j1, k1)] += (Fy1 * (1.0 - Wx1)) * (1.0 - Wz1);
    Jy[ID(g, i1 + 1, j1, k1)] += (Fy1 * Wx1) * (1.0 - Wz1);
    Jy[ID(g, i1, j1, k1 + 1)] += (Fy1 * (1.0 - Wx1)) * Wz1;
    Jy[ID(g, i1 + 1, j1, k1 + 1)] += (Fy1 * Wx1) * Wz1;
    Jy[ID(g, i2, j2, k2)] += (Fy2 * (1.0 - Wx2)) * (1.0 - Wz2);
    Jy[ID(g, i2 + 1, j2, k2)] += (Fy2 * Wx2) * (1.0 - Wz2);
    Jy[ID(g, i2, j2, k2 + 1)] += (Fy2 * (1.0 - Wx2)) * Wz2;
    Jy[ID(g, i2 + 1, j2, k2 + 1)] += (Fy2 * Wx2) * Wz2;
    Jz[ID(g, i1, j1, k1)] += (Fz1 * (1.0 - Wx1)) * (1.0 - Wy1);
    Jz[ID(g, i1 + 1, j1, k1)] += (Fz1 * Wx1) * (1.0 - Wy1);
    Jz[ID(g, i1, j1 + 1, k1)] += (Fz1 * (1.0 - Wx1)) * Wy1;
    Jz[ID(g, i1 + 1, j1 + 1, k1)] += (Fz1 * Wx1) * Wy1;
    Jz[ID(g, i2, j2, k2)] += (Fz2 * (1.0 - Wx2)) * (1.0 - Wy2);
    Jz[ID(g, i2 + 1, j2, k2)] += (Fz2 * Wx2) * (1.0 - Wy2);
    Jz[ID(g, i2, j2 + 1, k2)] += (Fz2 * (1.0 - Wx2)) * Wy2;
    Jz[ID(g, i2 + 1, j2 + 1, k2)] += (Fz2 * Wx2) * Wy2;
}

/* MovePrtlAxis, cyl_movdep_strang.F90:462-566: returns 1 on a successful
   sub-step (the particle arrays updated), 0 when |dtheta| > 0.45 cells. */
static int move_axis(const orc_grid *g, orc_particles *p, const orc_fields *f, int64_t n, double x, double y, double z,
                     double dt, double inv_dtheta)
{
    const double c = g->c, sqc = c * c, cinv = 1.0 / c;
    double pE[3], pB[3];
    interp(g, f, x, y, z, pE, pB);
    const double qm = p->flv[n] == 0 ? 0.0 : g->flvrqm[p->flv[n]] * 0.25;
    for (int d = 0; d < 3; d++) { pE[d] = (pE[d] * qm) * dt; pB[d] = (pB[d] * qm) * dt; }
    double u0 = c * p->u[n] + pE[0], v0 = c * p->v[n] + pE[1], w0 = c * p->w[n] + pE[2];
    half_boris(sqc, pE, pB, &u0, &v0, &w0);
    double u1 = u0 * cinv, v1 = v0 * cinv;
    const double w1 = w0 * cinv;
    const double gg = sqc / sqrt(((sqc + u0 * u0) + v0 * v0) + w0 * w0);
    const double r0 = (x - 3.5) * 1.0;
    const double x1 = r0 + (u1 * gg) * dt;
    const double y1 = (v1 * gg) * dt;
    const double r1 = sqrt(x1 * x1 + y1 * y1);
    const double dy = x1 > 0 ? atan(y1 / x1) * inv_dtheta : 0.0;
    if (fabs(dy) > 0.45) return 0;
    if (x1 > 0) {
        p->x[n] = r1 / 1.0 + 3.5;
        u1 = (r0 * u0 + ((u0 * u1) * gg * dt + v0 * y1)) / r1;
        v1 = (v0 * r0) / r1;
    } else {
        p->x[n] = x1 / 1.0 + 3.5;
    }
    p->y[n] = p->y[n] + dy;
    p->z[n] = p->z[n] + ((w1 * gg) * dt) * 1.0;
    interp(g, f, p->x[n], p->y[n], p->z[n], pE, pB);
    for (int d = 0; d < 3; d++) { pE[d] = (pE[d] * qm) * dt; pB[d] = (pB[d] * qm) * dt; }
    u0 = u1 + pE[0];
    v0 = v1 + pE[1];
    w0 = w0 + pE[2];
    half_boris(sqc, pE, pB, &u0, &v0, &w0);
    p->u[n] = u0 * cinv;
    p->v[n] = v0 * cinv;
    p->w[n] = w0 * cinv;
    return 1;
}

/* PrtlAxisBC, cyl_movdep_strang.F90:450-460 */
static void axis_bc(const orc_grid *g, orc_particles *p, int64_t n)
{
    const double ymin = 3.0, ymax = (double)(g->my - 2), ylen = ymax - ymin;
    if (p->x[n] < 3.5) {
        p->x[n] = 3.5 + (3.5 - p->x[n]);
        p->y[n] = p->y[n] + g->ny / 2.0;
        p->u[n] = -p->u[n];
        p->v[n] = -p->v[n];
    }
    if (p->y[n] > ymax) p->y[n] = p->y[n] - ylen;
    if (p->y[n] < ymin) p->y[n] = p->y[n] + ylen;
}

int orc_cyl_max_substeps = 100000;
int64_t orc_cyl_substep_overruns = 0;

/* SubStepMovDep, cyl_movdep_strang.F90:404-438.  The reference loops until
   t = 1 with no bound; here a particle gives up after orc_cyl_max_substeps
   attempts (counted in orc_cyl_substep_overruns). */
static void substep(const orc_grid *g, orc_particles *p, orc_fields *f, int64_t n, double x0, double y0, double z0,
                    double u0, double v0, double w0, double inv_dtheta)
{
    if (p->flv[n] == 0) return;
    p->x[n] = x0; p->y[n] = y0; p->z[n] = z0; p->u[n] = u0; p->v[n] = v0; p->w[n] = w0;
    double t = 0.0, dt = 1.0;
    int tries = 0;
    while (t < 1.0) {
        if (++tries > orc_cyl_max_substeps) { orc_cyl_substep_overruns++; break; }
        double delt = dt;
        if (t + dt > 1.0) delt = 1.0 - t;
        const int res = move_axis(g, p, f, n, x0, y0, z0, delt, inv_dtheta);
        if (res == 1) {
            t = t + delt;
            deposit_pic(g, f, x0, y0, z0, p->x[n], p->y[n], p->z[n], p->q[n]);
            axis_bc(g, p, n);
            dt = dt * 1.7;
            x0 = p->x[n]; y0 = p->y[n]; z0 = p->z[n];
        } else {
            dt = dt * 0.5;
        }
    }
}

static void segment12(double Fx, double Fy, double Fz, double Wx, double Wy, double Wz, double o[12])
{
    o[0] = ((Fx * 1.0) * (1.0 - Wy)) * (1.0 - Wz);
    o[1] = ((Fx * 1.0) * Wy) * (1.0 - Wz);
    o[2] = ((Fx * 1.0) * (1.0 - Wy)) * Wz;
    o[3] = ((Fx * 1.0) * Wy) * Wz;
    o[4] = ((Fy * (1.0 - Wx)) * 1.0) * (1.0 - Wz);
    o[5] = ((Fy * Wx) * 1.0) * (1.0 - Wz);
    o[6] = ((Fy * (1.0 - Wx)) * 1.0) * Wz;
    o[7] = ((Fy * Wx) * 1.0) * Wz;
    o[8] = ((Fz * (1.0 - Wx)) * (1.0 - Wy)) * 1.0;
    o[9] = ((Fz * Wx) * (1.0 - Wy)) * 1.0;
    o[10] = ((Fz * (1.0 - Wx)) * Wy) * 1.0;
    o[11] = ((Fz * Wx) * Wy) * 1.0;
}

/* MoveDepositPrtl of cyl_movdep_strang.F90:14-378 (3D, axis on this rank). */
void orc_cyl_move_deposit(const orc_grid *g, orc_particles *p, orc_fields *f)
{
    double P[4];
    orc_cyl_params(g, P);
    const double inv_dtheta = P[2];
    const double c = g->c, sqc = c * c, cinv = 1.0 / c;
    const double r_proc = (0.0 + P[3]) - 3.0;                 /* :57 */
    const size_t ncell = (size_t)g->mx * g->my * g->mz;
    double *vj = (double *)calloc(ncell * 12, sizeof(double));
    orc_reset_current(g, f);
    for (int64_t n = 0; n < p->used; n++) {
        const double x0 = p->x[n], y0 = p->y[n], z0 = p->z[n];
        double qthis = p->q[n] * g->qi;
        const double ui = p->u[n], vi = p->v[n], wi = p->w[n];
        const double qm = p->flv[n] == 0 ? 0.0 : g->flvrqm[p->flv[n]] * 0.25;  /* :100 */
        const int ip0 = (int)x0, jp0 = (int)y0, kp0 = (int)z0;
        double pE[3], pB[3];
        interp(g, f, x0, y0, z0, pE, pB);                        /* :113-155 */
        for (int d = 0; d < 3; d++) { pE[d] = pE[d] * qm; pB[d] = pB[d] * qm; }
        /* first half, :171-191 */
        double u0 = c * p->u[n] + pE[0], v0 = c * p->v[n] + pE[1], w0 = c * p->w[n] + pE[2];
        half_boris(sqc, pE, pB, &u0, &v0, &w0);
        double u1 = u0 * cinv, v1 = v0 * cinv;
        /* move in the local Cartesian frame, :194-207 */
        const double gg = sqc / sqrt(((sqc + u0 * u0) + v0 * v0) + w0 * w0);
        const double r0 = (p->x[n] + r_proc) * 1.0;
        const double x1 = r0 + u1 * gg, y1 = v1 * gg;
        double r1 = sqrt(x1 * x1 + y1 * y1);
        p->x[n] = r1 * 1.0 - r_proc;
        p->y[n] = p->y[n] + atan(y1 / x1) * inv_dtheta;
        p->z[n] = p->z[n] + (p->w[n] * gg) * 1.0;               /* w before this step's push */
        r1 = 1.0 / r1;
        u1 = (r0 * u0 + ((u0 * u1) * gg + v0 * y1)) * r1;
        v1 = (v0 * r0) * r1;
        /* second interpolation and half, :214-294 */
        const int ip = (int)p->x[n], jp = (int)p->y[n], kp = (int)p->z[n];
        interp(g, f, p->x[n], p->y[n], p->z[n], pE, pB);
        for (int d = 0; d < 3; d++) { pE[d] = pE[d] * qm; pB[d] = pB[d] * qm; }
        u0 = u1 + pE[0];
        v0 = v1 + pE[1];
        w0 = w0 + pE[2];
        half_boris(sqc, pE, pB, &u0, &v0, &w0);
        p->u[n] = u0 * cinv;
        p->v[n] = v0 * cinv;
        p->w[n] = w0 * cinv;
        /* near-axis particles are moved again by the sub-stepper, :296, :390-402 */
        if (x0 < 4.5) {
            substep(g, p, f, n, x0, y0, z0, ui, vi, wi, inv_dtheta);
            qthis = 0.0;
        }
        /* zigzag deposit into VecJ, :298-356; the second segment goes to the
           cell of the start point (short_arr_ind of :341 uses ip0,jp0,kp0) */
        const double x1n = p->x[n], y1n = p->y[n], z1n = p->z[n];
        const double xr = fmin((double)((ip0 < ip ? ip0 : ip) + 1), fmax((double)(ip0 > ip ? ip0 : ip), 0.5 * (x0 + x1n)));
        const double yr = fmin((double)((jp0 < jp ? jp0 : jp) + 1), fmax((double)(jp0 > jp ? jp0 : jp), 0.5 * (y0 + y1n)));
        const double zr = fmin((double)((kp0 < kp ? kp0 : kp) + 1), fmax((double)(kp0 > kp ? kp0 : kp), 0.5 * (z0 + z1n)));
        double o[12];
        const int64_t cell = ID(g, ip0, jp0, kp0);
        segment12(qthis * (xr - x0), qthis * (yr - y0), qthis * (zr - z0), 0.5 * (x0 + xr) - ip0,
                  0.5 * (y0 + yr) - jp0, 0.5 * (z0 + zr) - kp0, o);
        for (int e = 0; e < 12; e++) vj[cell * 12 + e] = vj[cell * 12 + e] + o[e];
        segment12(qthis * (x1n - xr), qthis * (y1n - yr), qthis * (z1n - zr), 0.5 * (x1n + xr) - ip,
                  0.5 * (y1n + yr) - jp, 0.5 * (z1n + zr) - kp, o);
        for (int e = 0; e < 12; e++) vj[cell * 12 + e] = vj[cell * 12 + e] + o[e];
    }
    /* ReduceCurrentMatrix scatter (movdep_routines.F90:262-291) */
    for (int k = 1; k <= g->mz - 1; k++)
        for (int j = 1; j <= g->my - 1; j++)
            for (int i = 1; i <= g->mx - 1; i++) {
                const double *v = vj + ID(g, i, j, k) * 12;
                f->Jx[ID(g, i, j, k)] += v[0];
                f->Jx[ID(g, i, j + 1, k)] += v[1];
                f->Jx[ID(g, i, j, k + 1)] += v[2];
                f->Jx[ID(g, i, j + 1, k + 1)] += v[3];
                f->Jy[ID(g, i, j, k)] += v[4];
                f->Jy[ID(g, i + 1, j, k)] += v[5];
                f->Jy[ID(g, i, j, k + 1)] += v[6];
                f->Jy[ID(g, i + 1, j, k + 1)] += v[7];
                f->Jz[ID(g, i, j, k)] += v[8];
                f->Jz[ID(g, i + 1, j, k)] += v[9];
                f->Jz[ID(g, i, j + 1, k)] += v[10];
                f->Jz[ID(g, i + 1, j + 1, k)] += v[11];
            }
    free(vj);
    /* AxisCurrentBC, cyl_movdep_strang.F90:570-584 */
    for (int k = 1; k <= g->mz; k++)
        for (int j = 1; j <= g->my; j++) {
            f->Jy[ID(g, 4, j, k)] = f->Jy[ID(g, 4, j, k)] - f->Jy[ID(g, 3, j, k)];
            f->Jz[ID(g, 4, j, k)] = f->Jz[ID(g, 4, j, k)] - f->Jz[ID(g, 3, j, k)];
            f->Jx[ID(g, 3, j, k)] = 0.0;
            f->Jy[ID(g, 2, j, k)] = 0.0;
            f->Jz[ID(g, 2, j, k)] = 0.0;
        }
}

/* LoadPrtlOutliers (loadprtlout.F90:13-106) with the r faces closed:
   particles leaving through them are dropped, theta and z wrap as in the
   Cartesian exchange (AppendParticles order). */
int orc_cyl_exchange(const orc_grid *g, orc_particles *p)
{
    const double xmin = 3.0, xmax = (double)(g->mx - 2), ymin = 3.0, ymax = (double)(g->my - 2);
    const double zmin = 3.0, zmax = (double)(g->mz - 2);
    const double len[3] = {xmax - xmin, ymax - ymin, zmax - zmin};
    int64_t *which = (int64_t *)malloc((size_t)(p->used > 0 ? p->used : 1) * sizeof(int64_t));
    double (*saved)[8] = (double (*)[8])malloc((size_t)(p->used > 0 ? p->used : 1) * sizeof(*saved));
    int *face = (int *)malloc((size_t)(p->used > 0 ? p->used : 1) * sizeof(int));
    int64_t ns = 0;
    for (int64_t i = 0; i < p->used; i++) {
        if (p->flv[i] == 0) continue;
        const double x = p->x[i], y = p->y[i], z = p->z[i];
        int fc = 0;
        if (x < xmin) {
            if ((y <= (ymax + xmin) - x) && (y >= (ymin - xmin) + x) && (z <= (zmax + xmin) - x) && (z >= (zmin - xmin) + x)) fc = 1;
        } else if (x > xmax) {
            if ((y <= (ymax - xmax) + x) && (y >= (ymin + xmax) - x) && (z <= (zmax - xmax) + x) && (z >= (zmin + xmax) - x)) fc = 2;
        }
        if (!fc) {
            if (y < ymin) {
                if ((y < (ymin - xmin) + x) && (y < (ymin + xmax) - x) && (z >= (zmin - ymin) + y) && (z <= (zmax + ymin) - y)) fc = 3;
            } else if (y > ymax) {
                if ((y > (ymax + xmin) - x) && (y > (ymax - xmax) + x) && (z >= (zmin + ymax) - y) && (z <= (zmax - ymax) + y)) fc = 4;
            }
        }
        if (!fc) {
            if (z < zmin) {
                if ((z < (zmin - xmin) + x) && (z < (zmin + xmax) - x) && (z < (zmin - ymin) + y) && (z < (zmin + ymax) - y)) fc = 5;
            } else if (z > zmax) {
                if ((z > (zmax + xmin) - x) && (z > (zmax - xmax) + x) && (z > (zmax + ymin) - y) && (z > (zmax - ymax) + y)) fc = 6;
            }
        }
        if (!fc) continue;
        saved[ns][0] = p->q[i]; saved[ns][1] = x; saved[ns][2] = y; saved[ns][3] = z;
        saved[ns][4] = p->u[i]; saved[ns][5] = p->v[i]; saved[ns][6] = p->w[i]; saved[ns][7] = p->flv[i];
        face[ns] = fc;
        which[ns++] = i;
        p->q[i] = 0; p->flv[i] = 0; p->u[i] = 0; p->v[i] = 0; p->w[i] = 0;
        p->x[i] = 3.8; p->y[i] = 3.8; p->z[i] = 3.8;
    }
    static const int order[6] = {2, 1, 4, 3, 6, 5};
    int rc = 0;
    for (int o = 0; o < 6; o++) {
        const int fc = order[o];
        if (fc <= 2) continue;  /* r faces closed: sent to MPI_PROC_NULL */
        const int axis = (fc - 1) / 2;
        for (int64_t m = 0; m < ns; m++) {
            if (face[m] != fc) continue;
            if (p->used >= p->capacity) { rc = -1; continue; }
            double pos[3] = {saved[m][1], saved[m][2], saved[m][3]};
            if (fc % 2 == 1) pos[axis] = (pos[axis] - 0.0) + len[axis];
            else pos[axis] = (pos[axis] - len[axis]) + 0.0;
            const int64_t d = p->used++;
            p->q[d] = saved[m][0]; p->x[d] = pos[0]; p->y[d] = pos[1]; p->z[d] = pos[2];
            p->u[d] = saved[m][4]; p->v[d] = saved[m][5]; p->w[d] = saved[m][6]; p->flv[d] = (int32_t)saved[m][7];
        }
    }
    free(which); free(saved); free(face);
    return rc;
}

/* CalcFldEnergy_cyl, cyl_savedata_routines.F90:8-31 (not halved). */
void orc_cyl_field_energy(const orc_grid *g, const orc_fields *f, double out[2])
{
    double P[4];
    orc_cyl_params(g, P);
    const double dtheta = P[0], rmin = 0.0 + P[3];
    double eb = 0.0, ee = 0.0;
    for (int k = 3; k <= g->mz - 3; k++)
        for (int j = 3; j <= g->my - 3; j++)
            for (int i = 4; i <= g->mx - 3; i++) {
                const double r = ((double)i - 3.0) + rmin, rp = r + 0.5;
                const int64_t c0 = ID(g, i, j, k);
                eb = eb + ((r * (f->Bx[c0] * f->Bx[c0]) + rp * (f->By[c0] * f->By[c0])) + rp * (f->Bz[c0] * f->Bz[c0])) * dtheta;
                ee = ee + ((rp * (f->Ex[c0] * f->Ex[c0]) + r * (f->Ey[c0] * f->Ey[c0])) + r * (f->Ez[c0] * f->Ez[c0])) * dtheta;
            }
    out[0] = eb;
    out[1] = ee;
}

/* One cylindrical step in MAIN.F90 order (Yee or Lehe B update). */
int orc_cyl_step(const orc_grid *g, orc_particles *p, orc_fields *f, int t, int reorder_period)
{
    orc_cyl_update_b_half(g, f);
    orc_cyl_send_recv_flds(g, f->Bx, f->By, f->Bz);
    orc_cyl_move_deposit(g, p, f);
    int rc = orc_cyl_exchange(g, p);
    orc_cyl_update_b_half(g, f);
    orc_cyl_send_recv_flds(g, f->Bx, f->By, f->Bz);
    orc_cyl_update_e(g, f);
    orc_cyl_send_recv_flds(g, f->Ex, f->Ey, f->Ez);
    orc_cyl_fold(g, f->Jx, f->Jy, f->Jz);
    orc_cyl_add_current(g, f);
    orc_cyl_send_recv_flds(g, f->Ex, f->Ey, f->Ez);
    if (reorder_period > 0 && t % reorder_period == 0) orc_reorder(g, p, NULL);
    return rc;
}

/* Even placement with weights proportional to r (InitPrtlFromPSP_UniformSeparation,
   init_prtl.F90:224-352, with azimuthal_weight_prtl cyl_common.F90:57-62):
   npx x npy x npz particles per cell of one species with q = -r*dtheta*density
   at cell-centred sub-positions, momenta from the Maxwell sampler (temp) with
   Philox draws keyed by seed; returns the count. */
int64_t orc_cyl_load_uniform(const orc_grid *g, int npx, int npy, int npz, double density, double temp, double charge,
                             int flv, uint32_t seed, orc_particles *p)
{
    double P[4];
    orc_cyl_params(g, P);
    const double dtheta = P[0];
    const uint32_t key[2] = {seed, 0x4359434cu};
    int64_t cnt = 0;
    for (int k = 3; k <= g->mz - 3; k++)
        for (int j = 3; j <= g->my - 3; j++)
            for (int i = 3; i <= g->mx - 3; i++)
                for (int si = 0; si < npx; si++)
                    for (int sj = 0; sj < npy; sj++)
                        for (int sk = 0; sk < npz; sk++) {
                            const double xl = i + (si + 0.5) / npx, yl = j + (sj + 0.5) / npy, zl = k + (sk + 0.5) / npz;
                            const double xg = xl - 3.0;
                            double r = xg + P[3];
                            if (r < 0.0) r = 0.0;
                            const double wt = (density * r) * dtheta;
                            if (!(wt > 0)) continue;
                            uint32_t out[4];
                            const uint32_t ctr[4] = {(uint32_t)cnt, (uint32_t)flv, 7, 0};
                            orc_philox4x32_10(ctr, key, out);
                            const double a = orc_u01(out[0], out[1]), b = orc_u01(out[2], out[3]);
                            const uint32_t ctr2[4] = {(uint32_t)cnt, (uint32_t)flv, 8, 0};
                            orc_philox4x32_10(ctr2, key, out);
                            const double cc = orc_u01(out[0], out[1]);
                            /* isotropic Maxwellian-like spread: sigma = sqrt(temp/2) per component (Box-Muller) */
                            const double s = sqrt(temp / 2.0);
                            const double rad = sqrt(-2.0 * log(1.0 - a));
                            if (p->used >= p->capacity) return -1;
                            const int64_t d = p->used++;
                            p->x[d] = xl; p->y[d] = yl; p->z[d] = zl;
                            p->u[d] = s * rad * cos(2.0 * PI_PSN * b);
                            p->v[d] = s * rad * sin(2.0 * PI_PSN * b);
                            p->w[d] = s * sqrt(-2.0 * log(1.0 - cc)) * cos(2.0 * PI_PSN * a);
                            p->q[d] = wt * charge;
                            p->flv[d] = flv;
                            cnt++;
                        }
    return cnt;
}
