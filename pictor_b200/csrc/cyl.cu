// cyl.cu -- the cylindrical (r, theta, z) step in the reference's FP64 form.
//
// Reference: src/cyl/cyl_common.F90:19-32 (dtheta = 2 pi/ny, ax_perm_area =
// 4/ny, rshift = -0.5), cyl_em_update.F90 (Yee with 1/r metrics, axis
// treatment), cyl_em_update_lehe.F90 (Lehe, restated with its syntax fixed),
// cyl_movdep_strang.F90 (Strang-split mover with a local Cartesian move,
// adaptive near-axis sub-stepping, AxisCurrentBC), deposit.F90 (the scalar
// deposit the sub-stepper uses).
//
// Set-up: the rank holds the axis (x = 3.5 is r = 0); theta (y) and z are
// periodic, r is not (no halo or fold across the r faces, particles leaving at
// r_max are dropped).  With the axis included the reference exchanges the y
// faces before the z faces (indepLBaxis = 2), with the y faces over all x and
// the interior z only.  Every kernel keeps the reference's loop ranges and
// operation order; the file is compiled without FMA contraction, so fields,
// momenta and positions equal the serial CPU build bit for bit.
#include "common.cuh"
#include "kernels.cuh"
#include "tile64.cuh"
#include "particle_math.cuh"
#include "tile.cuh"

namespace pic {

struct CylP {
    double dtheta, ax_perm_area, inv_dtheta, rmin;
};

template <typename T>
__device__ __forceinline__ T ldd(const T *p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// Fields
// ---------------------------------------------------------------------------

// Lehe directional differences of cyl_em_update_lehe.F90:255-289.
template <typename T>
__device__ __forceinline__ T lgx(const GridP &g, const T *F, long long c0)
{
    T r = (T)g.lehe[0] * (ldd(F + c0 + 1) - ldd(F + c0));
    r = r + (T)g.lehe[4] * (ldd(F + c0 + 1 + g.sz) - ldd(F + c0 + g.sz));
    r = r + (T)g.lehe[4] * (ldd(F + c0 + 1 - g.sz) - ldd(F + c0 - g.sz));
    return r;
}
template <typename T>
__device__ __forceinline__ T lgx1(const GridP &g, const T *F, long long c0, T rp, T rr)
{
    T r = (T)g.lehe[0] * (rp * ldd(F + c0 + 1) - rr * ldd(F + c0));
    r = r + (T)g.lehe[4] * (rp * ldd(F + c0 + 1 + g.sz) - rr * ldd(F + c0 + g.sz));
    r = r + (T)g.lehe[4] * (rp * ldd(F + c0 + 1 - g.sz) - rr * ldd(F + c0 - g.sz));
    return r;
}
template <typename T>
__device__ __forceinline__ T lgy(const GridP &g, const T *F, long long c0)
{
    T r = (T)(g.lehe[1] * 1.0) * (ldd(F + c0 + g.sy) - ldd(F + c0));
    r = r + (T)(g.lehe[6] * 1.0) * (ldd(F + c0 + g.sy + g.sz) - ldd(F + c0 + g.sz));
    r = r + (T)(g.lehe[6] * 1.0) * (ldd(F + c0 + g.sy - g.sz) - ldd(F + c0 - g.sz));
    return r;
}
template <typename T>
__device__ __forceinline__ T lgz(const GridP &g, const T *F, long long c0)
{
    const long long sy = g.sy, sz = g.sz;
    T r = (T)g.lehe[2] * (ldd(F + c0 + sz) - ldd(F + c0));
    r = r + (T)g.lehe[7] * (ldd(F + c0 + 1 + sz) - ldd(F + c0 + 1));
    r = r + (T)g.lehe[7] * (ldd(F + c0 - 1 + sz) - ldd(F + c0 - 1));
    r = r + (T)g.lehe[8] * (ldd(F + c0 + sy + sz) - ldd(F + c0 + sy));
    r = r + (T)g.lehe[8] * (ldd(F + c0 - sy + sz) - ldd(F + c0 - sy));
    r = r + (T)g.lehe[11] * (ldd(F + c0 + 2 * sz) - ldd(F + c0 - sz));
    return r;
}

// UpdateBfieldHalf main loop (cyl_em_update.F90:66-83): i 4..mx-1, j 1..my-1,
// k 1..mz-1 (Lehe: k 2..mz-2, see the oracle for why).  T = double is the
// reference form; T = float the FP32 form (same expressions).
// Each thread walks kCylZChunk consecutive k of its (i, j) column, so the
// planes its stencil reads above and below were loaded by its CTA one step
// earlier and come from L1 rather than L2.
constexpr int kCylZChunk = 16;

// i from 4 on the rank holding the axis (its cells 3 take the axis
// updates), from 1 elsewhere (cyl_em_update.F90:49-51).
template <typename T, int FDTD>
__global__ void k_cyl_bhalf(GridP g, CylP cp, const T *__restrict__ Ex, const T *__restrict__ Ey,
                            const T *__restrict__ Ez, T *Bx, T *By, T *Bz)
{
    const int i = (g.inc_axis ? 4 : 1) + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
    if (i > g.mx - 1 || j > g.my - 1) return;
    const int k0 = (FDTD == PIC_FDTD_LEHE ? 2 : 1) + blockIdx.z * kCylZChunk;
    const int k1 = min(k0 + kCylZChunk - 1, FDTD == PIC_FDTD_LEHE ? g.mz - 2 : g.mz - 1);
    const T h = (T)g.h, dtheta = (T)cp.dtheta;
    const T r = (((T)i - (T)3.0) + (T)cp.rmin) * (T)1.0;
    const T rp_half = r + (T)0.5 * (T)1.0, rp = r + (T)1.0;
    const long long sy = g.sy, sz = g.sz;
    for (int k = k0; k <= k1; k++) {
        const long long c0 = cidx(g, i, j, k);
        if (FDTD == PIC_FDTD_YEE) {
            Bx[c0] = (Bx[c0] - (h * (ldd(Ez + c0 + sy) - ldd(Ez + c0))) / (r * dtheta)) + (h * (T)1.0) * (ldd(Ey + c0 + sz) - ldd(Ey + c0));
            By[c0] = (By[c0] - (h * (T)1.0) * (ldd(Ex + c0 + sz) - ldd(Ex + c0))) + (h * (T)1.0) * (ldd(Ez + c0 + 1) - ldd(Ez + c0));
            Bz[c0] = Bz[c0] - (h * (((T)1.0 * (rp * ldd(Ey + c0 + 1) - r * ldd(Ey + c0))) - (ldd(Ex + c0 + sy) - ldd(Ex + c0)) / dtheta)) / rp_half;
        } else {
            Bx[c0] = (Bx[c0] - (h * lgy(g, Ez, c0)) / (r * dtheta)) + (h * (T)1.0) * lgz(g, Ey, c0);
            By[c0] = (By[c0] - (h * (T)1.0) * lgz(g, Ex, c0)) + (h * (T)1.0) * lgx(g, Ez, c0);
            Bz[c0] = Bz[c0] - (h * (((T)1.0 * lgx1(g, Ey, c0, rp, r)) - lgy(g, Ex, c0) / dtheta)) / rp_half;
        }
    }
}

// UpdateBzAxis (cyl_em_update.F90:231-246) + Bz(3,j,k) = Bz_ax(k): one
// thread per k sums Ey(4,j,k) over j in the reference's order.
template <typename T>
__global__ void k_cyl_bz_axis(GridP g, CylP cp, const T *__restrict__ Ey, T *Bz)
{
    const int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (k > g.mz - 1) return;
    const T hax = (T)(g.h * cp.ax_perm_area);
    T s = (T)0.0;
    for (int j = 3; j <= g.my - 3; j++) s = s - hax * Ey[cidx(g, 4, j, k)];
    const T v = Bz[cidx(g, 3, 3, k)] + s;
    for (int j = 1; j <= g.my - 1; j++) Bz[cidx(g, 3, j, k)] = v;
}

__device__ __forceinline__ int axis_partner(const GridP &g, int j)
{
    int p = j + g.ny / 2;
    if (p > g.my - 3) p -= g.ny;
    return p;
}

// UpdateBFldAxis (cyl_em_update.F90:187-227), all j, k.
template <typename T>
__global__ void k_cyl_b_axis(GridP g, T *Bx, T *By, T *Bz)
{
    const int j = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 1 + blockIdx.y;
    if (j > g.my) return;
    const int jpp = axis_partner(g, j);
    By[cidx(g, 3, j, k)] = (T)0.5 * (By[cidx(g, 4, j, k)] - By[cidx(g, 4, jpp, k)]);
    By[cidx(g, 2, j, k)] = -By[cidx(g, 4, jpp, k)];
    Bx[cidx(g, 3, j, k)] = -Bx[cidx(g, 4, jpp, k)];
    Bz[cidx(g, 2, j, k)] = Bz[cidx(g, 4, jpp, k)];
}

// UpdateEFldAxis (cyl_em_update.F90:143-185), all j, k.
template <typename T>
__global__ void k_cyl_e_axis(GridP g, T *Ex, T *Ey, T *Ez)
{
    const int j = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 1 + blockIdx.y;
    if (j > g.my) return;
    const int jpp = axis_partner(g, j);
    Ex[cidx(g, 3, j, k)] = (T)0.5 * (Ex[cidx(g, 4, j, k)] - Ex[cidx(g, 4, jpp, k)]);
    Ex[cidx(g, 2, j, k)] = -Ex[cidx(g, 4, jpp, k)];
    Ey[cidx(g, 3, j, k)] = -Ey[cidx(g, 4, jpp, k)];
    Ez[cidx(g, 3, j, k)] = Ez[cidx(g, 4, jpp, k)];
}

// UpdateEfield (MODE 0, cyl_em_update.F90:24-41) or AddCurrent (MODE 2,
// :128-137): i 4..mx-3 on the rank holding the axis, 3..mx-3 elsewhere;
// j, k 3..m-3.
template <typename T, int MODE>
__global__ void k_cyl_e(GridP g, CylP cp, T *Ex, T *Ey, T *Ez, const T *__restrict__ Bx, const T *__restrict__ By,
                        const T *__restrict__ Bz, const T *__restrict__ Jx, const T *__restrict__ Jy,
                        const T *__restrict__ Jz)
{
    const int i = (g.inc_axis ? 4 : 3) + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 3 + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = 3 + blockIdx.z;
    if (i > g.mx - 3 || j > g.my - 3) return;
    const T dtheta = (T)cp.dtheta;
    const T r = (((T)i - (T)3.0) + (T)cp.rmin) * (T)1.0;
    const T rp_half = r + (T)0.5 * (T)1.0, rm_half = r - (T)0.5 * (T)1.0;
    const long long c0 = cidx(g, i, j, k);
    if (MODE == 0) {
        const T fc = (T)g.fc;
        Ex[c0] = (Ex[c0] + (fc * (ldd(Bz + c0) - ldd(Bz + c0 - g.sy))) / (rp_half * dtheta)) - (fc * (T)1.0) * (ldd(By + c0) - ldd(By + c0 - g.sz));
        Ey[c0] = (Ey[c0] + (fc * (T)1.0) * (ldd(Bx + c0) - ldd(Bx + c0 - g.sz))) - (fc * (T)1.0) * (ldd(Bz + c0) - ldd(Bz + c0 - 1));
        Ez[c0] = (Ez[c0] + ((fc * (T)1.0) * (rp_half * ldd(By + c0) - rm_half * ldd(By + c0 - 1))) / r) - (fc * (ldd(Bx + c0) - ldd(Bx + c0 - g.sy))) / (r * dtheta);
    } else {
        Ex[c0] = Ex[c0] - (ldd(Jx + c0) * (T)1.0) / (rp_half * dtheta);
        Ey[c0] = Ey[c0] - (ldd(Jy + c0) * (T)1.0) * (T)1.0;
        Ez[c0] = Ez[c0] - (ldd(Jz + c0) * (T)1.0) / (r * dtheta);
    }
}

// Halo along y over x 1..mx and z 3..mz-3, then along z over all x, y.
template <typename T>
__global__ void k_cyl_halo_y(GridP g, T *F)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 3 + blockIdx.y;
    if (i > g.mx) return;
    const int m = g.my;
    for (int l = 0; l < 3; l++) F[cidx(g, i, m - 2 + l, k)] = F[cidx(g, i, 3 + l, k)];
    for (int l = 0; l < 2; l++) F[cidx(g, i, 1 + l, k)] = F[cidx(g, i, m - 4 + l, k)];
}
template <typename T>
__global__ void k_cyl_halo_z(GridP g, T *F)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    if (i > g.mx) return;
    const int m = g.mz;
    for (int l = 0; l < 3; l++) F[cidx(g, i, j, m - 2 + l)] = F[cidx(g, i, j, 3 + l)];
    for (int l = 0; l < 2; l++) F[cidx(g, i, j, 1 + l)] = F[cidx(g, i, j, m - 4 + l)];
}

// Current fold: z faces over all x, y, then y faces over x 1..mx, z 3..mz-3.
template <typename T>
__global__ void k_cyl_fold_z(GridP g, T *F)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = 1 + blockIdx.y;
    if (i > g.mx) return;
    const int m = g.mz;
    T hi3[3], lo2[2];
    for (int l = 0; l < 3; l++) hi3[l] = F[cidx(g, i, j, m - 2 + l)];
    for (int l = 0; l < 2; l++) lo2[l] = F[cidx(g, i, j, 1 + l)];
    for (int l = 0; l < 3; l++) F[cidx(g, i, j, 3 + l)] = F[cidx(g, i, j, 3 + l)] + hi3[l];
    for (int l = 0; l < 2; l++) F[cidx(g, i, j, m - 4 + l)] = F[cidx(g, i, j, m - 4 + l)] + lo2[l];
}
template <typename T>
__global__ void k_cyl_fold_y(GridP g, T *F)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 3 + blockIdx.y;
    if (i > g.mx) return;
    const int m = g.my;
    T hi3[3], lo2[2];
    for (int l = 0; l < 3; l++) hi3[l] = F[cidx(g, i, m - 2 + l, k)];
    for (int l = 0; l < 2; l++) lo2[l] = F[cidx(g, i, 1 + l, k)];
    for (int l = 0; l < 3; l++) F[cidx(g, i, 3 + l, k)] = F[cidx(g, i, 3 + l, k)] + hi3[l];
    for (int l = 0; l < 2; l++) F[cidx(g, i, m - 4 + l, k)] = F[cidx(g, i, m - 4 + l, k)] + lo2[l];
}

static CylP cyl_params(const GridP &g)
{
    CylP c;
    const double pi = 3.14159265358979323846264;
    c.dtheta = 2.0 * pi / g.ny;
    c.ax_perm_area = 4.0 / g.ny;
    c.inv_dtheta = 1.0 / c.dtheta;
    c.rmin = g.rmin;  // xborders(procxind) + rshift: -0.5 on the rank holding the axis
    return c;
}

template <typename T>
static void halo(const GridP &g, T *const F[3], cudaStream_t s)
{
    for (int c = 0; c < 3; c++) {
        k_cyl_halo_y<T><<<dim3((g.mx + 127) / 128, g.mz - 5), 128, 0, s>>>(g, F[c]);
        k_cyl_halo_z<T><<<dim3((g.mx + 127) / 128, g.my), 128, 0, s>>>(g, F[c]);
    }
    count_launches(6);
}

template <typename T>
void launch_cyl_bhalf(const GridP &g, T *const E[3], T *const B[3], cudaStream_t s)
{
    const CylP cp = cyl_params(g);
    const int nk = g.fdtd == PIC_FDTD_LEHE ? g.mz - 3 : g.mz - 1;
    const int ni = g.mx - (g.inc_axis ? 4 : 1);   // i .. mx-1
    const dim3 grid((ni + 31) / 32, (g.my - 1 + 3) / 4, (nk + kCylZChunk - 1) / kCylZChunk), block(32, 4, 1);
    if (g.fdtd == PIC_FDTD_LEHE)
        k_cyl_bhalf<T, PIC_FDTD_LEHE><<<grid, block, 0, s>>>(g, cp, E[0], E[1], E[2], B[0], B[1], B[2]);
    else
        k_cyl_bhalf<T, PIC_FDTD_YEE><<<grid, block, 0, s>>>(g, cp, E[0], E[1], E[2], B[0], B[1], B[2]);
    count_launches(1);
    if (g.inc_axis) {   // cyl_em_update.F90:85-105
        k_cyl_bz_axis<T><<<(g.mz + 127) / 128, 128, 0, s>>>(g, cp, E[1], B[2]);
        k_cyl_b_axis<T><<<dim3((g.my + 127) / 128, g.mz), 128, 0, s>>>(g, B[0], B[1], B[2]);
        count_launches(2);
    }
    halo<T>(g, B, s);
}

template <typename T>
void launch_cyl_efield(const GridP &g, int mode, T *const E[3], T *const B[3], T *const J[3], cudaStream_t s)
{
    const CylP cp = cyl_params(g);
    const int ni = g.mx - 2 - (g.inc_axis ? 4 : 3);   // i .. mx-3
    const dim3 grid((ni + 31) / 32, (g.my - 5 + 7) / 8, g.mz - 5), block(32, 8, 1);
    if (mode == 0) k_cyl_e<T, 0><<<grid, block, 0, s>>>(g, cp, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2]);
    else k_cyl_e<T, 2><<<grid, block, 0, s>>>(g, cp, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2]);
    count_launches(1);
    if (g.inc_axis) {   // UpdateEFldAxis
        k_cyl_e_axis<T><<<dim3((g.my + 127) / 128, g.mz), 128, 0, s>>>(g, E[0], E[1], E[2]);
        count_launches(1);
    }
    halo<T>(g, E, s);
}

template <typename T>
void launch_cyl_fold(const GridP &g, T *const J[3], cudaStream_t s)
{
    for (int c = 0; c < 3; c++) k_cyl_fold_z<T><<<dim3((g.mx + 127) / 128, g.my), 128, 0, s>>>(g, J[c]);
    for (int c = 0; c < 3; c++) k_cyl_fold_y<T><<<dim3((g.mx + 127) / 128, g.mz - 5), 128, 0, s>>>(g, J[c]);
    count_launches(6);
}

template void launch_cyl_bhalf<double>(const GridP &, double *const[3], double *const[3], cudaStream_t);
template void launch_cyl_bhalf<float>(const GridP &, float *const[3], float *const[3], cudaStream_t);
template void launch_cyl_efield<double>(const GridP &, int, double *const[3], double *const[3], double *const[3],
                                        cudaStream_t);
template void launch_cyl_efield<float>(const GridP &, int, float *const[3], float *const[3], float *const[3],
                                       cudaStream_t);
template void launch_cyl_fold<double>(const GridP &, double *const[3], cudaStream_t);
template void launch_cyl_fold<float>(const GridP &, float *const[3], cudaStream_t);

// ---------------------------------------------------------------------------
// Mover
// ---------------------------------------------------------------------------

// Interp_VecEM_GridPoints at (x, y, z): node averages of GatherVecEfld /
// GatherVecBfld with the trilinear weights (3D).
__device__ __forceinline__ void interp3(const GridP &g, const double *Ex, const double *Ey, const double *Ez,
                                        const double *Bx, const double *By, const double *Bz, double x, double y,
                                        double z, double pE[3], double pB[3])
{
    const int ip = (int)x, jp = (int)y, kp = (int)z;
    const double dx = x - ip, dy = y - jp, dz = z - kp;
    double wt[8];
#pragma unroll
    for (int nn = 0; nn < 8; nn++) {
        const double wx = (nn & 1) ? (0.0 + 1.0 * dx) : (1.0 + -1.0 * dx);
        const double wy = (nn & 2) ? (0.0 + 1.0 * dy) : (1.0 + -1.0 * dy);
        const double wz = (nn & 4) ? (0.0 + 1.0 * dz) : (1.0 + -1.0 * dz);
        wt[nn] = (wx * wy) * wz;
    }
    const long long sy = g.sy, sz = g.sz;
    const long long c0 = cidx(g, ip, jp, kp);
    pE[0] = pE[1] = pE[2] = pB[0] = pB[1] = pB[2] = 0.0;
#pragma unroll
    for (int nn = 0; nn < 8; nn++) {
        const long long nd = c0 + (nn & 1) + ((nn >> 1) & 1) * sy + ((nn >> 2) & 1) * sz;
        const double vex = (ldd(Ex + nd - 1) + ldd(Ex + nd)) * 0.5;
        const double vey = (ldd(Ey + nd - sy) + ldd(Ey + nd)) * 0.5;
        const double vez = (ldd(Ez + nd - sz) + ldd(Ez + nd)) * 0.5;
        const double vbx = (((ldd(Bx + nd - sy - sz) + ldd(Bx + nd - sz)) + ldd(Bx + nd - sy)) + ldd(Bx + nd)) * 0.25 + g.bext[0];
        const double vby = (((ldd(By + nd - 1 - sz) + ldd(By + nd - 1)) + ldd(By + nd - sz)) + ldd(By + nd)) * 0.25 + g.bext[1];
        const double vbz = (((ldd(Bz + nd - 1 - sy) + ldd(Bz + nd - 1)) + ldd(Bz + nd - sy)) + ldd(Bz + nd)) * 0.25 + g.bext[2];
        pE[0] = pE[0] + wt[nn] * vex;
        pE[1] = pE[1] + wt[nn] * vey;
        pE[2] = pE[2] + wt[nn] * vez;
        pB[0] = pB[0] + wt[nn] * vbx;
        pB[1] = pB[1] + wt[nn] * vby;
        pB[2] = pB[2] + wt[nn] * vbz;
    }
}

__device__ __forceinline__ void half_boris_d(double sqc, const double pE[3], const double pB[3], double &u0, double &v0,
                                           double &w0)
{
    const double gg = 1.0 / sqrt(((sqc + u0 * u0) + v0 * v0) + w0 * w0);
    const double bx = gg * pB[0], by = gg * pB[1], bz = gg * pB[2];
    const double ff = 2.0 / (((1.0 + bx * bx) + by * by) + bz * bz);
    const double u1 = ((u0 + v0 * bz) - w0 * by) * ff;
    const double v1 = ((v0 + w0 * bx) - u0 * bz) * ff;
    const double w1 = ((w0 + u0 * by) - v0 * bx) * ff;
    u0 = ((u0 + v1 * bz) - w1 * by) + pE[0];
    v0 = ((v0 + w1 * bx) - u1 * bz) + pE[1];
    w0 = ((w0 + u1 * by) - v1 * bx) + pE[2];
}

// DepositCurrentPIC (deposit.F90:11-103, 3D) with atomics.
__device__ void deposit_pic(const GridP &g, double *Jx, double *Jy, double *Jz, double x0, double y0, double z0,
                            double x, double y, double z, double q)
{
    const double qthis = q * g.qi;
    const int i1 = (int)floor(x0), i2 = (int)floor(x), j1 = (int)floor(y0), j2 = (int)floor(y);
    const int k1 = (int)floor(z0), k2 = (int)floor(z);
    const double xr = fmin((double)(min(i1, i2) + 1), fmax((double)max(i1, i2), 0.5 * (x0 + x)));
    const double yr = fmin((double)(min(j1, j2) + 1), fmax((double)max(j1, j2), 0.5 * (y0 + y)));
    const double zr = fmin((double)(min(k1, k2) + 1), fmax((double)max(k1, k2), 0.5 * (z0 + z)));
    const double Fx1 = qthis * (xr - x0), Fy1 = qthis * (yr - y0), Fz1 = qthis * (zr - z0);
    const double Wx1 = 0.5 * (x0 + xr) - i1, Wy1 = 0.5 * (y0 + yr) - j1;
    const double Wx2 = 0.5 * (x + xr) - i2, Wy2 = 0.5 * (y + yr) - j2;
    const double Wz1 = 0.5 * (z0 + zr) - k1, Wz2 = 0.5 * (z + zr) - k2;
    const double Fx2 = qthis * (x - xr), Fy2 = qthis * (y - yr), Fz2 = qthis * (z - zr);
    atomicAdd(Jx + cidx(g, i1, j1, k1), (Fx1 * (1.0 - Wy1)) * (1.0 - Wz1));
    atomicAdd(Jx + cidx(g, i1, j1 + 1, k1), (Fx1 * Wy1) * (1.0 - Wz1));
    atomicAdd(Jx + cidx(g, i1, j1, k1 + 1), (Fx1 * (1.0 - Wy1)) * Wz1);
    atomicAdd(Jx + cidx(g, i1, j1 + 1, k1 + 1), (Fx1 * Wy1) * Wz1);
    atomicAdd(Jx + cidx(g, i2, j2, k2), (Fx2 * (1.0 - Wy2)) * (1.0 - Wz2));
    atomicAdd(Jx + cidx(g, i2, j2 + 1, k2), (Fx2 * Wy2) * (1.0 - Wz2));
    atomicAdd(Jx + cidx(g, i2, j2, k2 + 1), (Fx2 * (1.0 - Wy2)) * Wz2);
    atomicAdd(Jx + cidx(g, i2, j2 + 1, k2 + 1), (Fx2 * Wy2) * Wz2);
    atomicAdd(Jy + cidx(g, i1, j1, k1), (Fy1 * (1.0 - Wx1)) * (1.0 - Wz1));
    atomicAdd(Jy + cidx(g, i1 + 1, j1, k1), (Fy1 * Wx1) * (1.0 - Wz1));
    atomicAdd(Jy + cidx(g, i1, j1, k1 + 1), (Fy1 * (1.0 - Wx1)) * Wz1);
    atomicAdd(Jy + cidx(g, i1 + 1, j1, k1 + 1), (Fy1 * Wx1) * Wz1);
    atomicAdd(Jy + cidx(g, i2, j2, k2), (Fy2 * (1.0 - Wx2)) * (1.0 - Wz2));
    atomicAdd(Jy + cidx(g, i2 + 1, j2, k2), (Fy2 * Wx2) * (1.0 - Wz2));
    atomicAdd(Jy + cidx(g, i2, j2, k2 + 1), (Fy2 * (1.0 - Wx2)) * Wz2);
    atomicAdd(Jy + cidx(g, i2 + 1, j2, k2 + 1), (Fy2 * Wx2) * Wz2);
    atomicAdd(Jz + cidx(g, i1, j1, k1), (Fz1 * (1.0 - Wx1)) * (1.0 - Wy1));
    atomicAdd(Jz + cidx(g, i1 + 1, j1, k1), (Fz1 * Wx1) * (1.0 - Wy1));
    atomicAdd(Jz + cidx(g, i1, j1 + 1, k1), (Fz1 * (1.0 - Wx1)) * Wy1);
    atomicAdd(Jz + cidx(g, i1 + 1, j1 + 1, k1), (Fz1 * Wx1) * Wy1);
    atomicAdd(Jz + cidx(g, i2, j2, k2), (Fz2 * (1.0 - Wx2)) * (1.0 - Wy2));
    atomicAdd(Jz + cidx(g, i2 + 1, j2, k2), (Fz2 * Wx2) * (1.0 - Wy2));
    atomicAdd(Jz + cidx(g, i2, j2 + 1, k2), (Fz2 * (1.0 - Wx2)) * Wy2);
    atomicAdd(Jz + cidx(g, i2 + 1, j2 + 1, k2), (Fz2 * Wx2) * Wy2);
}

constexpr int kMaxSubsteps = 100000;

// One particle of the cylindrical mover (cyl_movdep_strang.F90:14-378, the
// near-axis sub-stepper :404-566).  interp(x, y, z, pE, pB) is
// Interp_VecEM_GridPoints at a position; dep(i, j, k, o, far) adds the VecJ
// entries o of the zigzag at start cell (i, j, k), far when the particle
// crossed more than one cell along an axis.  Returns false when the particle
// keeps its state (range or non-finite momenta); nc receives its new cell.
template <class Interp, class Dep>
__device__ __forceinline__ bool cyl_move_one(const GridP &g, const CylP &cp, const PartF64 &p, long long n,
                                             int flv, double qn, double x0, double y0, double z0, double ui,
                                             double vi, double wi, const double *__restrict__ Ex,
                                             const double *__restrict__ Ey, const double *__restrict__ Ez,
                                             const double *__restrict__ Bx, const double *__restrict__ By,
                                             const double *__restrict__ Bz, double *Jx, double *Jy, double *Jz,
                                             int *err, Interp &&interp, Dep &&dep, int *nc)
{
    const double c = g.c, sqc = g.sqc, cinv = g.cinv;
    const double r_proc = cp.rmin - 3.0;  // xborders + rshift - xmin
    if (flv < 0 || flv > PIC_MAX_FLVR || !(x0 >= 2.5 && x0 < (double)(g.mx - 1)) ||
        !(y0 >= 2.0 && y0 < (double)(g.my - 1)) || !(z0 >= 2.0 && z0 < (double)(g.mz - 1))) {
        raise_error(err, PIC_DEVERR_RANGE);
        return false;
    }
    if (flv == 0) return false;  // a hole moves nowhere and deposits zero
    double qthis = qn * g.qi;
    const double qm = g.qm[flv] * 0.25;  // cyl_movdep_strang.F90:100
    // MovDepAxis re-moves the particles within 1.5 cells of the axis on the
    // rank holding it (:296, 390-402)
    const bool near_axis = g.inc_axis && x0 < 4.5;
    const int ip0 = (int)x0, jp0 = (int)y0, kp0 = (int)z0;
    double pE[3], pB[3];
    interp(x0, y0, z0, pE, pB);
    for (int d = 0; d < 3; d++) {
        pE[d] = pE[d] * qm;
        pB[d] = pB[d] * qm;
    }
    double u0 = c * ui + pE[0], v0 = c * vi + pE[1], w0 = c * wi + pE[2];
    half_boris_d(sqc, pE, pB, u0, v0, w0);
    if (!finite3(u0, v0, w0)) {   // the particle keeps its state (see finite3)
        raise_error(err, PIC_DEVERR_NAN);
        return false;
    }
    double u1 = u0 * cinv, v1 = v0 * cinv;
    const double gg = sqc / sqrt(((sqc + u0 * u0) + v0 * v0) + w0 * w0);
    const double r0 = (x0 + r_proc) * 1.0;
    const double xx1 = r0 + u1 * gg, yy1 = v1 * gg;
    double r1 = sqrt(xx1 * xx1 + yy1 * yy1);
    double xn = r1 * 1.0 - r_proc;
    double yn = y0 + atan(yy1 / xx1) * cp.inv_dtheta;
    double zn = z0 + (wi * gg) * 1.0;  // z moves with this step's initial w (:202)
    r1 = 1.0 / r1;
    u1 = (r0 * u0 + ((u0 * u1) * gg + v0 * yy1)) * r1;
    v1 = (v0 * r0) * r1;
    if (!near_axis && (!(xn >= 2.0 && xn < (double)(g.mx - 1)) || !(yn >= 2.0 && yn < (double)(g.my - 1)) ||
                      !(zn >= 2.0 && zn < (double)(g.mz - 1)))) {
        raise_error(err, PIC_DEVERR_RANGE);  // the azimuthal step left the ghost frame
        return false;
    }
    const int ip = (int)xn, jp = (int)yn, kp = (int)zn;
    if (!near_axis) {
        interp(xn, yn, zn, pE, pB);
    } else {
        pE[0] = pE[1] = pE[2] = pB[0] = pB[1] = pB[2] = 0.0;  // redone by the sub-stepper below
    }
    for (int d = 0; d < 3; d++) {
        pE[d] = pE[d] * qm;
        pB[d] = pB[d] * qm;
    }
    u0 = u1 + pE[0];
    v0 = v1 + pE[1];
    w0 = w0 + pE[2];
    half_boris_d(sqc, pE, pB, u0, v0, w0);
    double un = u0 * cinv, vn = v0 * cinv, wn = w0 * cinv;
    if (near_axis) {
        // SubStepMovDep (:404-438) from the step's initial state
        qthis = 0.0;
        xn = x0; yn = y0; zn = z0; un = ui; vn = vi; wn = wi;
        double t = 0.0, dt = 1.0, sx0 = x0, sy0 = y0, sz0 = z0;
        int tries = 0;
        while (t < 1.0) {
            if (++tries > kMaxSubsteps) {
                raise_error(err, PIC_DEVERR_SUBSTEP);
                break;
            }
            const double delt = (t + dt > 1.0) ? 1.0 - t : dt;
            // MovePrtlAxis (:462-566)
            interp3(g, Ex, Ey, Ez, Bx, By, Bz, sx0, sy0, sz0, pE, pB);
            for (int d = 0; d < 3; d++) {
                pE[d] = (pE[d] * qm) * delt;
                pB[d] = (pB[d] * qm) * delt;
            }
            double a0 = c * un + pE[0], b0 = c * vn + pE[1], c0 = c * wn + pE[2];
            half_boris_d(sqc, pE, pB, a0, b0, c0);
            if (!finite3(a0, b0, c0)) {
                raise_error(err, PIC_DEVERR_NAN);
                return false;   // the particle keeps its state
            }
            double a1 = a0 * cinv, b1 = b0 * cinv;
            const double c1 = c0 * cinv;
            const double g2 = sqc / sqrt(((sqc + a0 * a0) + b0 * b0) + c0 * c0);
            const double rr0 = (sx0 - 3.5) * 1.0;
            const double X1 = rr0 + (a1 * g2) * delt;
            const double Y1 = (b1 * g2) * delt;
            const double R1 = sqrt(X1 * X1 + Y1 * Y1);
            const double dy = X1 > 0 ? atan(Y1 / X1) * cp.inv_dtheta : 0.0;
            if (fabs(dy) > 0.45) {
                dt = dt * 0.5;
                continue;
            }
            double nx;
            if (X1 > 0) {
                nx = R1 / 1.0 + 3.5;
                a1 = (rr0 * a0 + ((a0 * a1) * g2 * delt + b0 * Y1)) / R1;
                b1 = (b0 * rr0) / R1;
            } else {
                nx = X1 / 1.0 + 3.5;
            }
            const double ny = yn + dy;
            const double nz = zn + ((c1 * g2) * delt) * 1.0;
            interp3(g, Ex, Ey, Ez, Bx, By, Bz, nx, ny, nz, pE, pB);
            for (int d = 0; d < 3; d++) {
                pE[d] = (pE[d] * qm) * delt;
                pB[d] = (pB[d] * qm) * delt;
            }
            a0 = a1 + pE[0];
            b0 = b1 + pE[1];
            c0 = c0 + pE[2];
            half_boris_d(sqc, pE, pB, a0, b0, c0);
            xn = nx; yn = ny; zn = nz;
            un = a0 * cinv; vn = b0 * cinv; wn = c0 * cinv;
            t = t + delt;
            deposit_pic(g, Jx, Jy, Jz, sx0, sy0, sz0, xn, yn, zn, qn);
            // PrtlAxisBC (:450-460)
            if (xn < 3.5) {
                xn = 3.5 + (3.5 - xn);
                yn = yn + g.ny / 2.0;
                un = -un;
                vn = -vn;
            }
            if (yn > g.ymax) yn = yn - g.ylen;
            if (yn < g.ymin) yn = yn + g.ylen;
            dt = dt * 1.7;
            sx0 = xn; sy0 = yn; sz0 = zn;
        }
    }
    // zigzag deposit; both segments use the start cell (:341)
    if (qthis != 0.0) {
        const double xr = fmin((double)(min(ip0, ip) + 1), fmax((double)max(ip0, ip), 0.5 * (x0 + xn)));
        const double yr = fmin((double)(min(jp0, jp) + 1), fmax((double)max(jp0, jp), 0.5 * (y0 + yn)));
        const double zr = fmin((double)(min(kp0, kp) + 1), fmax((double)max(kp0, kp), 0.5 * (z0 + zn)));
        double o[12], o2[12];
        segment<double, 3>(qthis * (xr - x0), qthis * (yr - y0), qthis * (zr - z0), 0.5 * (x0 + xr) - ip0,
                           0.5 * (y0 + yr) - jp0, 0.5 * (z0 + zr) - kp0, o);
        segment<double, 3>(qthis * (xn - xr), qthis * (yn - yr), qthis * (zn - zr), 0.5 * (xn + xr) - ip,
                           0.5 * (yn + yr) - jp, 0.5 * (zn + zr) - kp, o2);
        for (int e = 0; e < 12; e++) o[e] = o[e] + o2[e];
        dep(ip0, jp0, kp0, o, abs(ip - ip0) > 1 || abs(jp - jp0) > 1 || abs(kp - kp0) > 1);
    }
    p.x[n] = xn;
    p.y[n] = yn;
    p.z[n] = zn;
    p.u[n] = un;
    p.v[n] = vn;
    p.w[n] = wn;
    nc[0] = (int)xn;
    nc[1] = (int)yn;
    nc[2] = (int)zn;
    return true;
}

// The per-particle mover over slots first .. used - 1 (first: all of them
// when null; after a reorder of the tiled form, the particles appended since).
__global__ void __launch_bounds__(kThreads) k_cyl_move(GridP g, CylP cp, PartF64 p, const Counters *__restrict__ cnt,
                                                       const long long *__restrict__ first,
                                                       const double *__restrict__ Ex, const double *__restrict__ Ey,
                                                       const double *__restrict__ Ez, const double *__restrict__ Bx,
                                                       const double *__restrict__ By, const double *__restrict__ Bz,
                                                       double *Jx, double *Jy, double *Jz, int *err)
{
    const long long used = cnt->used, n0 = first ? *first : 0;
    auto interp = [&](double x, double y, double z, double pE[3], double pB[3]) {
        interp3(g, Ex, Ey, Ez, Bx, By, Bz, x, y, z, pE, pB);
    };
    auto dep = [&](int i, int j, int k, const double *o, bool) { scatter<double, 3>(g, Jx, Jy, Jz, cidx(g, i, j, k), o); };
    for (long long n = n0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; n < used;
         n += (long long)gridDim.x * blockDim.x) {
        int nc[3];
        cyl_move_one(g, cp, p, n, p.flv[n], p.q[n], p.x[n], p.y[n], p.z[n], p.u[n], p.v[n], p.w[n], Ex, Ey, Ez, Bx,
                     By, Bz, Jx, Jy, Jz, err, interp, dep, nc);
    }
}

// The tiled form after a reorder: tile64.cuh's boxes, widened by one cell so
// that the gather at the moved position (the second half of the Strang
// split) finds its nodes; a particle within one cell of its start deposits
// into the fixed-point box (two segments of at most one cell per axis add at
// most 2 q qi to a word), the rest (near-axis sub-steps, long azimuthal
// steps, cells outside the box) through global memory.
__global__ void __launch_bounds__(kT64Threads, 2) k_cyl_move_tiled(GridP g, CylP cp, PartF64 p, Tiles64 T,
                                                                   const double *__restrict__ Ex,
                                                                   const double *__restrict__ Ey,
                                                                   const double *__restrict__ Ez,
                                                                   const double *__restrict__ Bx,
                                                                   const double *__restrict__ By,
                                                                   const double *__restrict__ Bz, double *Jx,
                                                                   double *Jy, double *Jz, int *err)
{
    extern __shared__ __align__(16) double smem64[];
    move_tile64<3, 1>(g, p, T, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, 2.0, smem64,
                      [&](const P64 &s, uint32_t n, const Tile64Ctx &ctx, int *nc) {
        auto interp = [&](double x, double y, double z, double pE[3], double pB[3]) {
            const int i = (int)x, j = (int)y, k = (int)z;
            int nb;
            if (ctx.use_box && in_box<3>(ctx.bx, i, j, k, nb)) {
                double wt[8];
                weights<double, 3>(x - i, y - j, z - k, wt);
                gather_box64<3>(ctx.bx, ctx.sN, nb, wt, pE, pB);
            } else {
                interp3(g, Ex, Ey, Ez, Bx, By, Bz, x, y, z, pE, pB);
            }
        };
        auto dep = [&](int i, int j, int k, const double *o, bool far) {
            if (!far && ctx.use_box && ctx.in_jbox<3>(i, j, k))
                deposit_box64<3>(ctx.bx, ctx.sJ, ctx.jcell<3>(i, j, k), o, ctx.S);
            else
                scatter<double, 3>(g, Jx, Jy, Jz, cidx(g, i, j, k), o);
        };
        if (!cyl_move_one(g, cp, p, n, s.flv, s.q, s.x, s.y, s.z, s.u, s.v, s.w, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz,
                          err, interp, dep, nc))
            return false;
        // the particles that stay in the interior bound the next box
        return nc[0] >= 3 && nc[0] <= g.mx - 3 && nc[1] >= 3 && nc[1] <= g.my - 3 && nc[2] >= 3 && nc[2] <= g.mz - 3;
    });
}

// AxisCurrentBC (cyl_movdep_strang.F90:570-584), all j, k.
template <typename T>
__global__ void k_cyl_axis_current(GridP g, T *Jx, T *Jy, T *Jz)
{
    const int j = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 1 + blockIdx.y;
    if (j > g.my) return;
    Jy[cidx(g, 4, j, k)] = Jy[cidx(g, 4, j, k)] - Jy[cidx(g, 3, j, k)];
    Jz[cidx(g, 4, j, k)] = Jz[cidx(g, 4, j, k)] - Jz[cidx(g, 3, j, k)];
    Jx[cidx(g, 3, j, k)] = (T)0.0;
    Jy[cidx(g, 2, j, k)] = (T)0.0;
    Jz[cidx(g, 2, j, k)] = (T)0.0;
}

void launch_cyl_move_deposit(const GridP &g, const PartF64 &p, const Counters *cnt, double *const E[3],
                             double *const B[3], double *const J[3], int *err, cudaStream_t s, const Tiles64 *T)
{
    const CylP cp = cyl_params(g);
    if (T) {
        static bool attr_set = false;
        if (!attr_set) {
            cudaFuncSetAttribute(k_cyl_move_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, kTile64SmemBytes);
            attr_set = true;
        }
        k_cyl_move_tiled<<<T->ntiles, kT64Threads, T->smem_bytes, s>>>(g, cp, p, *T, E[0], E[1], E[2], B[0], B[1],
                                                                        B[2], J[0], J[1], J[2], err);
        count_launches(1);
    }
    // every particle, or the ones appended since the reorder
    k_cyl_move<<<kSMs * 8, kThreads, 0, s>>>(g, cp, p, cnt, T ? T->np : nullptr, E[0], E[1], E[2], B[0], B[1], B[2],
                                             J[0], J[1], J[2], err);
    count_launches(1);
    if (g.inc_axis) {   // AxisCurrentBC on the rank holding the axis
        k_cyl_axis_current<double><<<dim3((g.my + 127) / 128, g.mz), 128, 0, s>>>(g, J[0], J[1], J[2]);
        count_launches(1);
    }
}

// ---------------------------------------------------------------------------
// FP32 cell-relative form of the cylindrical mover.  The algorithm is the
// one of k_cyl_move (cyl_movdep_strang.F90:14-378 with the near-axis
// sub-stepper :404-566); positions are (cell, offset) as in the Cartesian
// FP32 form, and the radial, azimuthal and axial displacements are added to
// the offsets, never to absolute coordinates: the new radius is r0 + dr with
// dr = (dx (2 r0 + dx) + dy^2) / (r1 + r0) (= r1 - r0 without cancellation),
// so FP32 keeps sub-cell resolution far from the axis and along a long z.
// Near the axis (x < 4.5) the sub-stepper runs on absolute x and theta
// (small numbers there) and on z relative to the start cell.  The periodic
// wrap in theta and z and the drop of particles leaving the outer radius are
// integer updates of the cell, inside the mover.
// ---------------------------------------------------------------------------

// Interp_VecEM_GridPoints at cell (ip, jp, kp) + offsets (dx, dy, dz).
__device__ __forceinline__ void interp3f(const GridP &g, const float *__restrict__ Ex, const float *__restrict__ Ey,
                                         const float *__restrict__ Ez, const float *__restrict__ Bx,
                                         const float *__restrict__ By, const float *__restrict__ Bz, int ip, int jp,
                                         int kp, float dx, float dy, float dz, float pE[3], float pB[3])
{
    float wt[8];
#pragma unroll
    for (int nn = 0; nn < 8; nn++) {
        const float wx = (nn & 1) ? dx : 1.f - dx;
        const float wy = (nn & 2) ? dy : 1.f - dy;
        const float wz = (nn & 4) ? dz : 1.f - dz;
        wt[nn] = (wx * wy) * wz;
    }
    const long long sy = g.sy, sz = g.sz;
    const long long c0 = cidx(g, ip, jp, kp);
    pE[0] = pE[1] = pE[2] = pB[0] = pB[1] = pB[2] = 0.f;
#pragma unroll
    for (int nn = 0; nn < 8; nn++) {
        const long long nd = c0 + (nn & 1) + ((nn >> 1) & 1) * sy + ((nn >> 2) & 1) * sz;
        const float vex = (ldd(Ex + nd - 1) + ldd(Ex + nd)) * 0.5f;
        const float vey = (ldd(Ey + nd - sy) + ldd(Ey + nd)) * 0.5f;
        const float vez = (ldd(Ez + nd - sz) + ldd(Ez + nd)) * 0.5f;
        const float vbx = (((ldd(Bx + nd - sy - sz) + ldd(Bx + nd - sz)) + ldd(Bx + nd - sy)) + ldd(Bx + nd)) * 0.25f + g.bext_f[0];
        const float vby = (((ldd(By + nd - 1 - sz) + ldd(By + nd - 1)) + ldd(By + nd - sz)) + ldd(By + nd)) * 0.25f + g.bext_f[1];
        const float vbz = (((ldd(Bz + nd - 1 - sy) + ldd(Bz + nd - 1)) + ldd(Bz + nd - sy)) + ldd(Bz + nd)) * 0.25f + g.bext_f[2];
        pE[0] = fmaf(wt[nn], vex, pE[0]);
        pE[1] = fmaf(wt[nn], vey, pE[1]);
        pE[2] = fmaf(wt[nn], vez, pE[2]);
        pB[0] = fmaf(wt[nn], vbx, pB[0]);
        pB[1] = fmaf(wt[nn], vby, pB[1]);
        pB[2] = fmaf(wt[nn], vbz, pB[2]);
    }
}

// Absolute (cell + offset) coordinate x split into cell and offset.
__device__ __forceinline__ int split_coord(float x, float &off)
{
    const float f = floorf(x);
    off = x - f;
    return (int)f;
}

__device__ __forceinline__ void half_boris_f(float sqc, const float pE[3], const float pB[3], float &u0, float &v0,
                                             float &w0)
{
    const float gg = rsqrtf(fmaf(w0, w0, fmaf(v0, v0, fmaf(u0, u0, sqc))));
    const float bx = gg * pB[0], by = gg * pB[1], bz = gg * pB[2];
    const float ff = __fdividef(2.f, fmaf(bz, bz, fmaf(by, by, fmaf(bx, bx, 1.f))));
    const float u1 = fmaf(-w0, by, fmaf(v0, bz, u0)) * ff;
    const float v1 = fmaf(-u0, bz, fmaf(w0, bx, v0)) * ff;
    const float w1 = fmaf(-v0, bx, fmaf(u0, by, w0)) * ff;
    u0 = fmaf(-w1, by, fmaf(v1, bz, u0)) + pE[0];
    v0 = fmaf(-u1, bz, fmaf(w1, bx, v0)) + pE[1];
    w0 = fmaf(-v1, bx, fmaf(u1, by, w0)) + pE[2];
}

// DepositCurrentPIC (deposit.F90:11-103) for the sub-stepper: x, y absolute,
// z relative to cell kb.
__device__ void deposit_pic_f(const GridP &g, float *Jx, float *Jy, float *Jz, float x0, float y0, float z0, float x,
                              float y, float z, int kb, float qthis)
{
    const int i1 = (int)floorf(x0), i2 = (int)floorf(x), j1 = (int)floorf(y0), j2 = (int)floorf(y);
    const int kk1 = (int)floorf(z0), kk2 = (int)floorf(z);
    const float xr = fminf((float)(min(i1, i2) + 1), fmaxf((float)max(i1, i2), 0.5f * (x0 + x)));
    const float yr = fminf((float)(min(j1, j2) + 1), fmaxf((float)max(j1, j2), 0.5f * (y0 + y)));
    const float zr = fminf((float)(min(kk1, kk2) + 1), fmaxf((float)max(kk1, kk2), 0.5f * (z0 + z)));
    const float Fx1 = qthis * (xr - x0), Fy1 = qthis * (yr - y0), Fz1 = qthis * (zr - z0);
    const float Wx1 = 0.5f * (x0 + xr) - i1, Wy1 = 0.5f * (y0 + yr) - j1;
    const float Wx2 = 0.5f * (x + xr) - i2, Wy2 = 0.5f * (y + yr) - j2;
    const float Wz1 = 0.5f * (z0 + zr) - kk1, Wz2 = 0.5f * (z + zr) - kk2;
    const float Fx2 = qthis * (x - xr), Fy2 = qthis * (y - yr), Fz2 = qthis * (z - zr);
    const int k1 = kb + kk1, k2 = kb + kk2;
    atomicAdd(Jx + cidx(g, i1, j1, k1), (Fx1 * (1.f - Wy1)) * (1.f - Wz1));
    atomicAdd(Jx + cidx(g, i1, j1 + 1, k1), (Fx1 * Wy1) * (1.f - Wz1));
    atomicAdd(Jx + cidx(g, i1, j1, k1 + 1), (Fx1 * (1.f - Wy1)) * Wz1);
    atomicAdd(Jx + cidx(g, i1, j1 + 1, k1 + 1), (Fx1 * Wy1) * Wz1);
    atomicAdd(Jx + cidx(g, i2, j2, k2), (Fx2 * (1.f - Wy2)) * (1.f - Wz2));
    atomicAdd(Jx + cidx(g, i2, j2 + 1, k2), (Fx2 * Wy2) * (1.f - Wz2));
    atomicAdd(Jx + cidx(g, i2, j2, k2 + 1), (Fx2 * (1.f - Wy2)) * Wz2);
    atomicAdd(Jx + cidx(g, i2, j2 + 1, k2 + 1), (Fx2 * Wy2) * Wz2);
    atomicAdd(Jy + cidx(g, i1, j1, k1), (Fy1 * (1.f - Wx1)) * (1.f - Wz1));
    atomicAdd(Jy + cidx(g, i1 + 1, j1, k1), (Fy1 * Wx1) * (1.f - Wz1));
    atomicAdd(Jy + cidx(g, i1, j1, k1 + 1), (Fy1 * (1.f - Wx1)) * Wz1);
    atomicAdd(Jy + cidx(g, i1 + 1, j1, k1 + 1), (Fy1 * Wx1) * Wz1);
    atomicAdd(Jy + cidx(g, i2, j2, k2), (Fy2 * (1.f - Wx2)) * (1.f - Wz2));
    atomicAdd(Jy + cidx(g, i2 + 1, j2, k2), (Fy2 * Wx2) * (1.f - Wz2));
    atomicAdd(Jy + cidx(g, i2, j2, k2 + 1), (Fy2 * (1.f - Wx2)) * Wz2);
    atomicAdd(Jy + cidx(g, i2 + 1, j2, k2 + 1), (Fy2 * Wx2) * Wz2);
    atomicAdd(Jz + cidx(g, i1, j1, k1), (Fz1 * (1.f - Wx1)) * (1.f - Wy1));
    atomicAdd(Jz + cidx(g, i1 + 1, j1, k1), (Fz1 * Wx1) * (1.f - Wy1));
    atomicAdd(Jz + cidx(g, i1, j1 + 1, k1), (Fz1 * (1.f - Wx1)) * Wy1);
    atomicAdd(Jz + cidx(g, i1 + 1, j1 + 1, k1), (Fz1 * Wx1) * Wy1);
    atomicAdd(Jz + cidx(g, i2, j2, k2), (Fz2 * (1.f - Wx2)) * (1.f - Wy2));
    atomicAdd(Jz + cidx(g, i2 + 1, j2, k2), (Fz2 * Wx2) * (1.f - Wy2));
    atomicAdd(Jz + cidx(g, i2, j2 + 1, k2), (Fz2 * (1.f - Wx2)) * Wy2);
    atomicAdd(Jz + cidx(g, i2 + 1, j2 + 1, k2), (Fz2 * Wx2) * Wy2);
}

// The box current of a thread's consecutive particles that start in the same
// cell, summed in registers (FP32, in the box's fixed-point units) and added
// to the 64-bit box when the cell changes: a thread of the tiled mover walks
// one row of its brick, which the reorder fills with the particles of one or
// two cells.
constexpr uint32_t kNoCell = 0xffffffffu;
struct JAcc {
    float v[12];
    uint32_t a;   // box byte address of the cell's Jx word, or kNoCell
};

// One particle of the FP32 cylindrical mover: slot n, loaded state st.
// TILED (one CTA per brick, tile.cuh): the two gathers of the Strang step
// read the node box when their cell is in it, and the step's current (both
// segments in the start cell, :341) goes to the box (through acc) when the
// start cell is in it; otherwise, and always for the near-axis sub-stepper,
// global memory with the same arithmetic, so both forms move particles bit
// for bit alike.  The new cell, unwrapped from the brick centre, widens bd.
template <bool TILED>
__device__ __forceinline__ void cyl_push_f32(const GridP &g, const CylP &cp, const PartF32 &p, uint32_t n,
                                             const PState &st, const float *__restrict__ Ex,
                                             const float *__restrict__ Ey, const float *__restrict__ Ez,
                                             const float *__restrict__ Bx, const float *__restrict__ By,
                                             const float *__restrict__ Bz, float *Jx, float *Jy, float *Jz, int *err,
                                             const TileBox &tb, Bounds &bd, JAcc &acc, uint32_t *subq,
                                             uint32_t *subq_n)
{
    const float c = g.c_f, sqc = g.sqc_f, cinv = g.cinv_f, qi = g.qi_f;
    const float inv_dtheta = (float)cp.inv_dtheta;
    const float ymin = (float)g.ymin, ymax = (float)g.ymax, ylen = (float)g.ylen;
    const uint32_t key = st.key;
    const int flv = (int)(key >> kFlvShift);
    if (flv == 0) return;  // a hole moves nowhere and deposits zero
    int i, j, k;
    decode_cell(g, (int)(key & kCellMask), i, j, k);
    if (flv > PIC_MAX_FLVR || i < 3 || i > g.mx - 3 || j < 3 || j > g.my - 3 || k < 3 || k > g.mz - 3) {
        raise_error(err, PIC_DEVERR_RANGE);
        return;
    }
    const float dx = st.dx, dy = st.dy, dz = st.dz;
    const float ui = st.ux, vi = st.uy, wi = st.uz, w8 = st.w;
    const float qm = (float)(g.qm[flv] * 0.25);  // cyl_movdep_strang.F90:100
    int ni, nj, nk;            // new cell
    float ox, oy, oz;          // new offsets
    float un, vn, wn;
    const bool strang = i > 4 || (i == 4 && dx >= 0.5f);
    if (TILED) {
        // near-axis particles are left to k_cyl_substep_f32 (their slots
        // queued); the box of the next step covers their cell +- 1
        const uint32_t m = __ballot_sync(__activemask(), !strang);
        if (!strang) {
            const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(subq_n, (uint32_t)__popc(m));
            base = __shfl_sync(m, base, leader);
            subq[base + __popc(m & ((1u << lane) - 1u))] = n;
            const int u0 = i - tb.hc[0], u1 = unwrap_offset(j, tb.hc[1], g.ny), u2 = unwrap_offset(k, tb.hc[2], g.nz);
            bd.lo[0] = min(bd.lo[0], u0 - 1); bd.hi[0] = max(bd.hi[0], u0 + 1);
            bd.lo[1] = min(bd.lo[1], u1 - 1); bd.hi[1] = max(bd.hi[1], u1 + 1);
            bd.lo[2] = min(bd.lo[2], u2 - 1); bd.hi[2] = max(bd.hi[2], u2 + 1);
            return;
        }
    }
    if (strang) {
        // Strang step away from the axis (:104-341)
        int l0 = 0, l1 = 0, l2 = 0;   // box cell of the start cell
        bool in1 = false;
        if (TILED) {
            l0 = i - tb.hc[0] - tb.lo[0];
            l1 = unwrap_offset(j, tb.hc[1], g.ny) - tb.lo[1];
            l2 = unwrap_offset(k, tb.hc[2], g.nz) - tb.lo[2];
            in1 = (unsigned)l0 < (unsigned)tb.C[0] && (unsigned)l1 < (unsigned)tb.C[1] &&
                  (unsigned)l2 < (unsigned)tb.C[2];
        }
        float pE[3], pB[3];
        if (TILED && in1) {
            float wt[8];
            weights_f32<3>(dx, dy, dz, wt);
            pE[0] = pE[1] = pE[2] = pB[0] = pB[1] = pB[2] = 0.f;
            gather_box<3>(tb, l0 + tb.NX * l1 + tb.NXY * l2, wt, pE, pB);
        } else {
            interp3f(g, Ex, Ey, Ez, Bx, By, Bz, i, j, k, dx, dy, dz, pE, pB);
        }
        for (int d = 0; d < 3; d++) {
            pE[d] *= qm;
            pB[d] *= qm;
        }
        float u0 = fmaf(c, ui, pE[0]), v0 = fmaf(c, vi, pE[1]), w0 = fmaf(c, wi, pE[2]);
        half_boris_f(sqc, pE, pB, u0, v0, w0);
        if (!finite3(u0, v0, w0)) {   // the particle keeps its state (see finite3)
            raise_error(err, PIC_DEVERR_NAN);
            return;
        }
        float u1 = u0 * cinv, v1 = v0 * cinv;
        const float gg = sqc * rsqrtf(fmaf(w0, w0, fmaf(v0, v0, fmaf(u0, u0, sqc))));
        const float r0 = ((float)i - 3.5f) + dx;          // x - 3 + rmin, rmin = -0.5
        const float ddx = u1 * gg, ddy = v1 * gg;
        const float xx1 = r0 + ddx;
        const float r1 = sqrtf(fmaf(xx1, xx1, ddy * ddy));
        const float dr = __fdividef(fmaf(ddx, 2.f * r0 + ddx, ddy * ddy), r1 + r0);
        const float dth = atanf(__fdividef(ddy, xx1)) * inv_dtheta;
        const float dzz = wi * gg;                          // z moves with this step's initial w (:202)
        const float rinv = 1.f / r1;
        u1 = fmaf(r0, u0, fmaf(u0 * u1, gg, v0 * ddy)) * rinv;
        v1 = (v0 * r0) * rinv;
        // new cell and offsets (each displacement is below one cell here)
        const float Xn = dx + dr, Yn = dy + dth, Zn = dz + dzz;
        const int sx = Xn >= 1.f ? 1 : (Xn < 0.f ? -1 : 0);
        const int sy = Yn >= 1.f ? 1 : (Yn < 0.f ? -1 : 0);
        const int sz = Zn >= 1.f ? 1 : (Zn < 0.f ? -1 : 0);
        ni = i + sx;
        nj = j + sy;
        nk = k + sz;
        ox = Xn - (float)sx;
        oy = Yn - (float)sy;
        oz = Zn - (float)sz;
        bool in2 = false;
        if (TILED)
            in2 = (unsigned)(l0 + sx) < (unsigned)tb.C[0] && (unsigned)(l1 + sy) < (unsigned)tb.C[1] &&
                  (unsigned)(l2 + sz) < (unsigned)tb.C[2];
        if (TILED && in2) {
            float wt[8];
            weights_f32<3>(ox, oy, oz, wt);
            pE[0] = pE[1] = pE[2] = pB[0] = pB[1] = pB[2] = 0.f;
            gather_box<3>(tb, (l0 + sx) + tb.NX * (l1 + sy) + tb.NXY * (l2 + sz), wt, pE, pB);
        } else {
            interp3f(g, Ex, Ey, Ez, Bx, By, Bz, ni, nj, nk, ox, oy, oz, pE, pB);
        }
        for (int d = 0; d < 3; d++) {
            pE[d] *= qm;
            pB[d] *= qm;
        }
        u0 = u1 + pE[0];
        v0 = v1 + pE[1];
        w0 = w0 + pE[2];
        half_boris_f(sqc, pE, pB, u0, v0, w0);
        un = u0 * cinv;
        vn = v0 * cinv;
        wn = w0 * cinv;
        // zigzag deposit; both segments use the start cell (:341)
        const float qthis = w8 * qi * (TILED && in1 ? tb.S : 1.f);
        const float xr = fminf((float)(min(0, sx) + 1), fmaxf((float)max(0, sx), 0.5f * (dx + Xn)));
        const float yr = fminf((float)(min(0, sy) + 1), fmaxf((float)max(0, sy), 0.5f * (dy + Yn)));
        const float zr = fminf((float)(min(0, sz) + 1), fmaxf((float)max(0, sz), 0.5f * (dz + Zn)));
        float o[12], o2[12];
        segment<float, 3>(qthis * (xr - dx), qthis * (yr - dy), qthis * (zr - dz), 0.5f * (dx + xr),
                          0.5f * (dy + yr), 0.5f * (dz + zr), o);
        segment<float, 3>(qthis * (Xn - xr), qthis * (Yn - yr), qthis * (Zn - zr), 0.5f * (Xn + xr) - (float)sx,
                          0.5f * (Yn + yr) - (float)sy, 0.5f * (Zn + zr) - (float)sz, o2);
        for (int e = 0; e < 12; e++) o[e] = o[e] + o2[e];
        if (TILED && in1) {
            const uint32_t a = tb.sJ + 8u * (uint32_t)((l0 + 1) + tb.JX * (l1 + 1) + tb.JXY * (l2 + 1));
            if (a == acc.a) {
#pragma unroll
                for (int e = 0; e < 12; e++) acc.v[e] += o[e];
            } else {
                if (acc.a != kNoCell) red_entries_box_wide(acc.a, tb.jo, acc.v);
                acc.a = a;
#pragma unroll
                for (int e = 0; e < 12; e++) acc.v[e] = o[e];
            }
        } else {
            scatter<float, 3>(g, Jx, Jy, Jz, cidx(g, i, j, k), o);
        }
    } else {
        // SubStepMovDep (:404-438) from the step's initial state: x and
        // theta absolute (small here), z relative to the start cell
        float pE[3], pB[3];
        float xn = (float)i + dx, yn = (float)j + dy, zn = dz;
        un = ui;
        vn = vi;
        wn = wi;
        float t = 0.f, dt = 1.f, sx0 = xn, sy0 = yn, sz0 = zn;
        int tries = 0;
        while (t < 1.f) {
            if (++tries > kMaxSubsteps) {
                raise_error(err, PIC_DEVERR_SUBSTEP);
                break;
            }
            const float delt = (t + dt > 1.f) ? 1.f - t : dt;
            // MovePrtlAxis (:462-566)
            {
                float fx, fy, fz;
                const int ci = split_coord(sx0, fx), cj = split_coord(sy0, fy), ck = k + split_coord(sz0, fz);
                interp3f(g, Ex, Ey, Ez, Bx, By, Bz, ci, cj, ck, fx, fy, fz, pE, pB);
            }
            for (int d = 0; d < 3; d++) {
                pE[d] = (pE[d] * qm) * delt;
                pB[d] = (pB[d] * qm) * delt;
            }
            float a0 = fmaf(c, un, pE[0]), b0 = fmaf(c, vn, pE[1]), c0 = fmaf(c, wn, pE[2]);
            half_boris_f(sqc, pE, pB, a0, b0, c0);
            if (!finite3(a0, b0, c0)) {   // the particle keeps its state (see finite3)
                raise_error(err, PIC_DEVERR_NAN);
                return;
            }
            float a1 = a0 * cinv, b1 = b0 * cinv;
            const float c1 = c0 * cinv;
            const float g2 = sqc * rsqrtf(fmaf(c0, c0, fmaf(b0, b0, fmaf(a0, a0, sqc))));
            const float rr0 = sx0 - 3.5f;
            const float X1 = rr0 + (a1 * g2) * delt;
            const float Y1 = (b1 * g2) * delt;
            const float R1 = sqrtf(fmaf(X1, X1, Y1 * Y1));
            const float ddy = X1 > 0.f ? atanf(__fdividef(Y1, X1)) * inv_dtheta : 0.f;
            if (fabsf(ddy) > 0.45f) {
                dt = dt * 0.5f;
                continue;
            }
            float nx;
            if (X1 > 0.f) {
                nx = R1 + 3.5f;
                a1 = fmaf(rr0, a0, fmaf((a0 * a1) * g2, delt, b0 * Y1)) / R1;
                b1 = (b0 * rr0) / R1;
            } else {
                nx = X1 + 3.5f;
            }
            const float ny = yn + ddy;
            const float nz = zn + (c1 * g2) * delt;
            {
                float fx, fy, fz;
                const int ci = split_coord(nx, fx), cj = split_coord(ny, fy), ck = k + split_coord(nz, fz);
                interp3f(g, Ex, Ey, Ez, Bx, By, Bz, ci, cj, ck, fx, fy, fz, pE, pB);
            }
            for (int d = 0; d < 3; d++) {
                pE[d] = (pE[d] * qm) * delt;
                pB[d] = (pB[d] * qm) * delt;
            }
            a0 = a1 + pE[0];
            b0 = b1 + pE[1];
            c0 = c0 + pE[2];
            half_boris_f(sqc, pE, pB, a0, b0, c0);
            xn = nx;
            yn = ny;
            zn = nz;
            un = a0 * cinv;
            vn = b0 * cinv;
            wn = c0 * cinv;
            t = t + delt;
            deposit_pic_f(g, Jx, Jy, Jz, sx0, sy0, sz0, xn, yn, zn, k, w8 * qi);
            // PrtlAxisBC (:450-460)
            if (xn < 3.5f) {
                xn = 3.5f + (3.5f - xn);
                yn = yn + 0.5f * (float)g.ny;
                un = -un;
                vn = -vn;
            }
            if (yn > ymax) yn = yn - ylen;
            if (yn < ymin) yn = yn + ylen;
            dt = dt * 1.7f;
            sx0 = xn;
            sy0 = yn;
            sz0 = zn;
        }
        ni = split_coord(xn, ox);
        nj = split_coord(yn, oy);
        nk = k + split_coord(zn, oz);
    }
    // periodic theta and z, particles past the outer radius leave
    nj = wrap_index(nj, g.my);
    nk = wrap_index(nk, g.mz);
    uint32_t nkey = 0;
    if (ni >= 3 && ni <= g.mx - 3) {
        nkey = ((uint32_t)flv << kFlvShift) | (uint32_t)cidx(g, ni, nj, nk);
        if (TILED) {
            const int u0 = ni - tb.hc[0], u1 = unwrap_offset(nj, tb.hc[1], g.ny), u2 = unwrap_offset(nk, tb.hc[2], g.nz);
            bd.lo[0] = min(bd.lo[0], u0); bd.hi[0] = max(bd.hi[0], u0);
            bd.lo[1] = min(bd.lo[1], u1); bd.hi[1] = max(bd.hi[1], u1);
            bd.lo[2] = min(bd.lo[2], u2); bd.hi[2] = max(bd.hi[2], u2);
        }
    }
    p.key[n] = nkey;
    p.dx[n] = ox;
    p.dy[n] = oy;
    p.dz[n] = oz;
    p.ux[n] = un;
    p.uy[n] = vn;
    p.uz[n] = wn;
}

__global__ void __launch_bounds__(kThreads) k_cyl_move_f32(GridP g, CylP cp, PartF32 p, const Counters *__restrict__ cnt,
                                                           const float *__restrict__ Ex, const float *__restrict__ Ey,
                                                           const float *__restrict__ Ez, const float *__restrict__ Bx,
                                                           const float *__restrict__ By, const float *__restrict__ Bz,
                                                           float *Jx, float *Jy, float *Jz, int *err)
{
    const long long used = cnt->used;
    const TileBox tb = {};
    Bounds bd;
    JAcc acc;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < used; n += (long long)gridDim.x * blockDim.x)
        cyl_push_f32<false>(g, cp, p, (uint32_t)n, load_state<3>(p, (uint32_t)n), Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz,
                            err, tb, bd, acc, nullptr, nullptr);
}

// The near-axis particles the tiled mover queued (slots q[0 .. *qn)): the
// sub-stepper, spread over every SM (a brick next to the axis would
// otherwise hold its CTA for many times a brick's Strang steps, with the
// lanes of its warps waiting on the few that sub-step).
__global__ void __launch_bounds__(kThreads) k_cyl_substep_f32(GridP g, CylP cp, PartF32 p, const uint32_t *__restrict__ q,
                                                              const uint32_t *__restrict__ qn,
                                                              const float *__restrict__ Ex, const float *__restrict__ Ey,
                                                              const float *__restrict__ Ez, const float *__restrict__ Bx,
                                                              const float *__restrict__ By, const float *__restrict__ Bz,
                                                              float *Jx, float *Jy, float *Jz, int *err)
{
    const uint32_t nq = *qn;
    const TileBox tb = {};
    Bounds bd;
    JAcc acc;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nq; t += gridDim.x * blockDim.x) {
        const uint32_t n = q[t];
        cyl_push_f32<false>(g, cp, p, n, load_state<3>(p, n), Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, err, tb, bd, acc,
                            nullptr, nullptr);
    }
}

// Tiled form: one CTA per brick (after a reorder).  The box is the stored
// bounds of the brick's particles widened by one cell (the second gather is
// at the cell a particle moves to); the radius is not periodic.  Each thread
// loads its next particle while it moves this one.
__global__ void __launch_bounds__(kTileThreads, 2)
    k_cyl_move_f32_tiled(GridP g, CylP cp, PartF32 p, Bricks bk, const float *__restrict__ Ex,
                         const float *__restrict__ Ey, const float *__restrict__ Ez, const float *__restrict__ Bx,
                         const float *__restrict__ By, const float *__restrict__ Bz, float *Jx, float *Jy, float *Jz,
                         int *err)
{
    extern __shared__ __align__(16) float sm[];
    __shared__ TileShared ts;
    const int b = blockIdx.x;
    const uint32_t p0 = bk.tile_start[b], p1 = bk.tile_start[b + 1];
    if (p0 >= p1) return;
    TileBox tb;
    int home_lo[3], home_hi[3];
    brick_home<3>(g, bk, b, tb, home_lo, home_hi);
    // a Strang move is below one cell per axis, a sub-stepped one below two
    tile_setup<3, false, true>(g, bk, b, p1 - p0, 1, 2.f, sm, ts, tb, home_lo, home_hi, Ex, Ey, Ez, Bx, By, Bz);
    Bounds bd;
    bd.init();
    JAcc acc;
    acc.a = kNoCell;
    const uint32_t n0 = p0 + threadIdx.x;
    if (n0 < p1) {
        PState cur = load_state<3>(p, n0);
        for (uint32_t n = n0; n < p1; n += kTileThreads) {
            PState nxt = cur;
            if (p1 - n > kTileThreads) nxt = load_state<3>(p, n + kTileThreads);
            cyl_push_f32<true>(g, cp, p, n, cur, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, err, tb, bd, acc, bk.bid,
                               bk.count);
            cur = nxt;
        }
    }
    if (acc.a != kNoCell) red_entries_box_wide(acc.a, tb.jo, acc.v);
    __syncthreads();
    tile_finish<3, false, true>(g, bk, b, tb, sm, ts, bd, home_lo, home_hi, Jx, Jy, Jz);
}

void launch_cyl_move_deposit_f32(const GridP &g, const PartF32 &p, const Counters *cnt, float *const E[3],
                                 float *const B[3], float *const J[3], int *err, cudaStream_t s)
{
    const CylP cp = cyl_params(g);
    k_cyl_move_f32<<<kSMs * 8, kThreads, 0, s>>>(g, cp, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2],
                                                 err);
    k_cyl_axis_current<float><<<dim3((g.my + 127) / 128, g.mz), 128, 0, s>>>(g, J[0], J[1], J[2]);
    count_launches(2);
}

void launch_cyl_move_deposit_f32_tiled(const GridP &g, const PartF32 &p, const Bricks &bk, float *const E[3],
                                       float *const B[3], float *const J[3], int *err, cudaStream_t s)
{
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_cyl_move_f32_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
        attr_set = true;
    }
    const CylP cp = cyl_params(g);
    // the queue of near-axis slots: the brick-id scratch of the reorder, its
    // length in the scan scratch (both free between reorders)
    cudaMemsetAsync(bk.count, 0, sizeof(uint32_t), s);
    k_cyl_move_f32_tiled<<<bk.ntiles, kTileThreads, bk.smem_floats * 4, s>>>(g, cp, p, bk, E[0], E[1], E[2], B[0],
                                                                            B[1], B[2], J[0], J[1], J[2], err);
    k_cyl_substep_f32<<<kSMs * 4, kThreads, 0, s>>>(g, cp, p, bk.bid, bk.count, E[0], E[1], E[2], B[0], B[1], B[2],
                                                   J[0], J[1], J[2], err);
    k_cyl_axis_current<float><<<dim3((g.my + 127) / 128, g.mz), 128, 0, s>>>(g, J[0], J[1], J[2]);
    count_launches(3);
}

}  // namespace pic
