// pml.cu -- the convolutional PML of the reference (src/bc/bc_pml.F90) on
// the device, FP64 or FP32 fields, Cartesian single domain.
//
// The reference updates, after the second B half step (UpdateMagFld_PML,
// bc_pml.F90:146-264) and after the E update (UpdateElcFld_PML, :83-144),
// every cell of i, j, k = 2..m-1 that is not strictly inside the box of
// pml_pos_ind: two auxiliary fields per component (pml_*_psi1/2) relax
// towards the curl terms with the coefficients a, b of pml_ab, the field gets
// the psi difference and the kappa term c of pml_c, and any component beyond
// the layers (pos -+ thickness) is zeroed.  SendRecvFlds follows both
// (MAIN.F90:104-110).
//
// Design: the coefficients depend on one coordinate each, so the host builds
// them once per axis (a, b, c at the integer and at the half-integer
// positions, and the interior / beyond-the-layer flags) with the same double
// arithmetic and libm exp the reference evaluates per cell; the kernels read
// three table rows per cell.  One thread per cell of the 2..m-1 box, in
// place: a cell's update reads only the other field (E for the B update, B
// for the E update) and its own psi entries, so the cells are independent.
// The halo that follows is one pass writing every ghost cell from its fully
// wrapped interior image (the single-rank SendRecvFlds of the field kernels).
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"

namespace pic {

namespace {

// The profile of the six faces: SetPMLParameters (bc_pml.F90:42-53) for a
// 'pml' face, the pml_params type defaults (:6-12) and +-huge(1) positions
// (:14-15) for the others; alpha_max is the default-kind literal 9.0e-4.
struct PmlProfile {
    double pos[6], ind[6], L[6], kmax[6], smax[6], amax[6];
    int n[6];
};

PmlProfile pml_profile(int faces, const double *pos, const double *thickness)
{
    PmlProfile q;
    const double huge = 2147483647.0;
    for (int f = 0; f < 6; f++) {
        const bool upper = (f & 1) != 0;
        q.n[f] = 4;
        q.kmax[f] = 1.0;
        if ((faces >> f) & 1) {
            q.L[f] = thickness[f];
            q.smax[f] = 1.0;
            q.amax[f] = (double)9.0e-4f;
            q.pos[f] = pos[f];
            q.ind[f] = upper ? std::ceil(pos[f]) + 1.0 : std::floor(pos[f]) - 1.0;   // Update_PML_Position
        } else {
            q.L[f] = 10.0;
            q.smax[f] = 0.0;
            q.amax[f] = 1.0;
            q.pos[f] = upper ? huge : -huge;
            q.ind[f] = upper ? huge : -huge;
        }
    }
    return q;
}

// x**n (n >= 0) by binary powering, the evaluation of a real to a variable
// integer power.
double powi(double x, int n)
{
    double y = (n & 1) ? x : 1.0;
    while (n >>= 1) {
        x = x * x;
        if (n & 1) y = y * x;
    }
    return y;
}

double kappa_of(const PmlProfile &q, double d, int f)   // pml_kappa
{
    const double k = 1.0 + powi(d / q.L[f], q.n[f]) * (q.kmax[f] - 1.0);
    return q.kmax[f] < k ? q.kmax[f] : k;
}

double sigma_of(const PmlProfile &q, double d, int f)   // pml_sigma
{
    const double s = q.smax[f] * powi(d / q.L[f], q.n[f]);
    return q.smax[f] < s ? q.smax[f] : s;
}

// a, b (pml_ab) and c (pml_c) at coordinate x of `axis`; the face beyond
// which x lies decides, the lower face last.
void coefficients(const PmlProfile &q, double fc, double x, int axis, double &a, double &b, double &c)
{
    a = b = c = 0.0;
    const int lo = 2 * axis, hi = lo + 1;
    for (int side = 0; side < 2; side++) {
        const int f = side == 0 ? hi : lo;
        if (side == 0 ? !(x > q.pos[hi]) : !(x < q.pos[lo])) continue;
        const double d = side == 0 ? x - q.pos[hi] : q.pos[lo] - x;
        const double alpha = q.amax[f], sigma = sigma_of(q, d, f), kappa = kappa_of(q, d, f);
        a = std::exp(-(sigma / kappa) - alpha);
        b = (sigma / (sigma * kappa + alpha * (kappa * kappa))) * (a - 1.0);
        c = fc * (1.0 / kappa - 1.0);
    }
}

bool beyond(const PmlProfile &q, double x, int axis)
{
    return x < q.pos[2 * axis] - q.L[2 * axis] || x > q.pos[2 * axis + 1] + q.L[2 * axis + 1];
}

template <typename T>
struct Psi {
    T *p[6];   // psi1 x, y, z, psi2 x, y, z
};

// coefficient row of 1-based index a of an axis: E (integer position) or B
// (half-integer position)
struct PmlRow {
    double a, b, c;
};
template <bool HALF>
__device__ __forceinline__ PmlRow pml_row(const PmlP &P, int axis, int a)
{
    const double *r = P.coef[axis] + 6 * (a - 1) + (HALF ? 3 : 0);
    return {ldro(r), ldro(r + 1), ldro(r + 2)};
}

// UpdateElcFld_PML (bc_pml.F90:83-144)
template <typename T, int DIMS>
__global__ void __launch_bounds__(kThreads) k_pml_e(GridP g, PmlP P, T *Ex, T *Ey, T *Ez, const T *__restrict__ Bx,
                                                    const T *__restrict__ By, const T *__restrict__ Bz, Psi<T> psi)
{
    const int ni = g.mx - 2, nj = g.my - 2, nk = DIMS == 3 ? g.mz - 2 : 1;
    const long long n = (long long)ni * nj * nk;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long r = t / ni;
        const int i = 2 + (int)(t - r * ni), j = 2 + (int)(r % nj), k = DIMS == 3 ? 2 + (int)(r / nj) : 1;
        const uint8_t fx = P.flag[0][i - 1], fy = P.flag[1][j - 1], fz = P.flag[2][k - 1];
        if (fx & fy & fz & kPmlInside) continue;
        const PmlRow X = pml_row<false>(P, 0, i), Y = pml_row<false>(P, 1, j), Z = pml_row<false>(P, 2, k);
        const T ax = (T)X.a, bx = (T)X.b, cx = (T)X.c, ay = (T)Y.a, by = (T)Y.b, cy = (T)Y.c;
        const T az = (T)Z.a, bz = (T)Z.b, cz = (T)Z.c, fc = (T)P.fc;
        const long long c = cidx(g, i, j, k), cxm = c - 1, cym = c - g.sy, czm = DIMS == 3 ? c - g.sz : c;
        T *p1x = psi.p[0], *p1y = psi.p[1], *p1z = psi.p[2], *p2x = psi.p[3], *p2y = psi.p[4], *p2z = psi.p[5];
        const T dBz_y = Bz[c] - Bz[cym], dBy_x = By[c] - By[cxm], dBz_x = Bz[c] - Bz[cxm], dBx_y = Bx[c] - Bx[cym];
        p1x[c] = ay * p1x[c] + (by * fc) * dBz_y;
        p1z[c] = ax * p1z[c] + (bx * fc) * dBy_x;
        T dBx_z = (T)0, dBy_z = (T)0;
        if (DIMS == 3) {
            dBx_z = Bx[c] - Bx[czm];
            dBy_z = By[c] - By[czm];
            p1y[c] = az * p1y[c] + (bz * fc) * dBx_z;
            p2x[c] = az * p2x[c] + (bz * fc) * dBy_z;
        }
        p2y[c] = ax * p2y[c] + (bx * fc) * dBz_x;
        p2z[c] = ay * p2z[c] + (by * fc) * dBx_y;
        T ex, ey;
        if (DIMS == 3) {
            ex = ((Ex[c] + cy * dBz_y) - cz * dBy_z) + p1x[c] - p2x[c];
            ey = ((Ey[c] + cz * dBx_z) - cx * dBz_x) + p1y[c] - p2y[c];
        } else {
            ex = (Ex[c] + cy * dBz_y) + p1x[c];
            ey = (Ey[c] - cx * dBz_x) - p2y[c];
        }
        const T ez = ((Ez[c] + cx * dBy_x) - cy * dBx_y) + p1z[c] - p2z[c];
        Ex[c] = ((fx & kPmlBeyondHalf) | ((fy | fz) & kPmlBeyond)) ? (T)0 : ex;
        Ey[c] = ((fy & kPmlBeyondHalf) | ((fx | fz) & kPmlBeyond)) ? (T)0 : ey;
        Ez[c] = ((fz & kPmlBeyondHalf) | ((fx | fy) & kPmlBeyond)) ? (T)0 : ez;
    }
}

// UpdateMagFld_PML (bc_pml.F90:146-264): coefficients at the half-integer
// positions, the component of each axis zeroed by its integer position.
template <typename T, int DIMS>
__global__ void __launch_bounds__(kThreads) k_pml_b(GridP g, PmlP P, const T *__restrict__ Ex,
                                                    const T *__restrict__ Ey, const T *__restrict__ Ez, T *Bx, T *By,
                                                    T *Bz, Psi<T> psi)
{
    const int ni = g.mx - 2, nj = g.my - 2, nk = DIMS == 3 ? g.mz - 2 : 1;
    const long long n = (long long)ni * nj * nk;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const long long r = t / ni;
        const int i = 2 + (int)(t - r * ni), j = 2 + (int)(r % nj), k = DIMS == 3 ? 2 + (int)(r / nj) : 1;
        const uint8_t fx = P.flag[0][i - 1], fy = P.flag[1][j - 1], fz = P.flag[2][k - 1];
        if (fx & fy & fz & kPmlInside) continue;
        const PmlRow X = pml_row<true>(P, 0, i), Y = pml_row<true>(P, 1, j), Z = pml_row<true>(P, 2, k);
        const T ax = (T)X.a, bx = (T)X.b, cx = (T)X.c, ay = (T)Y.a, by = (T)Y.b, cy = (T)Y.c;
        const T az = (T)Z.a, bz = (T)Z.b, cz = (T)Z.c, fc = (T)P.fc;
        const long long c = cidx(g, i, j, k), cxp = c + 1, cyp = c + g.sy, czp = DIMS == 3 ? c + g.sz : c;
        T *p1x = psi.p[0], *p1y = psi.p[1], *p1z = psi.p[2], *p2x = psi.p[3], *p2y = psi.p[4], *p2z = psi.p[5];
        const T dEz_y = Ez[cyp] - Ez[c], dEy_x = Ey[cxp] - Ey[c], dEz_x = Ez[cxp] - Ez[c], dEx_y = Ex[cyp] - Ex[c];
        p1x[c] = ay * p1x[c] + (by * fc) * dEz_y;
        p1z[c] = ax * p1z[c] + (bx * fc) * dEy_x;
        T dEx_z = (T)0, dEy_z = (T)0;
        if (DIMS == 3) {
            dEx_z = Ex[czp] - Ex[c];
            dEy_z = Ey[czp] - Ey[c];
            p1y[c] = az * p1y[c] + (bz * fc) * dEx_z;
            p2x[c] = az * p2x[c] + (bz * fc) * dEy_z;
        }
        p2y[c] = ax * p2y[c] + (bx * fc) * dEz_x;
        p2z[c] = ay * p2z[c] + (by * fc) * dEx_y;
        T bxn, byn;
        if (DIMS == 3) {
            bxn = ((Bx[c] - cy * dEz_y) + cz * dEy_z) - p1x[c] + p2x[c];
            byn = ((By[c] - cz * dEx_z) + cx * dEz_x) - p1y[c] + p2y[c];
        } else {
            bxn = (Bx[c] - cy * dEz_y) - p1x[c];
            byn = (By[c] + cx * dEz_x) + p2y[c];
        }
        const T bzn = ((Bz[c] - cx * dEy_x) + cy * dEx_y) - p1z[c] + p2z[c];
        Bx[c] = ((fx & kPmlBeyond) | ((fy | fz) & kPmlBeyondHalf)) ? (T)0 : bxn;
        By[c] = ((fy & kPmlBeyond) | ((fx | fz) & kPmlBeyondHalf)) ? (T)0 : byn;
        Bz[c] = ((fz & kPmlBeyond) | ((fx | fy) & kPmlBeyondHalf)) ? (T)0 : bzn;
    }
}

// Every ghost cell from its fully wrapped interior image (SendRecvFlds on one
// periodic rank, whatever the order of its axes).
template <typename T, int DIMS>
__global__ void __launch_bounds__(kThreads) k_halo3(GridP g, T *F0, T *F1, T *F2)
{
    const long long n = g.ncell;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const long long jk = c / g.mx;
        const int i = (int)(c - jk * g.mx) + 1, j = (int)(jk % g.my) + 1, k = (int)(jk / g.my) + 1;
        const int wi = wrap_index(i, g.mx), wj = wrap_index(j, g.my), wk = DIMS == 3 ? wrap_index(k, g.mz) : k;
        if (wi == i && wj == j && wk == k) continue;
        const long long s = cidx(g, wi, wj, wk);
        F0[c] = F0[s];
        F1[c] = F1[s];
        F2[c] = F2[s];
    }
}

int pml_grid(long long n)
{
    const long long b = (n + kThreads - 1) / kThreads;
    return (int)(b < kSMs * 8 ? (b > 0 ? b : 1) : kSMs * 8);
}

}  // namespace

bool pml_tables(const GridP &g, int faces, const double *pos, const double *thickness, double *coef, uint8_t *flag)
{
    const PmlProfile q = pml_profile(faces, pos, thickness);
    const int m[3] = {g.mx, g.my, g.mz};
    // no_pml_this_domain (bc_pml.F90:67-69) with the borders of one rank at 0
    const bool none = 1 - 3 > q.ind[0] && g.mx - 3 < q.ind[1] && 1 - 3 > q.ind[2] && g.my - 3 < q.ind[3] &&
                      1 - 3 > q.ind[4] && g.mz - 3 < q.ind[5];
    int o = 0;
    for (int axis = 0; axis < 3; axis++) {
        for (int a = 1; a <= m[axis]; a++, o++) {
            const double x = (double)(a - 3), xh = x + 0.5;
            coefficients(q, g.fc, x, axis, coef[6 * o], coef[6 * o + 1], coef[6 * o + 2]);
            coefficients(q, g.fc, xh, axis, coef[6 * o + 3], coef[6 * o + 4], coef[6 * o + 5]);
            uint8_t f = 0;
            if (x > q.ind[2 * axis] && x < q.ind[2 * axis + 1]) f |= kPmlInside;
            if (beyond(q, x, axis)) f |= kPmlBeyond;
            if (beyond(q, xh, axis)) f |= kPmlBeyondHalf;
            flag[o] = f;
        }
    }
    return !none;
}

template <typename T>
void launch_pml(const GridP &g, const PmlP &P, int which, T *const E[3], T *const B[3], T *const psi[6], cudaStream_t s)
{
    Psi<T> ps;
    for (int c = 0; c < 6; c++) ps.p[c] = psi[c];
    const long long n = (long long)(g.mx - 2) * (g.my - 2) * (g.dims == 3 ? g.mz - 2 : 1);
    const int grid = pml_grid(n);
    if (which == 0) {
        if (g.dims == 3)
            k_pml_b<T, 3><<<grid, kThreads, 0, s>>>(g, P, E[0], E[1], E[2], B[0], B[1], B[2], ps);
        else
            k_pml_b<T, 2><<<grid, kThreads, 0, s>>>(g, P, E[0], E[1], E[2], B[0], B[1], B[2], ps);
    } else {
        if (g.dims == 3)
            k_pml_e<T, 3><<<grid, kThreads, 0, s>>>(g, P, E[0], E[1], E[2], B[0], B[1], B[2], ps);
        else
            k_pml_e<T, 2><<<grid, kThreads, 0, s>>>(g, P, E[0], E[1], E[2], B[0], B[1], B[2], ps);
    }
    T *const *F = which == 0 ? B : E;
    if (g.dims == 3)
        k_halo3<T, 3><<<pml_grid(g.ncell), kThreads, 0, s>>>(g, F[0], F[1], F[2]);
    else
        k_halo3<T, 2><<<pml_grid(g.ncell), kThreads, 0, s>>>(g, F[0], F[1], F[2]);
    count_launches(2);
}

template void launch_pml<double>(const GridP &, const PmlP &, int, double *const[3], double *const[3],
                                 double *const[6], cudaStream_t);
template void launch_pml<float>(const GridP &, const PmlP &, int, float *const[3], float *const[3], float *const[6],
                                cudaStream_t);

}  // namespace pic
