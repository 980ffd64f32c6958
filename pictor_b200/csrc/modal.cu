// modal.cu -- the cylindrical field solve truncated to azimuthal modes m = 0, 1.
//
// The reference's theta-gridded field update (cyl_em_update.F90 and
// cyl_em_update_lehe.F90, restated in cyl.cu) is linear and invariant under
// shifts of the theta index on its ny periodic cells: every theta difference
// couples F(j) with F(j +- 1), the axis conditions couple F(j) with the
// partner F(j + ny/2) (cyl_em_update.F90:143-227), and the Bz axis update
// sums over all j (:231-246).  So it acts on each discrete Fourier mode of
// theta separately.  This form keeps m = 0 and m = 1 only: a component is
//
//     F(i, t, k) = a(i, k) + b(i, k) cos(phi t) + c(i, k) sin(phi t),
//     t = j - 3 (theta index), phi = 2 pi / ny,
//
// stored as three planes (a, b, c) of an (mx, 3, mz) array, and every update
// of cyl.cu is applied to the planes with the theta shifts written as
// rotations of (b, c):
//     F(t + 1) -> (a,  b cos(phi) + c sin(phi),  c cos(phi) - b sin(phi))
//     F(t - 1) -> (a,  b cos(phi) - c sin(phi),  c cos(phi) + b sin(phi))
//     F(t + ny/2) -> (a, -b, -c).
// On fields whose theta content is m <= 1 the result equals the
// theta-gridded update to round-off.  The particles keep the reference's
// theta-gridded mover: the theta-gridded E and B it gathers from are
// synthesised from the modes after every field update, and the current it
// deposits (after the fold) is projected onto the modes before AddCurrent.
// The projection of a charge-conserving current is charge-conserving mode by
// mode (the continuity equation is theta-shift invariant), so the truncated
// run keeps the theta-gridded scheme's Gauss law for m = 0, 1.
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"

namespace pic {

struct ModalP {
    double cphi, sphi;    // cos / sin of 2 pi / ny
    double dtheta, ax_perm_area, rmin;
    int ny;
};

// Three planes of one component at (i, k); T = double or float (the FP32 form).
template <typename T>
struct M3 {
    T a, b, c;
};

template <typename T>
__device__ __forceinline__ M3<T> operator+(M3<T> x, M3<T> y) { return {x.a + y.a, x.b + y.b, x.c + y.c}; }
template <typename T>
__device__ __forceinline__ M3<T> operator-(M3<T> x, M3<T> y) { return {x.a - y.a, x.b - y.b, x.c - y.c}; }
template <typename T>
__device__ __forceinline__ M3<T> operator*(T s, M3<T> x) { return {s * x.a, s * x.b, s * x.c}; }
template <typename T>
__device__ __forceinline__ M3<T> operator/(M3<T> x, T s) { return {x.a / s, x.b / s, x.c / s}; }

// modal grid: the theta dimension holds the planes a, b, c (j = 1, 2, 3)
template <typename T>
__device__ __forceinline__ M3<T> ld3(const GridP &gm, const T *F, int i, int k)
{
    const long long c0 = cidx(gm, i, 1, k);
    return {F[c0], F[c0 + gm.sy], F[c0 + 2 * gm.sy]};
}
template <typename T>
__device__ __forceinline__ void st3(const GridP &gm, T *F, int i, int k, M3<T> v)
{
    const long long c0 = cidx(gm, i, 1, k);
    F[c0] = v.a;
    F[c0 + gm.sy] = v.b;
    F[c0 + 2 * gm.sy] = v.c;
}
// F(t + 1), F(t - 1), F(t + ny/2)
template <typename T>
__device__ __forceinline__ M3<T> tp(const ModalP &m, M3<T> v)
{
    const T cp = (T)m.cphi, sp = (T)m.sphi;
    return {v.a, v.b * cp + v.c * sp, v.c * cp - v.b * sp};
}
template <typename T>
__device__ __forceinline__ M3<T> tm(const ModalP &m, M3<T> v)
{
    const T cp = (T)m.cphi, sp = (T)m.sphi;
    return {v.a, v.b * cp - v.c * sp, v.c * cp + v.b * sp};
}
template <typename T>
__device__ __forceinline__ M3<T> partner(M3<T> v) { return {v.a, -v.b, -v.c}; }

// Lehe directional differences (cyl_em_update_lehe.F90:255-289) on modes.
template <typename T>
__device__ __forceinline__ M3<T> mgx(const GridP &gm, const T *F, int i, int k)
{
    const double *L = gm.lehe;
    M3<T> r = (T)L[0] * (ld3(gm, F, i + 1, k) - ld3(gm, F, i, k));
    r = r + (T)L[4] * (ld3(gm, F, i + 1, k + 1) - ld3(gm, F, i, k + 1));
    r = r + (T)L[4] * (ld3(gm, F, i + 1, k - 1) - ld3(gm, F, i, k - 1));
    return r;
}
template <typename T>
__device__ __forceinline__ M3<T> mgx1(const GridP &gm, const T *F, int i, int k, T rp, T rr)
{
    const double *L = gm.lehe;
    M3<T> r = (T)L[0] * (rp * ld3(gm, F, i + 1, k) - rr * ld3(gm, F, i, k));
    r = r + (T)L[4] * (rp * ld3(gm, F, i + 1, k + 1) - rr * ld3(gm, F, i, k + 1));
    r = r + (T)L[4] * (rp * ld3(gm, F, i + 1, k - 1) - rr * ld3(gm, F, i, k - 1));
    return r;
}
template <typename T>
__device__ __forceinline__ M3<T> mgy(const GridP &gm, const ModalP &m, const T *F, int i, int k)
{
    const double *L = gm.lehe;
    const M3<T> f0 = ld3(gm, F, i, k), fp = ld3(gm, F, i, k + 1), fm = ld3(gm, F, i, k - 1);
    M3<T> r = (T)L[1] * (tp(m, f0) - f0);
    r = r + (T)L[6] * (tp(m, fp) - fp);
    r = r + (T)L[6] * (tp(m, fm) - fm);
    return r;
}
template <typename T>
__device__ __forceinline__ M3<T> mgz(const GridP &gm, const ModalP &m, const T *F, int i, int k)
{
    const double *L = gm.lehe;
    const M3<T> dz0 = ld3(gm, F, i, k + 1) - ld3(gm, F, i, k);
    M3<T> r = (T)L[2] * dz0;
    r = r + (T)L[7] * (ld3(gm, F, i + 1, k + 1) - ld3(gm, F, i + 1, k));
    r = r + (T)L[7] * (ld3(gm, F, i - 1, k + 1) - ld3(gm, F, i - 1, k));
    r = r + (T)L[8] * tp(m, dz0);
    r = r + (T)L[8] * tm(m, dz0);
    r = r + (T)L[11] * (ld3(gm, F, i, k + 2) - ld3(gm, F, i, k - 1));
    return r;
}

// B half step (cyl_em_update.F90:66-83; Lehe :62-118): i 4..mx-1, k 1..mz-1
// (Lehe 2..mz-2).
template <typename T, int FDTD>
__global__ void k_modal_bhalf(GridP gm, ModalP m, const T *__restrict__ Ex, const T *__restrict__ Ey,
                              const T *__restrict__ Ez, T *Bx, T *By, T *Bz)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = (FDTD == PIC_FDTD_LEHE ? 2 : 1) + blockIdx.y;
    if (i > gm.mx - 1) return;
    const T h = (T)gm.h, dtheta = (T)m.dtheta;
    const T r = ((T)i - (T)3.0) + (T)m.rmin;
    const T rp_half = r + (T)0.5, rp = r + (T)1.0;
    if (FDTD == PIC_FDTD_YEE) {
        const M3<T> ez = ld3(gm, Ez, i, k), ex = ld3(gm, Ex, i, k), ey = ld3(gm, Ey, i, k);
        const M3<T> bx = ld3(gm, Bx, i, k) - (h * (tp(m, ez) - ez)) / (r * dtheta) + h * (ld3(gm, Ey, i, k + 1) - ey);
        const M3<T> by = ld3(gm, By, i, k) - h * (ld3(gm, Ex, i, k + 1) - ex) + h * (ld3(gm, Ez, i + 1, k) - ez);
        const M3<T> bz = ld3(gm, Bz, i, k) - (h * ((rp * ld3(gm, Ey, i + 1, k) - r * ey) - (tp(m, ex) - ex) / dtheta)) / rp_half;
        st3(gm, Bx, i, k, bx);
        st3(gm, By, i, k, by);
        st3(gm, Bz, i, k, bz);
    } else {
        const M3<T> bx = ld3(gm, Bx, i, k) - (h * mgy(gm, m, Ez, i, k)) / (r * dtheta) + h * mgz(gm, m, Ey, i, k);
        const M3<T> by = ld3(gm, By, i, k) - h * mgz(gm, m, Ex, i, k) + h * mgx(gm, Ez, i, k);
        const M3<T> bz = ld3(gm, Bz, i, k) - (h * (mgx1(gm, Ey, i, k, rp, r) - mgy(gm, m, Ex, i, k) / dtheta)) / rp_half;
        st3(gm, Bx, i, k, bx);
        st3(gm, By, i, k, by);
        st3(gm, Bz, i, k, bz);
    }
}

// UpdateBzAxis (cyl_em_update.F90:231-246): the circulation of Ey(4, :, k)
// is ny times its m = 0 plane; Bz on the axis has no m = 1 part.
template <typename T>
__global__ void k_modal_bz_axis(GridP gm, ModalP m, const T *__restrict__ Ey, T *Bz)
{
    const int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (k > gm.mz - 1) return;
    const T s = -(T)(gm.h * m.ax_perm_area) * ((T)m.ny * ld3(gm, Ey, 4, k).a);
    st3<T>(gm, Bz, 3, k, {ld3(gm, Bz, 3, k).a + s, (T)0, (T)0});
}

// UpdateBFldAxis / UpdateEFldAxis (cyl_em_update.F90:143-227) on modes.
template <typename T>
__global__ void k_modal_b_axis(GridP gm, T *Bx, T *By, T *Bz)
{
    const int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (k > gm.mz) return;
    const M3<T> by4 = ld3(gm, By, 4, k), bx4 = ld3(gm, Bx, 4, k), bz4 = ld3(gm, Bz, 4, k);
    st3(gm, By, 3, k, (T)0.5 * (by4 - partner(by4)));
    st3<T>(gm, By, 2, k, {-by4.a, by4.b, by4.c});
    st3<T>(gm, Bx, 3, k, {-bx4.a, bx4.b, bx4.c});
    st3(gm, Bz, 2, k, partner(bz4));
}
template <typename T>
__global__ void k_modal_e_axis(GridP gm, T *Ex, T *Ey, T *Ez)
{
    const int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (k > gm.mz) return;
    const M3<T> ex4 = ld3(gm, Ex, 4, k), ey4 = ld3(gm, Ey, 4, k), ez4 = ld3(gm, Ez, 4, k);
    st3(gm, Ex, 3, k, (T)0.5 * (ex4 - partner(ex4)));
    st3<T>(gm, Ex, 2, k, {-ex4.a, ex4.b, ex4.c});
    st3<T>(gm, Ey, 3, k, {-ey4.a, ey4.b, ey4.c});
    st3(gm, Ez, 3, k, partner(ez4));
}

// UpdateEfield (MODE 0, cyl_em_update.F90:24-41) or AddCurrent (MODE 2,
// :128-137) on modes: i 4..mx-3, k 3..mz-3.
template <typename T, int MODE>
__global__ void k_modal_e(GridP gm, ModalP m, T *Ex, T *Ey, T *Ez, const T *__restrict__ Bx, const T *__restrict__ By,
                          const T *__restrict__ Bz, const T *__restrict__ Jx, const T *__restrict__ Jy,
                          const T *__restrict__ Jz)
{
    const int i = 4 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 3 + blockIdx.y;
    if (i > gm.mx - 3) return;
    const T dtheta = (T)m.dtheta;
    const T r = ((T)i - (T)3.0) + (T)m.rmin;
    const T rp_half = r + (T)0.5, rm_half = r - (T)0.5;
    if (MODE == 0) {
        const T fc = (T)gm.fc;
        const M3<T> bz = ld3(gm, Bz, i, k), by = ld3(gm, By, i, k), bx = ld3(gm, Bx, i, k);
        st3(gm, Ex, i, k, ld3(gm, Ex, i, k) + (fc * (bz - tm(m, bz))) / (rp_half * dtheta) - fc * (by - ld3(gm, By, i, k - 1)));
        st3(gm, Ey, i, k, ld3(gm, Ey, i, k) + fc * (bx - ld3(gm, Bx, i, k - 1)) - fc * (bz - ld3(gm, Bz, i - 1, k)));
        st3(gm, Ez, i, k,
            ld3(gm, Ez, i, k) + (fc * (rp_half * by - rm_half * ld3(gm, By, i - 1, k))) / r - (fc * (bx - tm(m, bx))) / (r * dtheta));
    } else {
        st3(gm, Ex, i, k, ld3(gm, Ex, i, k) - ld3(gm, Jx, i, k) / (rp_half * dtheta));
        st3(gm, Ey, i, k, ld3(gm, Ey, i, k) - ld3(gm, Jy, i, k));
        st3(gm, Ez, i, k, ld3(gm, Ez, i, k) - ld3(gm, Jz, i, k) / (r * dtheta));
    }
}

// Periodic z halo of the modal planes (the layer map of cyl.cu's halo).
template <typename T>
__global__ void k_modal_halo_z(GridP gm, T *F)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int p = 1 + blockIdx.y;
    if (i > gm.mx) return;
    const int mz = gm.mz;
    for (int l = 0; l < 3; l++) F[cidx(gm, i, p, mz - 2 + l)] = F[cidx(gm, i, p, 3 + l)];
    for (int l = 0; l < 2; l++) F[cidx(gm, i, p, 1 + l)] = F[cidx(gm, i, p, mz - 4 + l)];
}

// Theta-gridded F(i, j, k) for every ghosted j from the modes at (i, k).
template <typename T>
__global__ void k_modal_synth(GridP g, GridP gm, ModalP m, const T *__restrict__ Fm, T *F)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 1 + blockIdx.y;
    if (i > g.mx) return;
    const M3<T> v = ld3(gm, Fm, i, k);
    for (int j = 1; j <= g.my; j++) {
        int t = (j - 3) % m.ny;
        if (t < 0) t += m.ny;
        double sn, cs;
        sincospi(2.0 * (double)t / (double)m.ny, &sn, &cs);
        F[cidx(g, i, j, k)] = v.a + v.b * (T)cs + v.c * (T)sn;
    }
}

// Modes of the theta-gridded F over its ny interior theta cells:
// a = mean, b = 2/ny sum F cos, c = 2/ny sum F sin (summed in FP64).
template <typename T>
__global__ void k_modal_project(GridP g, GridP gm, ModalP m, const T *__restrict__ F, T *Fm)
{
    const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    const int k = 1 + blockIdx.y;
    if (i > g.mx) return;
    double a = 0.0, b = 0.0, c = 0.0;
    for (int t = 0; t < m.ny; t++) {
        const double v = (double)F[cidx(g, i, 3 + t, k)];
        double sn, cs;
        sincospi(2.0 * (double)t / (double)m.ny, &sn, &cs);
        a += v;
        b += v * cs;
        c += v * sn;
    }
    const double inv = 1.0 / (double)m.ny;
    st3<T>(gm, Fm, i, k, {(T)(a * inv), (T)(2.0 * b * inv), (T)(2.0 * c * inv)});
}

GridP modal_grid(const GridP &g)
{
    GridP gm = g;
    gm.my = 3;
    gm.sy = g.mx;
    gm.sz = (long long)g.mx * 3;
    gm.ncell = gm.sz * g.mz;
    return gm;
}

static ModalP modal_params(const GridP &g)
{
    ModalP m;
    const double pi = 3.14159265358979323846264;
    m.ny = g.ny;
    m.dtheta = 2.0 * pi / g.ny;
    m.cphi = std::cos(m.dtheta);
    m.sphi = std::sin(m.dtheta);
    m.ax_perm_area = 4.0 / g.ny;
    m.rmin = -0.5;
    return m;
}

template <typename T>
static void modal_halo(const GridP &gm, T *const F[3], cudaStream_t s)
{
    for (int c = 0; c < 3; c++) k_modal_halo_z<T><<<dim3((gm.mx + 127) / 128, 3), 128, 0, s>>>(gm, F[c]);
    count_launches(3);
}

template <typename T>
void launch_modal_bhalf(const GridP &g, T *const Em[3], T *const Bm[3], cudaStream_t s)
{
    const GridP gm = modal_grid(g);
    const ModalP m = modal_params(g);
    const int nk = g.fdtd == PIC_FDTD_LEHE ? g.mz - 3 : g.mz - 1;
    const dim3 grid((g.mx - 4 + 127) / 128, nk);
    if (g.fdtd == PIC_FDTD_LEHE)
        k_modal_bhalf<T, PIC_FDTD_LEHE><<<grid, 128, 0, s>>>(gm, m, Em[0], Em[1], Em[2], Bm[0], Bm[1], Bm[2]);
    else
        k_modal_bhalf<T, PIC_FDTD_YEE><<<grid, 128, 0, s>>>(gm, m, Em[0], Em[1], Em[2], Bm[0], Bm[1], Bm[2]);
    k_modal_bz_axis<T><<<(g.mz + 127) / 128, 128, 0, s>>>(gm, m, Em[1], Bm[2]);
    k_modal_b_axis<T><<<(g.mz + 127) / 128, 128, 0, s>>>(gm, Bm[0], Bm[1], Bm[2]);
    count_launches(3);
    modal_halo<T>(gm, Bm, s);
}

template <typename T>
void launch_modal_efield(const GridP &g, int mode, T *const Em[3], T *const Bm[3], T *const Jm[3], cudaStream_t s)
{
    const GridP gm = modal_grid(g);
    const ModalP m = modal_params(g);
    const dim3 grid((g.mx - 6 + 127) / 128, g.mz - 5);
    if (mode == 0)
        k_modal_e<T, 0><<<grid, 128, 0, s>>>(gm, m, Em[0], Em[1], Em[2], Bm[0], Bm[1], Bm[2], Jm[0], Jm[1], Jm[2]);
    else
        k_modal_e<T, 2><<<grid, 128, 0, s>>>(gm, m, Em[0], Em[1], Em[2], Bm[0], Bm[1], Bm[2], Jm[0], Jm[1], Jm[2]);
    k_modal_e_axis<T><<<(g.mz + 127) / 128, 128, 0, s>>>(gm, Em[0], Em[1], Em[2]);
    count_launches(2);
    modal_halo<T>(gm, Em, s);
}

template <typename T>
void launch_modal_synth(const GridP &g, T *const Fm[3], T *const F[3], cudaStream_t s)
{
    const GridP gm = modal_grid(g);
    const ModalP m = modal_params(g);
    for (int c = 0; c < 3; c++) k_modal_synth<T><<<dim3((g.mx + 127) / 128, g.mz), 128, 0, s>>>(g, gm, m, Fm[c], F[c]);
    count_launches(3);
}

template <typename T>
void launch_modal_project(const GridP &g, T *const F[3], T *const Fm[3], cudaStream_t s)
{
    const GridP gm = modal_grid(g);
    const ModalP m = modal_params(g);
    for (int c = 0; c < 3; c++) k_modal_project<T><<<dim3((g.mx + 127) / 128, g.mz), 128, 0, s>>>(g, gm, m, F[c], Fm[c]);
    count_launches(3);
}

template void launch_modal_bhalf<double>(const GridP &, double *const[3], double *const[3], cudaStream_t);
template void launch_modal_bhalf<float>(const GridP &, float *const[3], float *const[3], cudaStream_t);
template void launch_modal_efield<double>(const GridP &, int, double *const[3], double *const[3], double *const[3],
                                          cudaStream_t);
template void launch_modal_efield<float>(const GridP &, int, float *const[3], float *const[3], float *const[3],
                                         cudaStream_t);
template void launch_modal_synth<double>(const GridP &, double *const[3], double *const[3], cudaStream_t);
template void launch_modal_synth<float>(const GridP &, float *const[3], float *const[3], cudaStream_t);
template void launch_modal_project<double>(const GridP &, double *const[3], double *const[3], cudaStream_t);
template void launch_modal_project<float>(const GridP &, float *const[3], float *const[3], cudaStream_t);

}  // namespace pic
