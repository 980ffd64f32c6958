// field_math.cuh -- device functions of the field solver, shared by the
// field kernels (fields.cu) and the persistent ensemble step (mover_f32.cu):
// the Yee and Lehe stencils, the periodic images a thread writes, the
// current fold and AddCurrent.  See fields.cu for the design and the
// reference routines.
#pragma once

#include "common.cuh"

namespace pic {

template <typename T>
struct Coef {
    T h, fc;
    T L[12];
    __host__ __device__ Coef() {}
    __host__ __device__ explicit Coef(const GridP &g) : h((T)g.h), fc((T)g.fc)
    {
        for (int i = 0; i < 12; i++) L[i] = (T)g.lehe[i];
    }
};

// Ghost image along one axis of an interior index a (0 = none).
__device__ __forceinline__ int image_of(int a, int m)
{
    const int n = m - 5;
    if (a <= 5) return a + n;      // 3..5 -> m-2..m
    if (a >= m - 4) return a - n;  // m-4..m-3 -> 1..2
    return 0;
}

// Image along x: none in the slab form, whose x ghosts the neighbouring
// slabs fill (SendRecvFlds / UpdateCurrentAllFaces across ranks).
__device__ __forceinline__ int image_x(const GridP &g, int i) { return g.x_external ? 0 : image_of(i, g.mx); }

// Write v to interior cell (i,j,k) and all of its periodic ghost images.
template <typename T, int DIMS>
__device__ __forceinline__ void store_with_images(const GridP &g, T *F, int i, int j, int k, T v)
{
    const int ii[2] = {i, image_x(g, i)};
    const int jj[2] = {j, image_of(j, g.my)};
    const int kk[2] = {k, DIMS == 3 ? image_of(k, g.mz) : 0};
#pragma unroll
    for (int c = 0; c < (DIMS == 3 ? 2 : 1); c++) {
        if (kk[c] == 0) continue;
#pragma unroll
        for (int b = 0; b < 2; b++) {
            if (jj[b] == 0) continue;
#pragma unroll
            for (int a = 0; a < 2; a++) {
                if (ii[a] == 0) continue;
                F[cidx(g, ii[a], jj[b], kk[c])] = v;
            }
        }
    }
}

template <typename T>
__device__ __forceinline__ T ld(const T *p) { return ldro(p); }

// ---------------------------------------------------------------------------
// Lehe directional differences, em_update_lehe.F90:223-258 (inv_d = 1).
// ---------------------------------------------------------------------------
template <typename T, int DIMS>
__device__ __forceinline__ T gradX(const GridP &g, const Coef<T> &C, const T *F, long long c0)
{
    const long long sy = g.sy, sz = g.sz;
    T r = C.L[0] * (ld(F + c0 + 1) - ld(F + c0));
    r = r + C.L[3] * (ld(F + c0 + 1 + sy) - ld(F + c0 + sy));
    r = r + C.L[3] * (ld(F + c0 + 1 - sy) - ld(F + c0 - sy));
    if (DIMS == 3) {
        r = r + C.L[4] * (ld(F + c0 + 1 + sz) - ld(F + c0 + sz));
        r = r + C.L[4] * (ld(F + c0 + 1 - sz) - ld(F + c0 - sz));
    }
    r = r + C.L[9] * (ld(F + c0 + 2) - ld(F + c0 - 1));
    return r;
}

template <typename T, int DIMS>
__device__ __forceinline__ T gradY(const GridP &g, const Coef<T> &C, const T *F, long long c0)
{
    const long long sy = g.sy, sz = g.sz;
    T r = C.L[1] * (ld(F + c0 + sy) - ld(F + c0));
    r = r + C.L[5] * (ld(F + c0 + 1 + sy) - ld(F + c0 + 1));
    r = r + C.L[5] * (ld(F + c0 - 1 + sy) - ld(F + c0 - 1));
    if (DIMS == 3) {
        r = r + C.L[6] * (ld(F + c0 + sy + sz) - ld(F + c0 + sz));
        r = r + C.L[6] * (ld(F + c0 + sy - sz) - ld(F + c0 - sz));
    }
    r = r + C.L[10] * (ld(F + c0 + 2 * sy) - ld(F + c0 - sy));
    return r;
}

template <typename T>
__device__ __forceinline__ T gradZ(const GridP &g, const Coef<T> &C, const T *F, long long c0)
{
    const long long sy = g.sy, sz = g.sz;
    T r = C.L[2] * (ld(F + c0 + sz) - ld(F + c0));
    r = r + C.L[7] * (ld(F + c0 + 1 + sz) - ld(F + c0 + 1));
    r = r + C.L[7] * (ld(F + c0 - 1 + sz) - ld(F + c0 - 1));
    r = r + C.L[8] * (ld(F + c0 + sy + sz) - ld(F + c0 + sy));
    r = r + C.L[8] * (ld(F + c0 - sy + sz) - ld(F + c0 - sy));
    r = r + C.L[11] * (ld(F + c0 + 2 * sz) - ld(F + c0 - sz));
    return r;
}

struct CellIter {
    int i, j, k;
    bool ok;
};

// Interior cell of thread (tx, ty) (default: threadIdx.x, threadIdx.y of a
// (32, 8) block) in block (bx, by, bz) of the (32, 8) tiling of the interior.
template <int DIMS>
__device__ __forceinline__ CellIter interior_cell_at(const GridP &g, int bx, int by, int bz, int tx, int ty)
{
    CellIter it;
    it.i = 3 + bx * 32 + tx;
    it.j = 3 + by * 8 + ty;
    it.k = DIMS == 3 ? 3 + bz : 1;
    it.ok = it.i <= g.mx - 3 && it.j <= g.my - 3;
    return it;
}
template <int DIMS>
__device__ __forceinline__ CellIter interior_cell_at(const GridP &g, int bx, int by, int bz)
{
    return interior_cell_at<DIMS>(g, bx, by, bz, (int)threadIdx.x, (int)threadIdx.y);
}
template <int DIMS>
__device__ __forceinline__ CellIter interior_cell(const GridP &g)
{
    return interior_cell_at<DIMS>(g, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// B <- B - (c/2) curl E (UpdateBfieldHalf) + halo (SendRecvFlds(B)).
// ---------------------------------------------------------------------------
template <typename T, int DIMS, int FDTD>
__device__ __forceinline__ void bhalf_at(const GridP &g, const CellIter &it, const T *__restrict__ Ex,
                                         const T *__restrict__ Ey, const T *__restrict__ Ez, T *Bx, T *By, T *Bz)
{
    if (!it.ok) return;
    const Coef<T> C(g);
    const T h = C.h;
    const long long c0 = cidx(g, it.i, it.j, it.k);
    const long long sy = g.sy, sz = g.sz;
    T bx, by, bz;
    if (FDTD == PIC_FDTD_YEE) {  // em_update.F90:65-72
        if (DIMS == 3) {
            bx = (ldco(Bx + c0) - h * (ld(Ez + c0 + sy) - ld(Ez + c0))) + h * (ld(Ey + c0 + sz) - ld(Ey + c0));
            by = (ldco(By + c0) - h * (ld(Ex + c0 + sz) - ld(Ex + c0))) + h * (ld(Ez + c0 + 1) - ld(Ez + c0));
            bz = (ldco(Bz + c0) - h * (ld(Ey + c0 + 1) - ld(Ey + c0))) + h * (ld(Ex + c0 + sy) - ld(Ex + c0));
        } else {
            bx = ldco(Bx + c0) - h * (ld(Ez + c0 + sy) - ld(Ez + c0));
            by = ldco(By + c0) + h * (ld(Ez + c0 + 1) - ld(Ez + c0));
            bz = (ldco(Bz + c0) - h * (ld(Ey + c0 + 1) - ld(Ey + c0))) + h * (ld(Ex + c0 + sy) - ld(Ex + c0));
        }
    } else {  // em_update_lehe.F90:209-216
        if (DIMS == 3) {
            bx = (ldco(Bx + c0) - h * gradY<T, 3>(g, C, Ez, c0)) + h * gradZ<T>(g, C, Ey, c0);
            by = (ldco(By + c0) - h * gradZ<T>(g, C, Ex, c0)) + h * gradX<T, 3>(g, C, Ez, c0);
            bz = (ldco(Bz + c0) - h * gradX<T, 3>(g, C, Ey, c0)) + h * gradY<T, 3>(g, C, Ex, c0);
        } else {
            bx = ldco(Bx + c0) - h * gradY<T, 2>(g, C, Ez, c0);
            by = ldco(By + c0) + h * gradX<T, 2>(g, C, Ez, c0);
            bz = (ldco(Bz + c0) - h * gradX<T, 2>(g, C, Ey, c0)) + h * gradY<T, 2>(g, C, Ex, c0);
        }
    }
    store_with_images<T, DIMS>(g, Bx, it.i, it.j, it.k, bx);
    store_with_images<T, DIMS>(g, By, it.i, it.j, it.k, by);
    store_with_images<T, DIMS>(g, Bz, it.i, it.j, it.k, bz);
}


// Yee E update of one cell (em_update.F90:27-34; Lehe keeps it, em_update_lehe.F90:174-181).
template <typename T, int DIMS>
__device__ __forceinline__ void e_curl(const GridP &g, T fc, const T *Ex, const T *Ey, const T *Ez, const T *Bx,
                                       const T *By, const T *Bz, long long c0, T &ex, T &ey, T &ez)
{
    const long long sy = g.sy, sz = g.sz;
    if (DIMS == 3) {
        ex = (ldco(Ex + c0) + fc * (ld(Bz + c0) - ld(Bz + c0 - sy))) - fc * (ld(By + c0) - ld(By + c0 - sz));
        ey = (ldco(Ey + c0) + fc * (ld(Bx + c0) - ld(Bx + c0 - sz))) - fc * (ld(Bz + c0) - ld(Bz + c0 - 1));
        ez = (ldco(Ez + c0) + fc * (ld(By + c0) - ld(By + c0 - 1))) - fc * (ld(Bx + c0) - ld(Bx + c0 - sy));
    } else {
        ex = ldco(Ex + c0) + fc * (ld(Bz + c0) - ld(Bz + c0 - sy));
        ey = ldco(Ey + c0) - fc * (ld(Bz + c0) - ld(Bz + c0 - 1));
        ez = (ldco(Ez + c0) + fc * (ld(By + c0) - ld(By + c0 - 1))) - fc * (ld(Bx + c0) - ld(Bx + c0 - sy));
    }
}

// Fold partner along one axis of an interior index a (0 = none), see image_of.
// J1 = J + J(x-partner); J2 = J1 + J1(y-partner); J3 = J2 + J2(z-partner):
// the order of comm_fld.F90:15-33 (x faces, then y, then z).  Loads only.
template <typename T, int DIMS>
__device__ __forceinline__ T fold_cell(const GridP &g, const T *__restrict__ J, int i, int j, int k)
{
    const int pi = image_x(g, i), pj = image_of(j, g.my);
    const int pk = DIMS == 3 ? image_of(k, g.mz) : 0;
    auto J1 = [&](int b, int c) -> T {
        T v = ldco(J + cidx(g, i, b, c));
        if (pi) v = v + ldco(J + cidx(g, pi, b, c));
        return v;
    };
    auto J2 = [&](int c) -> T {
        T v = J1(j, c);
        if (pj) v = v + J1(pj, c);
        return v;
    };
    T v = J2(k);
    if (DIMS == 3 && pk) v = v + J2(pk);
    return v;
}

// Zero the J cells fold_cell read (ResetCurrent of the consumed current).
template <typename T, int DIMS>
__device__ __forceinline__ void zero_fold_cells(const GridP &g, T *__restrict__ J, int i, int j, int k)
{
    const int ii[2] = {i, image_x(g, i)};
    const int jj[2] = {j, image_of(j, g.my)};
    const int kk[2] = {k, DIMS == 3 ? image_of(k, g.mz) : 0};
#pragma unroll
    for (int c = 0; c < (DIMS == 3 ? 2 : 1); c++) {
        if (kk[c] == 0) continue;
#pragma unroll
        for (int b = 0; b < 2; b++) {
            if (jj[b] == 0) continue;
#pragma unroll
            for (int a = 0; a < 2; a++) {
                if (ii[a] == 0) continue;
                J[cidx(g, ii[a], jj[b], kk[c])] = (T)0;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// E <- E + c curl B (UpdateEfield) [- fold(J) (AddCurrent)] + halo.
// MODE 0: curl only; 1: curl + fold + AddCurrent, zeroing J; 2: AddCurrent of
// an already folded J alone (phase API); 3: curl + AddCurrent of an already
// folded (and filtered) J.  Every load of a thread precedes its stores, so
// the loads of a thread are in flight together (an interleaved load, zero,
// load sequence on J serialised the memory latency).
// ---------------------------------------------------------------------------
template <typename T, int DIMS, int MODE>
__device__ __forceinline__ void efield_at(const GridP &g, const CellIter &it, T *__restrict__ Ex, T *__restrict__ Ey,
                                          T *__restrict__ Ez, const T *__restrict__ Bx, const T *__restrict__ By,
                                          const T *__restrict__ Bz, T *__restrict__ Jx, T *__restrict__ Jy,
                                          T *__restrict__ Jz)
{
    if (!it.ok) return;
    const long long c0 = cidx(g, it.i, it.j, it.k);
    T ex, ey, ez, jx = (T)0, jy = (T)0, jz = (T)0;
    if (MODE == 2) {
        ex = ldco(Ex + c0);
        ey = ldco(Ey + c0);
        ez = ldco(Ez + c0);
    } else {
        e_curl<T, DIMS>(g, (T)g.fc, Ex, Ey, Ez, Bx, By, Bz, c0, ex, ey, ez);
    }
    if (MODE == 1) {
        jx = fold_cell<T, DIMS>(g, Jx, it.i, it.j, it.k);
        jy = fold_cell<T, DIMS>(g, Jy, it.i, it.j, it.k);
        jz = fold_cell<T, DIMS>(g, Jz, it.i, it.j, it.k);
    } else if (MODE == 2 || MODE == 3) {
        jx = ldco(Jx + c0);
        jy = ldco(Jy + c0);
        jz = ldco(Jz + c0);
    }
    if (MODE != 0) {  // em_update.F90:96-98 with grid_inv_d = 1
        ex = ex - (jx * (T)1) * (T)1;
        ey = ey - (jy * (T)1) * (T)1;
        ez = ez - (jz * (T)1) * (T)1;
    }
    store_with_images<T, DIMS>(g, Ex, it.i, it.j, it.k, ex);
    store_with_images<T, DIMS>(g, Ey, it.i, it.j, it.k, ey);
    store_with_images<T, DIMS>(g, Ez, it.i, it.j, it.k, ez);
    if (MODE == 1) {
        zero_fold_cells<T, DIMS>(g, Jx, it.i, it.j, it.k);
        zero_fold_cells<T, DIMS>(g, Jy, it.i, it.j, it.k);
        zero_fold_cells<T, DIMS>(g, Jz, it.i, it.j, it.k);
    }
}

}  // namespace pic
