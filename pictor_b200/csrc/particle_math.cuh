// particle_math.cuh -- device helpers shared by the Cartesian and the
// cylindrical movers: node-averaged gather, interpolation weights, the
// relativistic Boris rotation, the zigzag segment weights and their scatter.
#pragma once

#include "common.cuh"

namespace pic {


// Node-averaged field components at the 4 (2D) / 8 (3D) corners of the cell
// whose lower corner is at offset c0, interpolated with weights wt[]
// (GatherVecEfld/GatherVecBfld + movdep.F90:116-129).
template <typename T, int DIMS>
__device__ __forceinline__ void gather(const GridP &g, const T *__restrict__ Ex, const T *__restrict__ Ey,
                                       const T *__restrict__ Ez, const T *__restrict__ Bx, const T *__restrict__ By,
                                       const T *__restrict__ Bz, long long c0, const T *wt, T pE[3], T pB[3])
{
    const long long sy = g.sy, sz = g.sz;
    const T half = (T)0.5, quarter = (T)0.25;
    const T b0 = (T)g.bext[0], b1 = (T)g.bext[1], b2 = (T)g.bext[2];
    pE[0] = pE[1] = pE[2] = pB[0] = pB[1] = pB[2] = (T)0;
#pragma unroll
    for (int nn = 0; nn < (DIMS == 3 ? 8 : 4); nn++) {
        const long long nd = c0 + (nn & 1) + ((nn >> 1) & 1) * sy + ((nn >> 2) & 1) * sz;
        const T vex = (__ldg(Ex + nd - 1) + __ldg(Ex + nd)) * half;
        const T vey = (__ldg(Ey + nd - sy) + __ldg(Ey + nd)) * half;
        T vez, vbx, vby;
        if (DIMS == 3) {
            vez = (__ldg(Ez + nd - sz) + __ldg(Ez + nd)) * half;
            vbx = (((__ldg(Bx + nd - sy - sz) + __ldg(Bx + nd - sz)) + __ldg(Bx + nd - sy)) + __ldg(Bx + nd)) * quarter + b0;
            vby = (((__ldg(By + nd - 1 - sz) + __ldg(By + nd - 1)) + __ldg(By + nd - sz)) + __ldg(By + nd)) * quarter + b1;
        } else {
            vez = __ldg(Ez + nd);
            vbx = (__ldg(Bx + nd - sy) + __ldg(Bx + nd)) * half + b0;
            vby = (__ldg(By + nd - 1) + __ldg(By + nd)) * half + b1;
        }
        const T vbz = (((__ldg(Bz + nd - 1 - sy) + __ldg(Bz + nd - 1)) + __ldg(Bz + nd - sy)) + __ldg(Bz + nd)) * quarter + b2;
        pE[0] = pE[0] + wt[nn] * vex;
        pE[1] = pE[1] + wt[nn] * vey;
        pE[2] = pE[2] + wt[nn] * vez;
        pB[0] = pB[0] + wt[nn] * vbx;
        pB[1] = pB[1] + wt[nn] * vby;
        pB[2] = pB[2] + wt[nn] * vbz;
    }
}

// Interpolation weights (vars.F90:323-326, 339-344): corner nn uses
// (1-d) for a 0 bit and d for a 1 bit of nn, multiplied x, y, z left to right.
template <typename T, int DIMS>
__device__ __forceinline__ void weights(T dx, T dy, T dz, T *wt)
{
#pragma unroll
    for (int nn = 0; nn < (DIMS == 3 ? 8 : 4); nn++) {
        const T wx = (nn & 1) ? ((T)0 + (T)1 * dx) : ((T)1 + (T)-1 * dx);
        const T wy = (nn & 2) ? ((T)0 + (T)1 * dy) : ((T)1 + (T)-1 * dy);
        if (DIMS == 3) {
            const T wz = (nn & 4) ? ((T)0 + (T)1 * dz) : ((T)1 + (T)-1 * dz);
            wt[nn] = (wx * wy) * wz;
        } else {
            wt[nn] = wx * wy;
        }
    }
}

// Relativistic Boris rotation, movdep.F90:143-167.  On entry u,v,w hold
// gamma*v/c; pE, pB are already scaled by q/m * 0.5.  Returns the new
// momenta (u,v,w) and g = c^2/sqrt(c^2+|c u|^2).
template <typename T>
__device__ __forceinline__ void boris(T c, T sqc, T cinv, const T pE[3], const T pB[3], T &u, T &v, T &w, T &gout)
{
    T u0 = c * u + pE[0];
    T v0 = c * v + pE[1];
    T w0 = c * w + pE[2];
    const T gg = (T)1 / sqrt(((sqc + u0 * u0) + v0 * v0) + w0 * w0);
    const T bx = gg * pB[0], by = gg * pB[1], bz = gg * pB[2];
    const T ff = (T)2 / ((((T)1 + bx * bx) + by * by) + bz * bz);
    const T u1 = ((u0 + v0 * bz) - w0 * by) * ff;
    const T v1 = ((v0 + w0 * bx) - u0 * bz) * ff;
    const T w1 = ((w0 + u0 * by) - v0 * bx) * ff;
    u0 = ((u0 + v1 * bz) - w1 * by) + pE[0];
    v0 = ((v0 + w1 * bx) - u1 * bz) + pE[1];
    w0 = ((w0 + u1 * by) - v1 * bx) + pE[2];
    u = u0 * cinv;
    v = v0 * cinv;
    w = w0 * cinv;
    gout = sqc / sqrt(((sqc + u0 * u0) + v0 * v0) + w0 * w0);
}

// The 8 (2D) / 12 (3D) VecJ entries of one zigzag segment
// (movdep.F90:209,233 with the tables of vars.F90:328-355 expanded).
template <typename T, int DIMS>
__device__ __forceinline__ void segment(T Fx, T Fy, T Fz, T Wx, T Wy, T Wz, T *o)
{
    if (DIMS == 2) {
        o[0] = ((Fx * (T)1) * ((T)1 - Wy)) * (T)1;
        o[1] = ((Fx * (T)1) * Wy) * (T)1;
        o[2] = ((Fy * ((T)1 - Wx)) * (T)1) * (T)1;
        o[3] = ((Fy * Wx) * (T)1) * (T)1;
        o[4] = ((Fz * ((T)1 - Wx)) * ((T)1 - Wy)) * (T)1;
        o[5] = ((Fz * Wx) * ((T)1 - Wy)) * (T)1;
        o[6] = ((Fz * ((T)1 - Wx)) * Wy) * (T)1;
        o[7] = ((Fz * Wx) * Wy) * (T)1;
    } else {
        o[0] = ((Fx * (T)1) * ((T)1 - Wy)) * ((T)1 - Wz);
        o[1] = ((Fx * (T)1) * Wy) * ((T)1 - Wz);
        o[2] = ((Fx * (T)1) * ((T)1 - Wy)) * Wz;
        o[3] = ((Fx * (T)1) * Wy) * Wz;
        o[4] = ((Fy * ((T)1 - Wx)) * (T)1) * ((T)1 - Wz);
        o[5] = ((Fy * Wx) * (T)1) * ((T)1 - Wz);
        o[6] = ((Fy * ((T)1 - Wx)) * (T)1) * Wz;
        o[7] = ((Fy * Wx) * (T)1) * Wz;
        o[8] = ((Fz * ((T)1 - Wx)) * ((T)1 - Wy)) * (T)1;
        o[9] = ((Fz * Wx) * ((T)1 - Wy)) * (T)1;
        o[10] = ((Fz * ((T)1 - Wx)) * Wy) * (T)1;
        o[11] = ((Fz * Wx) * Wy) * (T)1;
    }
}

// Scatter of VecJ entries onto the cell edges, movdep_routines.F90:276-303.
template <typename T, int DIMS>
__device__ __forceinline__ void scatter(const GridP &g, T *Jx, T *Jy, T *Jz, long long c0, const T *o)
{
    const long long sy = g.sy, sz = g.sz;
    if (DIMS == 2) {
        atomicAdd(Jx + c0, o[0]);
        atomicAdd(Jx + c0 + sy, o[1]);
        atomicAdd(Jy + c0, o[2]);
        atomicAdd(Jy + c0 + 1, o[3]);
        atomicAdd(Jz + c0, o[4]);
        atomicAdd(Jz + c0 + 1, o[5]);
        atomicAdd(Jz + c0 + sy, o[6]);
        atomicAdd(Jz + c0 + 1 + sy, o[7]);
    } else {
        atomicAdd(Jx + c0, o[0]);
        atomicAdd(Jx + c0 + sy, o[1]);
        atomicAdd(Jx + c0 + sz, o[2]);
        atomicAdd(Jx + c0 + sy + sz, o[3]);
        atomicAdd(Jy + c0, o[4]);
        atomicAdd(Jy + c0 + 1, o[5]);
        atomicAdd(Jy + c0 + sz, o[6]);
        atomicAdd(Jy + c0 + 1 + sz, o[7]);
        atomicAdd(Jz + c0, o[8]);
        atomicAdd(Jz + c0 + 1, o[9]);
        atomicAdd(Jz + c0 + sy, o[10]);
        atomicAdd(Jz + c0 + 1 + sy, o[11]);
    }
}

}  // namespace pic
