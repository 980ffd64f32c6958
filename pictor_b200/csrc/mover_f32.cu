// mover_f32.cu -- the FP32 cell-relative mover: gather, relativistic Boris
// push, zigzag current deposit and periodic wrap, fused in one kernel.
//
// Reference: src/movdep/movdep.F90:12-258 (the per-particle algorithm),
// src/movdep/movdep_routines.F90:6-223 (node-averaged fields VecE/VecB),
// src/movdep/movdep_gpu.F90:56-334 (the reference's CUDA Fortran kernel),
// weight tables vars.F90:322-356.
//
// Particles carry key = (flv << 28) | ghosted linear cell and offsets in
// [0,1) from the cell's lower corner, so FP32 keeps full sub-cell resolution
// anywhere in the box and the periodic wrap is an integer update of the cell.
//
// Tiled form (after a reorder): particles are grouped by brick (a block of
// TX x TY x TZ interior cells, see bricks.cu) and one CTA moves one brick's
// particles.  The CTA stages the node-averaged E and B of its box in shared
// memory (each node value computed once per brick rather than 8 times per
// particle), accumulates the current of the box in shared memory, and adds
// the box to J once.  The box is the bounding box, in cells, of where the
// brick's particles were after the previous step (particles drift away from
// their brick between reorders); it is stored per brick relative to the
// brick's centre, unwrapped across the periodic boundary, and this kernel
// writes the box for the next step.  A box too large for shared memory falls
// back to the brick itself plus one cell; particles outside the box gather
// and deposit through global memory with the same arithmetic.  Box currents
// go straight to the periodic interior image of each cell.
//
// The node averages and interpolation sums are computed identically on both
// paths (same expressions, same order, explicit fmaf), so the tiled and the
// per-particle kernels move particles bit-identically; currents differ only
// in the order of the FP32 atomic sums.
#include "common.cuh"
#include "kernels.cuh"

namespace pic {

// Node-averaged fields at node offset nd (GatherVecEfld / GatherVecBfld,
// movdep_routines.F90:6-223): E averaged over the 2 edges, B over the 4 faces
// meeting at the node (2 in 2D), plus the external field.
template <int DIMS>
__device__ __forceinline__ void node_avg(const float *__restrict__ Ex, const float *__restrict__ Ey,
                                         const float *__restrict__ Ez, const float *__restrict__ Bx,
                                         const float *__restrict__ By, const float *__restrict__ Bz, long long nd,
                                         long long sy, long long sz, float b0, float b1, float b2, float4 &A,
                                         float2 &Bv)
{
    A.x = (__ldg(Ex + nd - 1) + __ldg(Ex + nd)) * 0.5f;
    A.y = (__ldg(Ey + nd - sy) + __ldg(Ey + nd)) * 0.5f;
    if (DIMS == 3) {
        A.z = (__ldg(Ez + nd - sz) + __ldg(Ez + nd)) * 0.5f;
        A.w = (((__ldg(Bx + nd - sy - sz) + __ldg(Bx + nd - sz)) + __ldg(Bx + nd - sy)) + __ldg(Bx + nd)) * 0.25f + b0;
        Bv.x = (((__ldg(By + nd - 1 - sz) + __ldg(By + nd - 1)) + __ldg(By + nd - sz)) + __ldg(By + nd)) * 0.25f + b1;
    } else {
        A.z = __ldg(Ez + nd);
        A.w = (__ldg(Bx + nd - sy) + __ldg(Bx + nd)) * 0.5f + b0;
        Bv.x = (__ldg(By + nd - 1) + __ldg(By + nd)) * 0.5f + b1;
    }
    Bv.y = (((__ldg(Bz + nd - 1 - sy) + __ldg(Bz + nd - 1)) + __ldg(Bz + nd - sy)) + __ldg(Bz + nd)) * 0.25f + b2;
}

__device__ __forceinline__ void accum(float w, const float4 &A, const float2 &Bv, float pE[3], float pB[3])
{
    pE[0] = fmaf(w, A.x, pE[0]);
    pE[1] = fmaf(w, A.y, pE[1]);
    pE[2] = fmaf(w, A.z, pE[2]);
    pB[0] = fmaf(w, A.w, pB[0]);
    pB[1] = fmaf(w, Bv.x, pB[1]);
    pB[2] = fmaf(w, Bv.y, pB[2]);
}

// Interpolation weights of the 4 / 8 corners (corner bit 0 = x, 1 = y, 2 = z).
template <int DIMS>
__device__ __forceinline__ void weights_f32(float dx, float dy, float dz, float wt[8])
{
    const float wx[2] = {1.f - dx, dx}, wy[2] = {1.f - dy, dy};
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const float xy = wx[c & 1] * wy[c >> 1];
        if (DIMS == 3) {
            wt[c] = xy * (1.f - dz);
            wt[c + 4] = xy * dz;
        } else {
            wt[c] = xy;
        }
    }
}

// Relativistic Boris rotation (movdep.F90:143-167) in FP32 with hardware
// reciprocal square root.  On entry u,v,w = gamma v / c and pE, pB are
// scaled by q/m * 0.5; returns new momenta and gg = c^2/sqrt(c^2 + |c u|^2).
__device__ __forceinline__ void boris_f32(float c, float sqc, float cinv, const float pE[3], const float pB[3],
                                          float &u, float &v, float &w, float &gout)
{
    float u0 = fmaf(c, u, pE[0]);
    float v0 = fmaf(c, v, pE[1]);
    float w0 = fmaf(c, w, pE[2]);
    const float gg = rsqrtf(fmaf(w0, w0, fmaf(v0, v0, fmaf(u0, u0, sqc))));
    const float bx = gg * pB[0], by = gg * pB[1], bz = gg * pB[2];
    const float ff = __fdividef(2.f, fmaf(bz, bz, fmaf(by, by, fmaf(bx, bx, 1.f))));
    const float u1 = fmaf(-w0, by, fmaf(v0, bz, u0)) * ff;
    const float v1 = fmaf(-u0, bz, fmaf(w0, bx, v0)) * ff;
    const float w1 = fmaf(-v0, bx, fmaf(u0, by, w0)) * ff;
    u0 = fmaf(-w1, by, fmaf(v1, bz, u0)) + pE[0];
    v0 = fmaf(-u1, bz, fmaf(w1, bx, v0)) + pE[1];
    w0 = fmaf(-v1, bx, fmaf(u1, by, w0)) + pE[2];
    u = u0 * cinv;
    v = v0 * cinv;
    w = w0 * cinv;
    gout = sqc * rsqrtf(fmaf(w0, w0, fmaf(v0, v0, fmaf(u0, u0, sqc))));
}

// VecJ entries of one zigzag segment (movdep.F90:209,233 with the tables of
// vars.F90:328-355): flux F, segment midpoint W within its cell.
template <int DIMS>
__device__ __forceinline__ void segment_f32(float Fx, float Fy, float Fz, float Wx, float Wy, float Wz, float *o)
{
    if (DIMS == 2) {
        o[0] = Fx * (1.f - Wy);
        o[1] = Fx * Wy;
        o[2] = Fy * (1.f - Wx);
        o[3] = Fy * Wx;
        const float a = Fz * (1.f - Wx), b = Fz * Wx;
        o[4] = a * (1.f - Wy);
        o[5] = b * (1.f - Wy);
        o[6] = a * Wy;
        o[7] = b * Wy;
    } else {
        const float xa = Fx * (1.f - Wy), xb = Fx * Wy;
        o[0] = xa * (1.f - Wz);
        o[1] = xb * (1.f - Wz);
        o[2] = xa * Wz;
        o[3] = xb * Wz;
        const float ya = Fy * (1.f - Wx), yb = Fy * Wx;
        o[4] = ya * (1.f - Wz);
        o[5] = yb * (1.f - Wz);
        o[6] = ya * Wz;
        o[7] = yb * Wz;
        const float za = Fz * (1.f - Wx), zb = Fz * Wx;
        o[8] = za * (1.f - Wy);
        o[9] = zb * (1.f - Wy);
        o[10] = za * Wy;
        o[11] = zb * Wy;
    }
}

// Scatter of one segment's entries at base offset c0 of an array with row
// stride sy and plane stride sz (movdep_routines.F90:276-303); A = atomics on
// global or shared memory alike.
template <int DIMS>
__device__ __forceinline__ void scatter_f32(float *Jx, float *Jy, float *Jz, long long c0, long long sy, long long sz,
                                            const float *o)
{
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

// Interior index 3..n+2 of a periodic (unwrapped) 1-based index a.
__device__ __forceinline__ int wrap_interior(int a, int n)
{
    int t = (a - 3) % n;
    if (t < 0) t += n;
    return 3 + t;
}

// Unwrapped offset of interior index i from centre hc on a periodic axis of
// n cells: the representative of (i - hc) mod n in [-n/2, n - n/2).
__device__ __forceinline__ int unwrap_offset(int i, int hc, int n)
{
    int u = i - hc;
    const int half = n >> 1;
    if (u >= n - half) u -= n;
    else if (u < -half) u += n;
    return u;
}

// Shared-memory view of a tile's box (unused by the per-particle kernel).
struct TileBox {
    const float4 *nA;   // node E x,y,z, B x
    const float2 *nB;   // node B y,z
    float *sJ;          // current box, 3 planar components
    int hc[3];          // brick centre (1-based interior indices)
    int lo[3];          // box lower corner, cells relative to hc
    int C[3];           // box extent in cells (1 on the unused z axis of 2D)
    int NX, NXY;        // node box strides
    int JX, JXY, njc;   // current box strides and size
};

// Running bounds of the particles' new cells (relative to the brick centre).
struct Bounds {
    int lo[3], hi[3];
    __device__ void init()
    {
        for (int d = 0; d < 3; d++) {
            lo[d] = 0x3fffffff;
            hi[d] = -0x3fffffff;
        }
    }
};

// Move one particle.  TILED: gather/deposit through the tile box when the
// particle's cell is inside it; otherwise (and always when !TILED) through the
// global arrays at the particle's wrapped cell.
template <int DIMS, bool TILED>
__device__ __forceinline__ void push_one(const GridP &g, const PartF32 &p, uint32_t n, const float *__restrict__ Ex,
                                         const float *__restrict__ Ey, const float *__restrict__ Ez,
                                         const float *__restrict__ Bx, const float *__restrict__ By,
                                         const float *__restrict__ Bz, float *Jx, float *Jy, float *Jz, int *err,
                                         const TileBox &tb, Bounds &bd)
{
    const uint32_t key = p.key[n];
    const int flv = (int)(key >> kFlvShift);
    if (flv == 0) return;
    const int cell = (int)(key & kCellMask);
    int i, j, k;
    decode_cell(g, cell, i, j, k);
    if (i < 3 || i > g.mx - 3 || j < 3 || j > g.my - 3 || (DIMS == 3 && (k < 3 || k > g.mz - 3)) ||
        (DIMS == 2 && k != 1)) {
        raise_error(err, PIC_DEVERR_RANGE);
        return;
    }
    const float dx = p.dx[n], dy = p.dy[n], dz = DIMS == 3 ? p.dz[n] : 0.f;
    float wt[8];
    weights_f32<DIMS>(dx, dy, dz, wt);
    const long long sy = g.sy, sz = g.sz;
    int uo[3] = {0, 0, 0};   // unwrapped offsets from the brick centre
    bool inside = false;
    int nb = 0;
    if (TILED) {
        uo[0] = unwrap_offset(i, tb.hc[0], g.nx);
        uo[1] = unwrap_offset(j, tb.hc[1], g.ny);
        if (DIMS == 3) uo[2] = unwrap_offset(k, tb.hc[2], g.nz);
        const int lx = uo[0] - tb.lo[0], ly = uo[1] - tb.lo[1], lz = DIMS == 3 ? uo[2] - tb.lo[2] : 0;
        inside = (unsigned)lx < (unsigned)tb.C[0] && (unsigned)ly < (unsigned)tb.C[1] &&
                 (DIMS == 2 || (unsigned)lz < (unsigned)tb.C[2]);
        nb = lx + tb.NX * ly + tb.NXY * lz;
    }
    float pE[3] = {0.f, 0.f, 0.f}, pB[3] = {0.f, 0.f, 0.f};
    if (inside) {
#pragma unroll
        for (int c8 = 0; c8 < (DIMS == 3 ? 8 : 4); c8++) {
            const int q = nb + (c8 & 1) + ((c8 >> 1) & 1) * tb.NX + ((c8 >> 2) & 1) * tb.NXY;
            accum(wt[c8], tb.nA[q], tb.nB[q], pE, pB);
        }
    } else {
        const float b0 = (float)g.bext[0], b1 = (float)g.bext[1], b2 = (float)g.bext[2];
#pragma unroll
        for (int c8 = 0; c8 < (DIMS == 3 ? 8 : 4); c8++) {
            const long long nd = (long long)cell + (c8 & 1) + ((c8 >> 1) & 1) * sy + ((c8 >> 2) & 1) * sz;
            float4 A;
            float2 Bv;
            node_avg<DIMS>(Ex, Ey, Ez, Bx, By, Bz, nd, sy, sz, b0, b1, b2, A, Bv);
            accum(wt[c8], A, Bv, pE, pB);
        }
    }
    const float qm = (float)g.qm[flv] * 0.5f;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        pE[d] *= qm;
        pB[d] *= qm;
    }
    float u = p.ux[n], v = p.uy[n], w = p.uz[n], gg;
    boris_f32((float)g.c, (float)g.sqc, (float)g.cinv, pE, pB, u, v, w, gg);
    // displacement in cell units, positions relative to this cell's corner
    const float x1 = fmaf(u, gg, dx), y1 = fmaf(v, gg, dy), z1 = DIMS == 3 ? fmaf(w, gg, dz) : 0.f;
    const int sxx = (int)floorf(x1), syy = (int)floorf(y1), szz = DIMS == 3 ? (int)floorf(z1) : 0;
    // zigzag relay point with ip0 = 0, ip = s (movdep.F90:183-185)
    const float xr = fminf((float)(min(0, sxx) + 1), fmaxf((float)max(0, sxx), 0.5f * (dx + x1)));
    const float yr = fminf((float)(min(0, syy) + 1), fmaxf((float)max(0, syy), 0.5f * (dy + y1)));
    const float qthis = p.w[n] * (float)g.qi;
    float Fz1, Fz2, Wz1 = 0.f, Wz2 = 0.f;
    if (DIMS == 3) {
        const float zr = fminf((float)(min(0, szz) + 1), fmaxf((float)max(0, szz), 0.5f * (dz + z1)));
        Fz1 = qthis * (zr - dz);
        Fz2 = qthis * (z1 - zr);
        Wz1 = 0.5f * (dz + zr);
        Wz2 = 0.5f * (z1 + zr) - (float)szz;
    } else {
        // out-of-plane motion: no cell crossing, the relay point is the midpoint
        Fz1 = qthis * (0.5f * (w * gg));
        Fz2 = Fz1;
    }
    float o1[12], o2[12];
    segment_f32<DIMS>(qthis * (xr - dx), qthis * (yr - dy), Fz1, 0.5f * (dx + xr), 0.5f * (dy + yr), Wz1, o1);
    segment_f32<DIMS>(qthis * (x1 - xr), qthis * (y1 - yr), Fz2, 0.5f * (x1 + xr) - (float)sxx,
                      0.5f * (y1 + yr) - (float)syy, Wz2, o2);
    const bool same = (sxx | syy | szz) == 0;
    if (inside) {
        const int lx = uo[0] - tb.lo[0], ly = uo[1] - tb.lo[1], lz = DIMS == 3 ? uo[2] - tb.lo[2] : 0;
        const int jb = (lx + 1) + tb.JX * (ly + 1) + (DIMS == 3 ? tb.JXY * (lz + 1) : 0);
        float *sJx = tb.sJ, *sJy = tb.sJ + tb.njc, *sJz = tb.sJ + 2 * tb.njc;
        if (same) {
#pragma unroll
            for (int e = 0; e < (DIMS == 3 ? 12 : 8); e++) o1[e] += o2[e];
            scatter_f32<DIMS>(sJx, sJy, sJz, jb, tb.JX, tb.JXY, o1);
        } else {
            scatter_f32<DIMS>(sJx, sJy, sJz, jb, tb.JX, tb.JXY, o1);
            scatter_f32<DIMS>(sJx, sJy, sJz, jb + sxx + syy * tb.JX + szz * tb.JXY, tb.JX, tb.JXY, o2);
        }
    } else {
        if (same) {
#pragma unroll
            for (int e = 0; e < (DIMS == 3 ? 12 : 8); e++) o1[e] += o2[e];
            scatter_f32<DIMS>(Jx, Jy, Jz, cell, sy, sz, o1);
        } else {
            scatter_f32<DIMS>(Jx, Jy, Jz, cell, sy, sz, o1);
            scatter_f32<DIMS>(Jx, Jy, Jz, (long long)cell + sxx + syy * sy + szz * sz, sy, sz, o2);
        }
    }
    // new offsets and periodic cell index
    float nx = x1 - (float)sxx, ny = y1 - (float)syy, nz = z1 - (float)szz;
    int ax = sxx, ay = syy, az = szz;
    if (nx >= 1.f) { nx -= 1.f; ax += 1; }
    if (ny >= 1.f) { ny -= 1.f; ay += 1; }
    if (DIMS == 3 && nz >= 1.f) { nz -= 1.f; az += 1; }
    if (TILED) {
        bd.lo[0] = min(bd.lo[0], uo[0] + ax); bd.hi[0] = max(bd.hi[0], uo[0] + ax);
        bd.lo[1] = min(bd.lo[1], uo[1] + ay); bd.hi[1] = max(bd.hi[1], uo[1] + ay);
        if (DIMS == 3) { bd.lo[2] = min(bd.lo[2], uo[2] + az); bd.hi[2] = max(bd.hi[2], uo[2] + az); }
    }
    const int ni = wrap_index(i + ax, g.mx), nj = wrap_index(j + ay, g.my);
    const int nk = DIMS == 3 ? wrap_index(k + az, g.mz) : 1;
    p.key[n] = ((uint32_t)flv << kFlvShift) | (uint32_t)((ni - 1) + g.mx * ((nj - 1) + g.my * (nk - 1)));
    p.dx[n] = nx;
    p.dy[n] = ny;
    if (DIMS == 3) p.dz[n] = nz;
    p.ux[n] = u;
    p.uy[n] = v;
    p.uz[n] = w;
}

// ---------------------------------------------------------------------------
// Per-particle form (before the first reorder): grid-stride over the array.
// ---------------------------------------------------------------------------
template <int DIMS>
__global__ void __launch_bounds__(kThreads) k_move_f32(GridP g, PartF32 p, const Counters *__restrict__ cnt,
                                                       const float *__restrict__ Ex, const float *__restrict__ Ey,
                                                       const float *__restrict__ Ez, const float *__restrict__ Bx,
                                                       const float *__restrict__ By, const float *__restrict__ Bz,
                                                       float *Jx, float *Jy, float *Jz, int *err)
{
    const long long used = cnt->used;
    TileBox tb = {};
    Bounds bd;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < used; n += (long long)gridDim.x * blockDim.x)
        push_one<DIMS, false>(g, p, (uint32_t)n, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, err, tb, bd);
}

void launch_move_deposit_f32(const GridP &g, const PartF32 &p, const Counters *cnt, float *const E[3],
                             float *const B[3], float *const J[3], int *err, cudaStream_t s)
{
    const int grid = kSMs * 16;
    if (g.dims == 3)
        k_move_f32<3><<<grid, kThreads, 0, s>>>(g, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2], err);
    else
        k_move_f32<2><<<grid, kThreads, 0, s>>>(g, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2], err);
    count_launches(1);
}

// ---------------------------------------------------------------------------
// Tiled form: one CTA per brick.
// ---------------------------------------------------------------------------
constexpr int kTileThreads = 256;
constexpr int kTileWarps = kTileThreads / 32;

// Shared floats a box of C cells needs: nodes (C+1) x 6 + current (C+3) x 3.
__host__ __device__ inline long long box_floats(int dims, int cx, int cy, int cz)
{
    const long long nn = (long long)(cx + 1) * (cy + 1) * (dims == 3 ? cz + 1 : 1);
    const long long nj = (long long)(cx + 3) * (cy + 3) * (dims == 3 ? cz + 3 : 1);
    return 6 * nn + 3 * nj;
}

template <int DIMS>
__global__ void __launch_bounds__(kTileThreads, 3)
    k_move_f32_tiled(GridP g, PartF32 p, Bricks bk, const float *__restrict__ Ex, const float *__restrict__ Ey,
                     const float *__restrict__ Ez, const float *__restrict__ Bx, const float *__restrict__ By,
                     const float *__restrict__ Bz, float *Jx, float *Jy, float *Jz, int *err)
{
    extern __shared__ __align__(16) float sm[];
    __shared__ int red[kTileWarps][6];
    const int b = blockIdx.x;
    const uint32_t p0 = bk.tile_start[b], p1 = bk.tile_start[b + 1];
    if (p0 >= p1) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // brick centre and home extent
    const int bx = b % bk.nb[0], byz = b / bk.nb[0], by = byz % bk.nb[1], bz = byz / bk.nb[1];
    const int n3[3] = {g.nx, g.ny, g.nz};
    const int bi[3] = {bx, by, bz};
    TileBox tb;
    int home_lo[3], home_hi[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const int lo = 3 + bi[d] * bk.t[d];
        const int hi = min(lo + bk.t[d] - 1, n3[d] + 2);
        tb.hc[d] = lo + (bk.t[d] >> 1);
        home_lo[d] = lo - tb.hc[d];
        home_hi[d] = hi - tb.hc[d];
    }
    if (DIMS == 2) {
        tb.hc[2] = 1;
        home_lo[2] = home_hi[2] = 0;
    }
    // box of this step: the stored bounds, or the brick +- 1 cell if too large
    const int *sb = bk.box + 8 * (size_t)b;
    int lo[3] = {sb[0], sb[1], DIMS == 3 ? sb[2] : 0}, hi[3] = {sb[3], sb[4], DIMS == 3 ? sb[5] : 0};
    if (hi[0] < lo[0] || hi[1] < lo[1] || hi[2] < lo[2] ||
        box_floats(DIMS, hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1) > bk.smem_floats) {
#pragma unroll
        for (int d = 0; d < DIMS; d++) {
            lo[d] = home_lo[d] - 1;
            hi[d] = home_hi[d] + 1;
        }
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        tb.lo[d] = lo[d];
        tb.C[d] = hi[d] - lo[d] + 1;
    }
    const int NX = tb.C[0] + 1, NY = tb.C[1] + 1, NZ = DIMS == 3 ? tb.C[2] + 1 : 1;
    const int JX = tb.C[0] + 3, JY = tb.C[1] + 3, JZ = DIMS == 3 ? tb.C[2] + 3 : 1;
    const int nnode = NX * NY * NZ;
    tb.NX = NX;
    tb.NXY = NX * NY;
    tb.JX = JX;
    tb.JXY = JX * JY;
    tb.njc = JX * JY * JZ;
    float4 *nA = reinterpret_cast<float4 *>(sm);
    float2 *nB = reinterpret_cast<float2 *>(sm + 4 * nnode);
    float *sJ = sm + 6 * nnode;
    tb.nA = nA;
    tb.nB = nB;
    tb.sJ = sJ;
    // stage node-averaged fields, one box row (fixed y,z) per warp pass
    {
        const long long sy = g.sy, sz = g.sz;
        const float b0 = (float)g.bext[0], b1 = (float)g.bext[1], b2 = (float)g.bext[2];
        for (int r = warp; r < NY * NZ; r += kTileWarps) {
            const int yy = r % NY, zz = r / NY;
            const int bj = wrap_interior(tb.hc[1] + lo[1] + yy, g.ny);
            const int ck = DIMS == 3 ? wrap_interior(tb.hc[2] + lo[2] + zz, g.nz) : 1;
            const long long row = cidx(g, 1, bj, ck);
            for (int xx = lane; xx < NX; xx += 32) {
                const int ai = wrap_interior(tb.hc[0] + lo[0] + xx, g.nx);
                float4 A;
                float2 Bv;
                node_avg<DIMS>(Ex, Ey, Ez, Bx, By, Bz, row + (ai - 1), sy, sz, b0, b1, b2, A, Bv);
                nA[r * NX + xx] = A;
                nB[r * NX + xx] = Bv;
            }
        }
    }
    for (int q = tid; q < 3 * tb.njc; q += kTileThreads) sJ[q] = 0.f;
    __syncthreads();

    Bounds bd;
    bd.init();
    for (uint32_t n = p0 + tid; n < p1; n += kTileThreads)
        push_one<DIMS, true>(g, p, n, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, err, tb, bd);
    __syncthreads();

    // add the box current to the periodic interior image of each cell
    {
        const int rows = JY * JZ;
        for (int r = warp; r < 3 * rows; r += kTileWarps) {
            const int comp = r / rows, rr = r - comp * rows;
            const int yy = rr % JY, zz = rr / JY;
            const int bj = wrap_interior(tb.hc[1] + lo[1] - 1 + yy, g.ny);
            const int ck = DIMS == 3 ? wrap_interior(tb.hc[2] + lo[2] - 1 + zz, g.nz) : 1;
            float *J = comp == 0 ? Jx : comp == 1 ? Jy : Jz;
            const long long row = cidx(g, 1, bj, ck);
            const float *src = sJ + (size_t)comp * tb.njc + (size_t)rr * JX;
            for (int xx = lane; xx < JX; xx += 32) {
                const float val = src[xx];
                if (val != 0.f) atomicAdd(J + row + (wrap_interior(tb.hc[0] + lo[0] - 1 + xx, g.nx) - 1), val);
            }
        }
    }
    // bounds of the new cells -> box of the next step (the brick itself if empty)
    int v[6] = {bd.lo[0], bd.lo[1], bd.lo[2], -bd.hi[0], -bd.hi[1], -bd.hi[2]};
#pragma unroll
    for (int e = 0; e < 6; e++) v[e] = __reduce_min_sync(0xffffffffu, v[e]);
    if (lane == 0)
#pragma unroll
        for (int e = 0; e < 6; e++) red[warp][e] = v[e];
    __syncthreads();
    if (tid < 6) {
        int m = red[0][tid];
        for (int w = 1; w < kTileWarps; w++) m = min(m, red[w][tid]);
        int *ob = bk.box + 8 * (size_t)b;
        const int d = tid % 3;
        const bool empty = red[0][0] == 0x3fffffff && [&] {
            for (int w = 1; w < kTileWarps; w++)
                if (red[w][0] != 0x3fffffff) return false;
            return true;
        }();
        if (d >= DIMS) ob[tid] = 0;
        else if (empty) ob[tid] = tid < 3 ? home_lo[d] : home_hi[d];
        else ob[tid] = tid < 3 ? m : -m;
    }
}

void launch_move_deposit_f32_tiled(const GridP &g, const PartF32 &p, const Bricks &bk, float *const E[3],
                                   float *const B[3], float *const J[3], int *err, cudaStream_t s)
{
    static bool attr_set = false;
    const int bytes = bk.smem_floats * 4;
    if (!attr_set) {
        cudaFuncSetAttribute(k_move_f32_tiled<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
        cudaFuncSetAttribute(k_move_f32_tiled<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
        attr_set = true;
    }
    if (g.dims == 3)
        k_move_f32_tiled<3><<<bk.ntiles, kTileThreads, bytes, s>>>(g, p, bk, E[0], E[1], E[2], B[0], B[1], B[2], J[0],
                                                                   J[1], J[2], err);
    else
        k_move_f32_tiled<2><<<bk.ntiles, kTileThreads, bytes, s>>>(g, p, bk, E[0], E[1], E[2], B[0], B[1], B[2], J[0],
                                                                   J[1], J[2], err);
    count_launches(1);
}

}  // namespace pic
