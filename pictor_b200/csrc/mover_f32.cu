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
// memory, so each node value is computed once per brick rather than 8 times
// per particle.  The box is the bounding box, in cells, of where the brick's
// particles were after the previous step (particles drift away from their
// brick between reorders); it is stored per brick relative to the brick's
// centre, unwrapped across the periodic boundary, and this kernel writes the
// box for the next step.  A box too large for shared memory falls back to the
// brick itself plus one cell; particles outside the box gather and deposit
// through global memory with the same arithmetic.
//
// The current of the brick is summed in a shared-memory box as 32-bit fixed
// point with native integer atomics (FP32 atomic adds on shared memory are
// slow here, and per-particle FP32 reductions into L2, as the reference GPU
// kernel does, movdep_gpu.F90:193-318, saturate the L2 tag lookups).  The
// scale is set per brick from N * max|w| * qi * c, an upper bound of any sum,
// so nothing overflows.  The box is added to J once, as FP32 reductions onto
// the periodic interior image of each cell.
//
// Each thread streams particles n, n+256, ... and loads particle n+256 before
// it moves particle n, so the DRAM latency of the next particle overlaps the
// arithmetic of this one.
//
// The node averages and interpolation sums are computed identically on both
// paths (same expressions, same order, explicit fmaf), so the tiled and the
// per-particle kernels move particles bit-identically; currents differ by the
// order of the FP32 sums and the fixed-point rounding of the box.
#include "common.cuh"
#include "kernels.cuh"

namespace pic {

// Node-averaged fields at node offset nd (GatherVecEfld / GatherVecBfld,
// movdep_routines.F90:6-223): E averaged over the 2 edges, B over the 4 faces
// meeting at the node (2 in 2D), plus the external field.
template <int DIMS>
__device__ __forceinline__ void node_avg(const float *__restrict__ Ex, const float *__restrict__ Ey,
                                         const float *__restrict__ Ez, const float *__restrict__ Bx,
                                         const float *__restrict__ By, const float *__restrict__ Bz, int nd, int sy,
                                         int sz, float b0, float b1, float b2, float4 &A, float2 &Bv)
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

// Shared-memory accesses with explicit .shared addressing (32-bit shared
// addresses), so no generic-address resolution is left to run time.
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ float4 lds4(uint32_t a)
{
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}
__device__ __forceinline__ float2 lds2(uint32_t a)
{
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
    return v;
}
__device__ __forceinline__ void red_shared(uint32_t a, int v)
{
    asm volatile("red.shared.add.s32 [%0], %1;" ::"r"(a), "r"(v));
}

// round(v * S) for |v * S| <= 2^22 with one FMA: adding 1.5 * 2^23 leaves the
// rounded integer in the low mantissa bits.
__device__ __forceinline__ int fixed_of(float v, float S)
{
    return __float_as_int(fmaf(v, S, 12582912.f)) - 0x4B400000;
}

// Cell step of a position x in (-1, 2) relative to its cell: floor(x) as
// -1, 0 or 1, and the same as float.
__device__ __forceinline__ int cell_step(float x, float &fs)
{
    fs = x >= 1.f ? 1.f : (x < 0.f ? -1.f : 0.f);
    return x >= 1.f ? 1 : (x < 0.f ? -1 : 0);
}

// One zigzag segment: flux F (charge x displacement) and the segment's
// midpoint W within its cell (movdep.F90:187-233).
struct Seg {
    float Fx, Fy, Fz, Wx, Wy, Wz;
};

// VecJ entry e of a segment (movdep.F90:209,233 with the tables of
// vars.F90:328-355): 3D e = 0..3 Jx, 4..7 Jy, 8..11 Jz; 2D e = 0..1 Jx,
// 2..3 Jy, 4..7 Jz.
template <int DIMS>
__device__ __forceinline__ float seg_entry(const Seg &s, int e)
{
    if (DIMS == 2) {
        switch (e) {
            case 0: return s.Fx * (1.f - s.Wy);
            case 1: return s.Fx * s.Wy;
            case 2: return s.Fy * (1.f - s.Wx);
            case 3: return s.Fy * s.Wx;
            case 4: return (s.Fz * (1.f - s.Wx)) * (1.f - s.Wy);
            case 5: return (s.Fz * s.Wx) * (1.f - s.Wy);
            case 6: return (s.Fz * (1.f - s.Wx)) * s.Wy;
            default: return (s.Fz * s.Wx) * s.Wy;
        }
    }
    switch (e) {
        case 0: return (s.Fx * (1.f - s.Wy)) * (1.f - s.Wz);
        case 1: return (s.Fx * s.Wy) * (1.f - s.Wz);
        case 2: return (s.Fx * (1.f - s.Wy)) * s.Wz;
        case 3: return (s.Fx * s.Wy) * s.Wz;
        case 4: return (s.Fy * (1.f - s.Wx)) * (1.f - s.Wz);
        case 5: return (s.Fy * s.Wx) * (1.f - s.Wz);
        case 6: return (s.Fy * (1.f - s.Wx)) * s.Wz;
        case 7: return (s.Fy * s.Wx) * s.Wz;
        case 8: return (s.Fz * (1.f - s.Wx)) * (1.f - s.Wy);
        case 9: return (s.Fz * s.Wx) * (1.f - s.Wy);
        case 10: return (s.Fz * (1.f - s.Wx)) * s.Wy;
        default: return (s.Fz * s.Wx) * s.Wy;
    }
}

// Offset of VecJ entry e from the cell's base offset and its component
// (movdep_routines.F90:276-303): 0 = Jx, 1 = Jy, 2 = Jz.
template <int DIMS>
__device__ __forceinline__ int entry_offset(int e, int sy, int sz, int &comp)
{
    if (DIMS == 2) {
        const int o[8] = {0, sy, 0, 1, 0, 1, sy, 1 + sy};
        comp = e < 2 ? 0 : e < 4 ? 1 : 2;
        return o[e];
    }
    const int o[12] = {0, sy, sz, sy + sz, 0, 1, sz, 1 + sz, 0, 1, sy, 1 + sy};
    comp = e >> 2;
    return o[e];
}

// Deposit of the two segments of one move into global J: segment 1 into the
// cell c0 it starts in, segment 2 into the cell c1 the particle ends in; when
// the move stays in its cell both are summed first and added once.
template <int DIMS>
__device__ __forceinline__ void deposit_f32(float *Jx, float *Jy, float *Jz, int c0, int c1, int sy, int sz,
                                            const Seg &s1, const Seg &s2)
{
    constexpr int NE = DIMS == 3 ? 12 : 8;
    float *J3[3] = {Jx, Jy, Jz};
    const bool same = c0 == c1;
#pragma unroll
    for (int e = 0; e < NE; e++) {
        int comp;
        const int o = entry_offset<DIMS>(e, sy, sz, comp);
        atomicAdd(J3[comp] + c0 + o, seg_entry<DIMS>(s1, e) + (same ? seg_entry<DIMS>(s2, e) : 0.f));
    }
    if (!same) {
#pragma unroll
        for (int e = 0; e < NE; e++) {
            int comp;
            const int o = entry_offset<DIMS>(e, sy, sz, comp);
            atomicAdd(J3[comp] + c1 + o, seg_entry<DIMS>(s2, e));
        }
    }
}

// The same deposit into the shared current box of a brick (shared address
// sJ0 of component 0; components njc words apart), as fixed-point integers
// (v * S rounded to nearest) added with native shared-memory integer atomics;
// S is chosen per brick so that no entry and no sum can overflow.
template <int DIMS>
__device__ __forceinline__ void deposit_box(uint32_t sJ0, int njc, int JX, int JXY, float S, int j0, int j1,
                                            const Seg &s1, const Seg &s2)
{
    constexpr int NE = DIMS == 3 ? 12 : 8;
    const bool same = j0 == j1;
#pragma unroll
    for (int e = 0; e < NE; e++) {
        int comp;
        const int o = entry_offset<DIMS>(e, JX, JXY, comp);
        red_shared(sJ0 + 4u * (uint32_t)(comp * njc + j0 + o),
                   fixed_of(seg_entry<DIMS>(s1, e) + (same ? seg_entry<DIMS>(s2, e) : 0.f), S));
    }
    if (!same) {
#pragma unroll
        for (int e = 0; e < NE; e++) {
            int comp;
            const int o = entry_offset<DIMS>(e, JX, JXY, comp);
            red_shared(sJ0 + 4u * (uint32_t)(comp * njc + j1 + o), fixed_of(seg_entry<DIMS>(s2, e), S));
        }
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

// Shared-memory boxes of a brick (unused by the per-particle kernel).
struct TileBox {
    uint32_t nA, nB;    // shared addresses: node E x,y,z, B x (16 B) / node B y,z (8 B)
    uint32_t sJ;        // shared address of the current box (3 planar components, fixed point)
    int hc[3];          // brick centre (1-based interior indices)
    int lo[3];          // box lower corner, cells relative to hc
    int C[3];           // box extent in cells (1 on the unused z axis of 2D)
    int NX, NXY;        // node box strides
    int JX, JXY, njc;   // current box strides and size
    float S;            // fixed-point scale of the current box
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

// One particle's state in registers.
struct PState {
    uint32_t key;
    float dx, dy, dz, ux, uy, uz, w;
};

template <int DIMS>
__device__ __forceinline__ PState load_state(const PartF32 &p, uint32_t n)
{
    PState s;
    s.key = p.key[n];
    s.dx = p.dx[n];
    s.dy = p.dy[n];
    s.dz = DIMS == 3 ? p.dz[n] : 0.f;
    s.ux = p.ux[n];
    s.uy = p.uy[n];
    s.uz = p.uz[n];
    s.w = p.w[n];
    return s;
}

// Move one particle (state s, slot n).  TILED: gather through the node box
// when the particle's cell is inside it, else (and always when !TILED)
// through the global arrays at the particle's wrapped cell.  The current of
// a particle inside the box goes to the box; otherwise to the global J at the
// wrapped cell (ghost layers included; the fold adds them to their periodic
// images).
template <int DIMS, bool TILED>
__device__ __forceinline__ void push_one(const GridP &g, const PartF32 &p, uint32_t n, const PState &s,
                                         const float *__restrict__ Ex, const float *__restrict__ Ey,
                                         const float *__restrict__ Ez, const float *__restrict__ Bx,
                                         const float *__restrict__ By, const float *__restrict__ Bz, float *Jx,
                                         float *Jy, float *Jz, int *err, const TileBox &tb, Bounds &bd)
{
    const int flv = (int)(s.key >> kFlvShift);
    if (flv == 0) return;
    const int cell = (int)(s.key & kCellMask);
    int i, j, k;
    decode_cell(g, cell, i, j, k);
    if (i < 3 || i > g.mx - 3 || j < 3 || j > g.my - 3 || (DIMS == 3 && (k < 3 || k > g.mz - 3)) ||
        (DIMS == 2 && k != 1)) {
        raise_error(err, PIC_DEVERR_RANGE);
        return;
    }
    const float dx = s.dx, dy = s.dy, dz = s.dz;
    float wt[8];
    weights_f32<DIMS>(dx, dy, dz, wt);
    const int sy = (int)g.sy, sz = (int)g.sz;
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
            accum(wt[c8], lds4(tb.nA + 16u * (uint32_t)q), lds2(tb.nB + 8u * (uint32_t)q), pE, pB);
        }
    } else {
#pragma unroll
        for (int c8 = 0; c8 < (DIMS == 3 ? 8 : 4); c8++) {
            const int nd = cell + (c8 & 1) + ((c8 >> 1) & 1) * sy + ((c8 >> 2) & 1) * sz;
            float4 A;
            float2 Bv;
            node_avg<DIMS>(Ex, Ey, Ez, Bx, By, Bz, nd, sy, sz, g.bext_f[0], g.bext_f[1], g.bext_f[2], A, Bv);
            accum(wt[c8], A, Bv, pE, pB);
        }
    }
    const float qm = g.qm_half_f[flv];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        pE[d] *= qm;
        pB[d] *= qm;
    }
    float u = s.ux, v = s.uy, w = s.uz, gg;
    boris_f32(g.c_f, g.sqc_f, g.cinv_f, pE, pB, u, v, w, gg);
    // displacement in cell units, positions relative to this cell's corner
    const float x1 = fmaf(u, gg, dx), y1 = fmaf(v, gg, dy), z1 = DIMS == 3 ? fmaf(w, gg, dz) : 0.f;
    // |displacement| < c < 1, so x1 lies in (-1, 2): the cell step is -1, 0 or 1
    float fsx, fsy, fsz = 0.f;
    const int sxx = cell_step(x1, fsx), syy = cell_step(y1, fsy), szz = DIMS == 3 ? cell_step(z1, fsz) : 0;
    // zigzag relay point with ip0 = 0, ip = s (movdep.F90:183-185)
    const float xr = fminf(fminf(fsx, 0.f) + 1.f, fmaxf(fmaxf(fsx, 0.f), 0.5f * (dx + x1)));
    const float yr = fminf(fminf(fsy, 0.f) + 1.f, fmaxf(fmaxf(fsy, 0.f), 0.5f * (dy + y1)));
    const float qthis = s.w * g.qi_f;
    float Fz1, Fz2, Wz1 = 0.f, Wz2 = 0.f;
    if (DIMS == 3) {
        const float zr = fminf(fminf(fsz, 0.f) + 1.f, fmaxf(fmaxf(fsz, 0.f), 0.5f * (dz + z1)));
        Fz1 = qthis * (zr - dz);
        Fz2 = qthis * (z1 - zr);
        Wz1 = 0.5f * (dz + zr);
        Wz2 = 0.5f * (z1 + zr) - fsz;
    } else {
        // out-of-plane motion: no cell crossing, the relay point is the midpoint
        Fz1 = qthis * (0.5f * (w * gg));
        Fz2 = Fz1;
    }
    const Seg s1 = {qthis * (xr - dx), qthis * (yr - dy), Fz1, 0.5f * (dx + xr), 0.5f * (dy + yr), Wz1};
    const Seg s2 = {qthis * (x1 - xr), qthis * (y1 - yr), Fz2, 0.5f * (x1 + xr) - fsx, 0.5f * (y1 + yr) - fsy, Wz2};
    if (inside) {
        const int lx = uo[0] - tb.lo[0], ly = uo[1] - tb.lo[1], lz = DIMS == 3 ? uo[2] - tb.lo[2] : 0;
        const int jb = (lx + 1) + tb.JX * (ly + 1) + (DIMS == 3 ? tb.JXY * (lz + 1) : 0);
        deposit_box<DIMS>(tb.sJ, tb.njc, tb.JX, tb.JXY, tb.S, jb, jb + sxx + syy * tb.JX + szz * tb.JXY, s1, s2);
    } else {
        deposit_f32<DIMS>(Jx, Jy, Jz, cell, cell + sxx + syy * sy + szz * sz, sy, sz, s1, s2);
    }
    // new offsets and periodic cell index
    float nx = x1 - fsx, ny = y1 - fsy, nz = z1 - fsz;
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

// Particles [n0, n1) with stride `step`, the next particle prefetched.
template <int DIMS, bool TILED>
__device__ __forceinline__ void push_range(const GridP &g, const PartF32 &p, uint32_t n0, uint32_t n1, uint32_t step,
                                           const float *__restrict__ Ex, const float *__restrict__ Ey,
                                           const float *__restrict__ Ez, const float *__restrict__ Bx,
                                           const float *__restrict__ By, const float *__restrict__ Bz, float *Jx,
                                           float *Jy, float *Jz, int *err, const TileBox &tb, Bounds &bd)
{
    if (n0 >= n1) return;
    PState cur = load_state<DIMS>(p, n0);
    for (uint32_t n = n0; n < n1; n += step) {
        PState nxt = cur;
        if (n1 - n > step) nxt = load_state<DIMS>(p, n + step);
        push_one<DIMS, TILED>(g, p, n, cur, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, err, tb, bd);
        cur = nxt;
    }
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
    TileBox tb = {};
    Bounds bd;
    const uint32_t step = gridDim.x * blockDim.x;
    push_range<DIMS, false>(g, p, blockIdx.x * blockDim.x + threadIdx.x, (uint32_t)cnt->used, step, Ex, Ey, Ez, Bx,
                            By, Bz, Jx, Jy, Jz, err, tb, bd);
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

// Interior index of the unwrapped 1-based index a (no division when a is
// already interior or one period away).
__device__ __forceinline__ int interior_of(int a, int n)
{
    if (a < 3) a += n;
    else if (a > n + 2) a -= n;
    if (a < 3 || a > n + 2) a = wrap_interior(a, n);
    return a;
}

template <int DIMS>
__global__ void __launch_bounds__(kTileThreads, 3)
    k_move_f32_tiled(GridP g, PartF32 p, Bricks bk, const float *__restrict__ Ex, const float *__restrict__ Ey,
                     const float *__restrict__ Ez, const float *__restrict__ Bx, const float *__restrict__ By,
                     const float *__restrict__ Bz, float *Jx, float *Jy, float *Jz, int *err)
{
    extern __shared__ __align__(16) float sm[];
    __shared__ int red[kTileWarps][6];
    __shared__ int s_off[3][kBoxAxisMax + 3];
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
    if (hi[0] < lo[0] || hi[1] < lo[1] || hi[2] < lo[2] || hi[0] - lo[0] >= kBoxAxisMax ||
        hi[1] - lo[1] >= kBoxAxisMax || hi[2] - lo[2] >= kBoxAxisMax ||
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
    int *sJ = reinterpret_cast<int *>(sm + 6 * nnode);
    tb.nA = smem_addr(nA);
    tb.nB = smem_addr(nB);
    tb.sJ = smem_addr(sJ);
    // fixed-point scale: a particle adds at most b = |w| qi c to any entry
    // (its displacement per axis is below c), so with S = 2^30 / (N b) no sum
    // of the N particles exceeds 2^30; S <= 2^22 / b keeps each contribution
    // below 2^22 (the range of fixed_of)
    {
        const float b1 = g.c_f * g.qi_f * __uint_as_float(*bk.wmax_bits);
        const float n = fmaxf((float)(p1 - p0), 256.f);
        tb.S = b1 > 0.f ? 1073741824.f / (b1 * n) : 1.f;
    }
    // periodic offsets of the box cells lo-1 .. lo+C+1 along each axis
    // (memory offset of the interior image, times the axis stride)
    {
        const int ext[3] = {JX, JY, JZ};
        const int str[3] = {1, (int)g.sy, (int)g.sz};
#pragma unroll
        for (int d = 0; d < DIMS; d++)
            for (int t = tid; t < ext[d]; t += kTileThreads)
                s_off[d][t] = (interior_of(tb.hc[d] + lo[d] - 1 + t, n3[d]) - 1) * str[d];
        if (DIMS == 2 && tid == 0) s_off[2][0] = 0;
    }
    for (int q = tid; q < 3 * tb.njc; q += kTileThreads) sJ[q] = 0;
    __syncthreads();
    // stage node-averaged fields: node q = xx + NX*(yy + NY*zz); q/NX and
    // r/NY by multiply-high (exact for q < 2^16, NX, NY < 2^16)
    {
        const int sy = (int)g.sy, sz = (int)g.sz;
        const uint32_t mX = 0xffffffffu / (uint32_t)NX + 1u, mY = 0xffffffffu / (uint32_t)NY + 1u;
        for (int q = tid; q < nnode; q += kTileThreads) {
            const int r = (int)__umulhi((uint32_t)q, mX), xx = q - r * NX;
            const int zz = (int)__umulhi((uint32_t)r, mY), yy = r - zz * NY;
            const int nd = s_off[0][xx + 1] + s_off[1][yy + 1] + (DIMS == 3 ? s_off[2][zz + 1] : 0);
            float4 A;
            float2 Bv;
            node_avg<DIMS>(Ex, Ey, Ez, Bx, By, Bz, nd, sy, sz, g.bext_f[0], g.bext_f[1], g.bext_f[2], A, Bv);
            nA[q] = A;
            nB[q] = Bv;
        }
    }
    __syncthreads();

    Bounds bd;
    bd.init();
    push_range<DIMS, true>(g, p, p0 + tid, p1, kTileThreads, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, err, tb, bd);
    __syncthreads();

    // add the box current to the periodic interior image of each cell
    {
        const float inv = 1.f / tb.S;
        const uint32_t mX = 0xffffffffu / (uint32_t)JX + 1u, mY = 0xffffffffu / (uint32_t)JY + 1u;
        for (int q = tid; q < tb.njc; q += kTileThreads) {
            const int r = (int)__umulhi((uint32_t)q, mX), xx = q - r * JX;
            const int zz = (int)__umulhi((uint32_t)r, mY), yy = r - zz * JY;
            const int off = s_off[0][xx] + s_off[1][yy] + (DIMS == 3 ? s_off[2][zz] : 0);
            const int vx = sJ[q], vy = sJ[tb.njc + q], vz = sJ[2 * tb.njc + q];
            if (vx != 0) atomicAdd(Jx + off, (float)vx * inv);
            if (vy != 0) atomicAdd(Jy + off, (float)vy * inv);
            if (vz != 0) atomicAdd(Jz + off, (float)vz * inv);
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
    if (tid == 0) {
        int m[6];
        for (int e = 0; e < 6; e++) {
            m[e] = red[0][e];
            for (int w2 = 1; w2 < kTileWarps; w2++) m[e] = min(m[e], red[w2][e]);
        }
        int *ob = bk.box + 8 * (size_t)b;
        const bool empty = m[0] == 0x3fffffff;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (d >= DIMS) {
                ob[d] = ob[d + 3] = 0;
            } else if (empty) {
                ob[d] = home_lo[d];
                ob[d + 3] = home_hi[d];
            } else {
                ob[d] = m[d];
                ob[d + 3] = -m[d + 3];
            }
        }
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
