// mover_f32.cuh -- the FP32 cell-relative mover: gather, relativistic Boris
// push, zigzag current deposit and periodic wrap (the device functions; the
// kernels and launchers are in mover_f32.cu, the persistent ensemble step
// in ensemble.cu).
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
// memory, so each node value is read once per brick rather than 8 times per
// particle; the averages themselves are computed once per move for the whole
// grid (k_node_avg, mover_f32.cu: a streaming pass that writes 24 bytes per
// node), so the staging is a copy rather than 20 scattered reads per node
// for a box about twice the brick's size.  The box is the bounding box, in cells, of where the brick's
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
// arithmetic of this one.  The reorder lays a brick's particles out so that
// the lanes of a warp hold particles of neighbouring cells (bricks.cu), which
// keeps their shared-memory accesses on distinct banks.  A particle that
// stays in its cell deposits its two zigzag segments in closed form in one
// pass; the second segments of the lanes that cross a face are queued per
// warp and deposited 32 at a time.  In 3D the form can instead give each
// segment the cross term of its exact line integral (Part), which conserves
// charge exactly.  The kernel runs at 80 registers (3 CTAs per SM); the
// bounds of the particles' new cells are packed two 16-bit halves to a
// register (PackedBounds) to stay there without spilling.
//
// The node averages and interpolation sums are computed identically on both
// paths (same expressions, same order, explicit fmaf), so the tiled and the
// per-particle kernels move particles bit-identically; currents differ by the
// order of the FP32 sums and the fixed-point rounding of the box.
#pragma once

#include "common.cuh"
#include "kernels.cuh"
#include "tile.cuh"

namespace pic {

// Relativistic Boris rotation (movdep.F90:143-167) in FP32 with hardware
// reciprocal square root.  On entry u,v,w = gamma v / c and pE, pB are
// scaled by q/m * 0.5; returns new momenta and gg = c^2/sqrt(c^2 + |c u|^2),
// and whether the new momentum is finite (the argument of that square root
// is NaN or infinite otherwise).
__device__ __forceinline__ bool boris_f32(float c, float sqc, float cinv, const float pE[3], const float pB[3],
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
    const float s2 = fmaf(w0, w0, fmaf(v0, v0, fmaf(u0, u0, sqc)));
    gout = sqc * rsqrtf(s2);
    return s2 <= 3.402823466e38f;
}

// Cell step of a position x in (-1, 2) relative to its cell: floor(x) as
// -1, 0 or 1, and the same as float.
__device__ __forceinline__ int cell_step(float x, float &fs)
{
    fs = x >= 1.f ? 1.f : (x < 0.f ? -1.f : 0.f);
    return x >= 1.f ? 1 : (x < 0.f ? -1 : 0);
}

// One part of a move's zigzag current (movdep.F90:177-237 with the weight
// tables of vars.F90:322-356): flux F (charge x displacement) per axis,
// midpoint weights W within the cell, and a cross term.
//
// A move is deposited as part A into the cell it starts in and part B into
// the cell it ends in.  When the particle stays in its cell the relay point
// is the midpoint and the two zigzag segments land in the same cell; their
// sum is written as one part, the whole move's F and midpoint W.  When the
// particle crosses a face, A is the first segment and B the second.
//
// 3D: the entries of a part are F (1-Wy)(1-Wz) + C for Jx at the (0,0)
// corner, the sign of C + for (1-W)(1-W) and W W and - for the mixed
// products, likewise for Jy and Jz with the same C; D[0] holds C.  With the
// reference's weights (vars.F90:343-355: products of segment-midpoint
// weights, which the FP64 form keeps) C = q dx dy dz / 16 for a same-cell
// move (the pair of segment midpoints) and 0 for the segments of a crossing
// move.  With pic_config.exact_charge (XC) each part is a straight segment
// inside one cell and its entries are the segment's exact line integrals of
// the bilinear weights, C = q dx dy dz / 12 for the segment's displacement
// (the 3D form of Villasenor and Buneman's weights): the current then
// satisfies the discrete continuity equation with the CIC charge exactly and
// the Gauss residual stays at the FP32 round-off of the field updates.
// 2D: the in-plane current needs no cross term to conserve charge; the
// out-of-plane Jz of a same-cell move keeps the reference's two-segment value
// F ((1-Wx)(1-Wy) + dx dy / 16), D[2] holding dx dy / 16.
struct Part {
    float F[3], W[3], D[3];
};

// The VecJ entries of a part (3D: 0..3 Jx at (y,z) corners, 4..7 Jy at
// (x,z), 8..11 Jz at (x,y); 2D: 0..1 Jx, 2..3 Jy, 4..7 Jz), scaled by the F
// the part carries.
template <int DIMS, bool CROSS = true>
__device__ __forceinline__ void part_entries(const Part &d, float v[12])
{
    const float ax = 1.f - d.W[0], ay = 1.f - d.W[1];
    if (!CROSS) {
        // D = 0: plain products (pairs of entries by packed multiplies)
        if (DIMS == 3) {
            const float az = 1.f - d.W[2];
            const float2 Fx = fmul2(make_float2(d.F[0], d.F[0]), make_float2(ay, d.W[1]));
            const float2 v01 = fmul2(Fx, make_float2(az, az)), v23 = fmul2(Fx, make_float2(d.W[2], d.W[2]));
            const float2 Fy = fmul2(make_float2(d.F[1], d.F[1]), make_float2(ax, d.W[0]));
            const float2 v45 = fmul2(Fy, make_float2(az, az)), v67 = fmul2(Fy, make_float2(d.W[2], d.W[2]));
            const float2 Fz = fmul2(make_float2(d.F[2], d.F[2]), make_float2(ax, d.W[0]));
            const float2 v89 = fmul2(Fz, make_float2(ay, ay)), vab = fmul2(Fz, make_float2(d.W[1], d.W[1]));
            v[0] = v01.x; v[1] = v01.y; v[2] = v23.x; v[3] = v23.y;
            v[4] = v45.x; v[5] = v45.y; v[6] = v67.x; v[7] = v67.y;
            v[8] = v89.x; v[9] = v89.y; v[10] = vab.x; v[11] = vab.y;
        } else {
            v[0] = d.F[0] * ay;
            v[1] = d.F[0] * d.W[1];
            v[2] = d.F[1] * ax;
            v[3] = d.F[1] * d.W[0];
            const float Ha = d.F[2] * ax, Hw = d.F[2] * d.W[0];
            v[4] = Ha * ay;
            v[5] = Hw * ay;
            v[6] = Ha * d.W[1];
            v[7] = Hw * d.W[1];
        }
        return;
    }
    if (DIMS == 3) {
        // (Fa, Fw) = F (1-W, W) along the entry's first transverse axis, then
        // each pair of entries by one packed FMA with the cross term +-Fd
        const float az = 1.f - d.W[2];
        const float Fd = d.D[0];   // C = q dx dy dz / 12, common to the three components
        {
            const float2 Fp = fmul2(make_float2(d.F[0], d.F[0]), make_float2(ay, d.W[1]));
            const float2 v01 = ffma2(Fp, make_float2(az, az), make_float2(Fd, -Fd));
            const float2 v23 = ffma2(Fp, make_float2(d.W[2], d.W[2]), make_float2(-Fd, Fd));
            v[0] = v01.x; v[1] = v01.y; v[2] = v23.x; v[3] = v23.y;
        }
        {
            const float2 Fp = fmul2(make_float2(d.F[1], d.F[1]), make_float2(ax, d.W[0]));
            const float2 v45 = ffma2(Fp, make_float2(az, az), make_float2(Fd, -Fd));
            const float2 v67 = ffma2(Fp, make_float2(d.W[2], d.W[2]), make_float2(-Fd, Fd));
            v[4] = v45.x; v[5] = v45.y; v[6] = v67.x; v[7] = v67.y;
        }
        {
            const float2 Fp = fmul2(make_float2(d.F[2], d.F[2]), make_float2(ax, d.W[0]));
            const float2 v89 = ffma2(Fp, make_float2(ay, ay), make_float2(Fd, -Fd));
            const float2 vab = ffma2(Fp, make_float2(d.W[1], d.W[1]), make_float2(-Fd, Fd));
            v[8] = v89.x; v[9] = v89.y; v[10] = vab.x; v[11] = vab.y;
        }
    } else {
        v[0] = d.F[0] * ay;
        v[1] = d.F[0] * d.W[1];
        v[2] = d.F[1] * ax;
        v[3] = d.F[1] * d.W[0];
        const float Fa = d.F[2] * ax, Fw = d.F[2] * d.W[0], Fd = d.F[2] * d.D[2];
        v[4] = fmaf(Fa, ay, Fd);
        v[5] = fmaf(Fw, ay, -Fd);
        v[6] = fmaf(Fa, d.W[1], -Fd);
        v[7] = fmaf(Fw, d.W[1], Fd);
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

// A part into global J at cell offset c (FP32 atomics).
template <int DIMS, bool CROSS = true>
__device__ __forceinline__ void deposit_part_global(float *Jx, float *Jy, float *Jz, int c, int sy, int sz,
                                                    const Part &d)
{
    constexpr int NE = DIMS == 3 ? 12 : 8;
    float *J3[3] = {Jx, Jy, Jz};
    float v[12];
    part_entries<DIMS, CROSS>(d, v);
#pragma unroll
    for (int e = 0; e < NE; e++) {
        int comp;
        const int o = entry_offset<DIMS>(e, sy, sz, comp);
        atomicAdd(J3[comp] + c + o, v[e]);
    }
}

// A part into the shared current box at byte address a (cell j's Jx word),
// F already scaled by the fixed-point scale S.
template <int DIMS, bool CROSS = true>
__device__ __forceinline__ void deposit_part_box(uint32_t a, const JOff &o, const Part &d)
{
    float v[12];
    part_entries<DIMS, CROSS>(d, v);
    red_entries_box<DIMS>(a, o, v);
}

// Bounds of the particles' new cells with lo and -hi of an axis packed as
// two signed 16-bit halves of one register (the offsets from the brick
// centre are far below 2^15), updated by one packed min.
struct PackedBounds {
    uint32_t p[3];
    __device__ void init() { p[0] = p[1] = p[2] = 0x3fff3fffu; }
    __device__ __forceinline__ void add(int a, int v)
    {
        const uint32_t nv = ((uint32_t)v & 0xffffu) | ((uint32_t)(-v) << 16);
        uint32_t d;
        asm("min.s16x2 %0, %1, %2;" : "=r"(d) : "r"(p[a]), "r"(nv));
        p[a] = d;
    }
    __device__ Bounds unpack() const
    {
        Bounds b;
        for (int a = 0; a < 3; a++) {
            const int lo = (int)(int16_t)(p[a] & 0xffffu), mhi = (int)(int16_t)(p[a] >> 16);
            b.lo[a] = lo == 0x3fff ? 0x3fffffff : lo;
            b.hi[a] = mhi == 0x3fff ? -0x3fffffff : -mhi;
        }
        return b;
    }
};

// Move one particle (state s, slot n).  TILED: gather through the node box
// when the particle's cell is inside it, else (and always when !TILED)
// through the global arrays at the particle's wrapped cell.  The current of
// a particle inside the box goes to the box; otherwise to the global J at the
// wrapped cell (ghost layers included; the fold adds them to their periodic
// images).  Returns true when the particle crossed a face inside the box: its
// second zigzag segment is then left to the caller (Bq, at box address qa),
// which deposits those of a warp together.  The cell range is checked where
// it guards a global access; a cell decoded inside the box is in range.
template <int DIMS, bool TILED, bool XC = false, bool XS = false>
__device__ __forceinline__ bool push_one(const GridP &g, const PartF32 &p, uint32_t n, const PState &s,
                                         const float *__restrict__ Ex, const float *__restrict__ Ey,
                                         const float *__restrict__ Ez, const float *__restrict__ Bx,
                                         const float *__restrict__ By, const float *__restrict__ Bz, float *Jx,
                                         float *Jy, float *Jz, int *err, const TileBox &tb, PackedBounds &bd, Part &Bq,
                                         uint32_t &qa)
{
    const int flv = (int)(s.key >> kFlvShift);
    if (flv == 0) return false;
    const int cell = (int)(s.key & kCellMask);
    int i, j, k;
    decode_cell(g, cell, i, j, k);
    const float dx = s.dx, dy = s.dy, dz = s.dz;
    float wt[8];
    weights_f32<DIMS>(dx, dy, dz, wt);
    const int sy = (int)g.sy, sz = (int)g.sz;
    int uo[3] = {0, 0, 0};   // unwrapped offsets from the brick centre
    bool inside = false;
    int nb = 0;
    if (TILED) {
        uo[0] = XS ? i - tb.hc[0] : unwrap_offset(i, tb.hc[0], g.nx);
        uo[1] = unwrap_offset(j, tb.hc[1], g.ny);
        if (DIMS == 3) uo[2] = unwrap_offset(k, tb.hc[2], g.nz);
        const int lx = uo[0] - tb.lo[0], ly = uo[1] - tb.lo[1], lz = DIMS == 3 ? uo[2] - tb.lo[2] : 0;
        inside = (unsigned)lx < (unsigned)tb.C[0] && (unsigned)ly < (unsigned)tb.C[1] &&
                 (DIMS == 2 || (unsigned)lz < (unsigned)tb.C[2]);
        nb = lx + tb.NX * ly + tb.NXY * lz;
    }
    if (!inside && (i < 3 || i > g.mx - 3 || j < 3 || j > g.my - 3 ||
                    (DIMS == 3 && (k < 3 || k > g.mz - 3)) || (DIMS == 2 && k != 1))) {
        raise_error(err, PIC_DEVERR_RANGE);
        return false;
    }
    float pE[3] = {0.f, 0.f, 0.f}, pB[3] = {0.f, 0.f, 0.f};
    if (inside) {
        gather_box<DIMS>(tb, nb, wt, pE, pB);
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
    // a non-finite momentum raises NAN; the particle's offsets then turn NaN
    // but its cell stays (cell_step of NaN is 0), so every index it forms
    // stays inside the box or the ghost frame (a branch that left the
    // particle as it was costs the kernel registers it does not have)
    if (!boris_f32(g.c_f, g.sqc_f, g.cinv_f, pE, pB, u, v, w, gg)) raise_error(err, PIC_DEVERR_NAN);
    // displacement in cell units, positions relative to this cell's corner
    const float x1 = fmaf(u, gg, dx), y1 = fmaf(v, gg, dy), z1 = DIMS == 3 ? fmaf(w, gg, dz) : 0.f;
    // |displacement| < c < 1, so x1 lies in (-1, 2): the cell step is -1, 0 or 1
    float fsx, fsy, fsz = 0.f;
    const int sxx = cell_step(x1, fsx), syy = cell_step(y1, fsy), szz = DIMS == 3 ? cell_step(z1, fsz) : 0;
    // zigzag relay point with ip0 = 0, ip = s (movdep.F90:183-185)
    const float xr = fminf(fminf(fsx, 0.f) + 1.f, fmaxf(fmaxf(fsx, 0.f), 0.5f * (dx + x1)));
    const float yr = fminf(fminf(fsy, 0.f) + 1.f, fmaxf(fmaxf(fsy, 0.f), 0.5f * (dy + y1)));
    const float zr = DIMS == 3 ? fminf(fminf(fsz, 0.f) + 1.f, fmaxf(fmaxf(fsz, 0.f), 0.5f * (dz + z1))) : 0.f;
    const bool stays = (sxx | syy | szz) == 0;
    // charge, times the box's fixed-point scale for a particle inside the box
    const float qthis = s.w * g.qi_f * (inside ? tb.S : 1.f);
    // part A: the whole move (stays) or the first segment, ending at e
    const float ex = stays ? x1 : xr, ey = stays ? y1 : yr, ez = stays ? z1 : zr;
    const float mx = ex - dx, my = ey - dy, mz = ez - dz;
    Part A, B;
    A.F[0] = qthis * mx;
    A.F[1] = qthis * my;
    A.W[0] = 0.5f * (dx + ex);
    A.W[1] = 0.5f * (dy + ey);
    A.D[2] = stays ? 0.0625f * (mx * my) : 0.f;
    B.F[0] = qthis * (x1 - xr);
    B.F[1] = qthis * (y1 - yr);
    B.W[0] = 0.5f * (x1 + xr) - fsx;
    B.W[1] = 0.5f * (y1 + yr) - fsy;
    B.D[0] = B.D[1] = B.D[2] = 0.f;
    if (DIMS == 3) {
        A.F[2] = qthis * mz;
        A.W[2] = 0.5f * (dz + ez);
        // C of part A: the exact line integral's (XC), else the reference's
        // two-segment value for a same-cell move (dy dz / 16 from the segment
        // midpoints) and none for the first segment of a crossing move
        A.D[0] = XC ? A.F[0] * (my * mz) * (1.f / 12.f) : (stays ? A.F[0] * (my * mz) * 0.0625f : 0.f);
        B.F[2] = qthis * (z1 - zr);
        B.W[2] = 0.5f * (z1 + zr) - fsz;
        A.D[2] = 0.f;
    } else {
        // out-of-plane motion: no cell crossing, each segment carries half
        const float fz = qthis * (0.5f * (w * gg));
        A.F[2] = stays ? 2.f * fz : fz;
        B.F[2] = fz;
        A.W[2] = B.W[2] = 0.f;
        A.D[0] = A.D[1] = 0.f;
    }
    bool queued = false;
    if (inside) {
        const int lx = uo[0] - tb.lo[0], ly = uo[1] - tb.lo[1], lz = DIMS == 3 ? uo[2] - tb.lo[2] : 0;
        const int jb = (lx + 1) + tb.JX * (ly + 1) + (DIMS == 3 ? tb.JXY * (lz + 1) : 0);
        deposit_part_box<DIMS>(tb.sJ + 4u * (uint32_t)jb, tb.jo, A);
        if (!stays) {
            if (DIMS == 3) B.D[0] = XC ? B.F[0] * ((y1 - yr) * (z1 - zr)) * (1.f / 12.f) : 0.f;   // C of part B
            Bq = B;
            qa = tb.sJ + 4u * (uint32_t)(jb + sxx + syy * tb.JX + szz * tb.JXY);
            queued = true;
        }
    } else {
        deposit_part_global<DIMS>(Jx, Jy, Jz, cell, sy, sz, A);
        if (!stays) {
            if (DIMS == 3) B.D[0] = XC ? B.F[0] * ((y1 - yr) * (z1 - zr)) * (1.f / 12.f) : 0.f;   // C of part B
            deposit_part_global<DIMS, DIMS == 3>(Jx, Jy, Jz, cell + sxx + syy * sy + szz * sz, sy, sz, B);
        }
    }
    // new offsets and periodic cell index
    float nx = x1 - fsx, ny = y1 - fsy, nz = z1 - fsz;
    int ax = sxx, ay = syy, az = szz;
    if (nx >= 1.f) { nx -= 1.f; ax += 1; }
    if (ny >= 1.f) { ny -= 1.f; ay += 1; }
    if (DIMS == 3 && nz >= 1.f) { nz -= 1.f; az += 1; }
    if (TILED) {
        bd.add(0, uo[0] + ax);
        bd.add(1, uo[1] + ay);
        if (DIMS == 3) bd.add(2, uo[2] + az);
    }
    // a slab (XS) leaves an x leaver in the ghost cell beside its face for
    // the exchange; the single domain wraps it periodically
    const int ni = XS ? i + ax : wrap_index(i + ax, g.mx), nj = wrap_index(j + ay, g.my);
    const int nk = DIMS == 3 ? wrap_index(k + az, g.mz) : 1;
    p.key[n] = ((uint32_t)flv << kFlvShift) | (uint32_t)((ni - 1) + g.mx * ((nj - 1) + g.my * (nk - 1)));
    p.dx[n] = nx;
    p.dy[n] = ny;
    if (DIMS == 3) p.dz[n] = nz;
    p.ux[n] = u;
    p.uy[n] = v;
    p.uz[n] = w;
    return queued;
}

// Particles [n0, n1) with stride `step`, the next particle prefetched (per-
// particle form: second segments deposited at once).
template <int DIMS, bool XC = false, bool XS = false>
__device__ __forceinline__ void push_range(const GridP &g, const PartF32 &p, uint32_t n0, uint32_t n1, uint32_t step,
                                           const float *__restrict__ Ex, const float *__restrict__ Ey,
                                           const float *__restrict__ Ez, const float *__restrict__ Bx,
                                           const float *__restrict__ By, const float *__restrict__ Bz, float *Jx,
                                           float *Jy, float *Jz, int *err, const TileBox &tb, PackedBounds &bd)
{
    if (n0 >= n1) return;
    PState cur = load_state<DIMS>(p, n0);
    Part Bq;
    uint32_t qa;
    for (uint32_t n = n0; n < n1; n += step) {
        PState nxt = cur;
        if (n1 - n > step) nxt = load_state<DIMS>(p, n + step);
        push_one<DIMS, false, XC, XS>(g, p, n, cur, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, err, tb, bd, Bq, qa);
        cur = nxt;
    }
}

__device__ __forceinline__ uint32_t lanemask_lt()
{
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Deposit the first k queued segments, one per lane, into the box.
template <int DIMS>
__device__ __forceinline__ void drain_queue(float (*q)[32], int k, const JOff &jo)
{
    const int lane = threadIdx.x & 31;
    __syncwarp();
    if (lane < k) {
        Part B;
        B.F[0] = q[0][lane];
        B.F[1] = q[1][lane];
        B.F[2] = q[2][lane];
        B.W[0] = q[3][lane];
        B.W[1] = q[4][lane];
        B.W[2] = q[5][lane];
        B.D[0] = q[7][lane];
        deposit_part_box<DIMS, DIMS == 3>(__float_as_uint(q[6][lane]), jo, B);
    }
    __syncwarp();
}

// Tiled form: warp w of the CTA moves slots p0 + 32 w + 256 t + lane, all
// lanes of a warp stepping together (lanes past p1 idle), so that the second
// segments of the lanes that crossed a face can be gathered into the warp's
// queue and deposited 32 at a time instead of in a branch that nearly every
// warp would take for a few of its lanes.  The next particle loads while
// this one moves.
template <int DIMS, bool XC = false, bool XS = false>
__device__ __forceinline__ void push_range_tiled(const GridP &g, const PartF32 &p, uint32_t p0, uint32_t p1,
                                                 const float *__restrict__ Ex, const float *__restrict__ Ey,
                                                 const float *__restrict__ Ez, const float *__restrict__ Bx,
                                                 const float *__restrict__ By, const float *__restrict__ Bz,
                                                 float *Jx, float *Jy, float *Jz, int *err, const TileBox &tb,
                                                 PackedBounds &bd, float (*q)[32])
{
    constexpr uint32_t step = kTileThreads;
    const int lane = threadIdx.x & 31;
    uint32_t base = p0 + 32u * (threadIdx.x >> 5);
    if (base >= p1) return;   // uniform across the warp
    int qn = 0;
    auto move = [&](const PState &st, uint32_t b) {
        Part Bq;
        uint32_t qa = 0;
        const bool cross = push_one<DIMS, true, XC, XS>(g, p, b + lane, st, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, err, tb,
                                                    bd, Bq, qa);
        const uint32_t m = __ballot_sync(0xffffffffu, cross);
        if (m) {
            const int c = __popc(m);
            if (qn + c > 32) {
                drain_queue<DIMS>(q, qn, tb.jo);
                qn = 0;
            }
            if (cross) {
                const int e = qn + __popc(m & lanemask_lt());
                q[0][e] = Bq.F[0];
                q[1][e] = Bq.F[1];
                q[2][e] = Bq.F[2];
                q[3][e] = Bq.W[0];
                q[4][e] = Bq.W[1];
                q[5][e] = Bq.W[2];
                q[6][e] = __uint_as_float(qa);
                q[7][e] = Bq.D[0];
            }
            qn += c;
        }
    };
    PState cur;
    cur.key = 0;
    if (base + lane < p1) cur = load_state<DIMS>(p, base + lane);
    for (; base < p1; base += step) {
        PState nxt = cur;
        nxt.key = 0;
        if (base + step + lane < p1) nxt = load_state<DIMS>(p, base + step + lane);
        move(cur, base);
        cur = nxt;
    }
    if (qn) drain_queue<DIMS>(q, qn, tb.jo);
}

// Move the particles of brick b (one CTA); PRE: the node averages were
// computed for the whole grid before the launch (bk.nodeA / nodeB); XS: the
// brick belongs to a slab (x not periodic: the box's x cells are the grid's
// own, ghosts included, and x leavers stay in the ghost layer).
template <int DIMS, bool XC, bool PRE = false, bool XS = false>
__device__ __forceinline__ void move_brick(const GridP &g, const PartF32 &p, const Bricks &bk, int b, float *sm,
                                           TileShared &ts, const float *__restrict__ Ex, const float *__restrict__ Ey,
                                           const float *__restrict__ Ez, const float *__restrict__ Bx,
                                           const float *__restrict__ By, const float *__restrict__ Bz, float *Jx,
                                           float *Jy, float *Jz, int *err)
{
    const uint32_t p0 = bk.tile_start[b], p1 = bk.tile_start[b + 1];
    if (p0 >= p1) return;
    TileBox tb;
    int home_lo[3], home_hi[3];
    brick_home<DIMS>(g, bk, b, tb, home_lo, home_hi);
    // a move is below c per axis; the box is the stored bounds (no margin)
    tile_setup<DIMS, !XS, false, PRE>(g, bk, b, p1 - p0, 0, g.c_f, sm, ts, tb, home_lo, home_hi, Ex, Ey, Ez, Bx, By,
                                      Bz);
    PackedBounds bd;
    bd.init();
    push_range_tiled<DIMS, XC, XS>(g, p, p0, p1, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, err, tb, bd,
                                   ts.s_q[threadIdx.x >> 5]);
    __syncthreads();
    tile_finish<DIMS, !XS>(g, bk, b, tb, sm, ts, bd.unpack(), home_lo, home_hi, Jx, Jy, Jz);
}

}  // namespace pic
