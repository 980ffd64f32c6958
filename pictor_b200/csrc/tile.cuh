// tile.cuh -- the shared-memory boxes of a brick, used by the tiled FP32
// movers (mover_f32.cu: Cartesian; cyl.cu: cylindrical).
//
// A CTA moves the particles of one brick (bricks.cu groups them).  It stages
// the node-averaged E and B of a box of cells around the brick in shared
// memory (each node once per brick instead of 8 times per particle; the
// Cartesian mover reads them from node arrays that one pass over the grid
// fills before the move, the cylindrical one averages them itself with
// node_avg) and sums the brick's current in a shared box of fixed-point
// words (32-bit; 64-bit for the cylindrical form, whose weights span the
// radius), added to the global J once at the end.  The box is the
// bounding box, in cells relative to the brick centre and unwrapped across
// periodic boundaries, of where the brick's particles were after the
// previous step (Bricks::box, rewritten by the mover for the next step); a
// box too large for shared memory falls back to the brick plus one cell.
#pragma once

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
    A.x = (ldro(Ex + nd - 1) + ldro(Ex + nd)) * 0.5f;
    A.y = (ldro(Ey + nd - sy) + ldro(Ey + nd)) * 0.5f;
    if (DIMS == 3) {
        A.z = (ldro(Ez + nd - sz) + ldro(Ez + nd)) * 0.5f;
        A.w = (((ldro(Bx + nd - sy - sz) + ldro(Bx + nd - sz)) + ldro(Bx + nd - sy)) + ldro(Bx + nd)) * 0.25f + b0;
        Bv.x = (((ldro(By + nd - 1 - sz) + ldro(By + nd - 1)) + ldro(By + nd - sz)) + ldro(By + nd)) * 0.25f + b1;
    } else {
        A.z = ldro(Ez + nd);
        A.w = (ldro(Bx + nd - sy) + ldro(Bx + nd)) * 0.5f + b0;
        Bv.x = (ldro(By + nd - 1) + ldro(By + nd)) * 0.5f + b1;
    }
    Bv.y = (((ldro(Bz + nd - 1 - sy) + ldro(Bz + nd - 1)) + ldro(Bz + nd - sy)) + ldro(Bz + nd)) * 0.25f + b2;
}

// Packed FP32 pair arithmetic of sm_100 (one instruction for two lanes of
// IEEE single precision, each rounded as the scalar operation would be).
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c)
{
    float2 d;
    asm("{.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %5};\n\t"
        "mov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\t"
        "mov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

__device__ __forceinline__ float2 fmul2(float2 a, float2 b)
{
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\t"
        "mov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 fadd2(float2 a, float2 b)
{
    float2 d;
    asm("{.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\t"
        "mov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

// pE += w * (E at a node), pB += w * (B at a node): the interpolation sums
// of movdep.F90:116-129, three packed FMAs (the same roundings as six fmaf).
__device__ __forceinline__ void accum(float w, const float4 &A, const float2 &Bv, float pE[3], float pB[3])
{
    const float2 ww = make_float2(w, w);
    const float2 a = ffma2(make_float2(A.x, A.y), ww, make_float2(pE[0], pE[1]));
    const float2 b = ffma2(make_float2(A.z, A.w), ww, make_float2(pE[2], pB[0]));
    const float2 c = ffma2(Bv, ww, make_float2(pB[1], pB[2]));
    pE[0] = a.x;
    pE[1] = a.y;
    pE[2] = b.x;
    pB[0] = b.y;
    pB[1] = c.x;
    pB[2] = c.y;
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

// Shared-memory accesses with explicit .shared addressing (32-bit shared
// addresses), so no generic-address resolution is left to run time.
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
template <int OFF>
__device__ __forceinline__ float4 lds4i(uint32_t a)
{
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4+%5];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"(a), "n"(OFF));
    return v;
}
template <int OFF>
__device__ __forceinline__ float2 lds2i(uint32_t a)
{
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2+%3];" : "=f"(v.x), "=f"(v.y) : "r"(a), "n"(OFF));
    return v;
}
template <int OFF>
__device__ __forceinline__ void red_shared_i(uint32_t a, int v)
{
    asm volatile("red.shared.add.s32 [%0+%1], %2;" ::"r"(a), "n"(OFF), "r"(v));
}
// q added to the 64-bit shared word at a + OFF with two native 32-bit
// atomics: the low halves (the old value comes back), then the high halves
// with the carry out of the low word.  Every add's carry is counted once, so
// the word holds the exact sum of everything added (mod 2^64) once the adds
// are done; a 64-bit add on shared memory is not a single native atomic.
template <int OFF>
__device__ __forceinline__ void red_shared_l(uint32_t a, long long q)
{
    const unsigned lo = (unsigned)(unsigned long long)q, hi = (unsigned)((unsigned long long)q >> 32);
    unsigned old;
    asm volatile("atom.shared.add.u32 %0, [%1+%2], %3;" : "=r"(old) : "r"(a), "n"(OFF), "r"(lo) : "memory");
    const unsigned h = hi + (old + lo < old ? 1u : 0u);
    if (h) asm volatile("red.shared.add.u32 [%0+%1], %2;" ::"r"(a), "n"(OFF + 4), "r"(h) : "memory");
}

// Shared byte offsets of the current box: component planes and the y / z
// strides (the x stride is 4 bytes, an immediate).
struct JOff {
    uint32_t cy, cz;      // Jy, Jz plane - Jx plane
    uint32_t y, z, yz;    // 4 JX, 4 JXY, 4 (JX + JXY)
};

// round(v) for |v| <= 2^22, v already scaled by the box's fixed-point scale:
// adding 1.5 * 2^23 leaves the rounded integer in the low mantissa bits.
__device__ __forceinline__ int fixed_round(float v)
{
    return __float_as_int(v + 12582912.f) - 0x4B400000;
}
// The same for a pair, with one packed add.
__device__ __forceinline__ int2 fixed_round2(float a, float b)
{
    const float2 t = fadd2(make_float2(a, b), make_float2(12582912.f, 12582912.f));
    return make_int2(__float_as_int(t.x) - 0x4B400000, __float_as_int(t.y) - 0x4B400000);
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
    uint32_t oY4, oZ4;  // node-box byte strides of the 16-byte nodes (8-byte nodes: half)
    JOff jo;            // current-box byte offsets
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
    s.key = ldco(p.key + n);
    s.dx = ldco(p.dx + n);
    s.dy = ldco(p.dy + n);
    s.dz = DIMS == 3 ? ldco(p.dz + n) : 0.f;
    s.ux = ldco(p.ux + n);
    s.uy = ldco(p.uy + n);
    s.uz = ldco(p.uz + n);
    s.w = ldco(p.w + n);
    return s;
}

constexpr int kTileThreads = 256;
constexpr int kTileWarps = kTileThreads / 32;

// Second zigzag segments queued by the lanes of one warp (structure of
// arrays: F x, y, z, W x, y, z, box address, cross term; 32 entries each).
constexpr int kQueueRows = 8;

// Interior index of the unwrapped 1-based index a (no division when a is
// already interior or one period away).
__device__ __forceinline__ int interior_of(int a, int n)
{
    if (a < 3) a += n;
    else if (a > n + 2) a -= n;
    if (a < 3 || a > n + 2) a = wrap_interior(a, n);
    return a;
}

// Static shared memory of one brick's move (the node and current boxes are
// the dynamic part, sm).
struct TileShared {
    int red[kTileWarps][6];
    int s_off[3][kBoxAxisMax + 3];
    float s_q[kTileWarps][kQueueRows][32];
};

// Centre of brick b (tb.hc, 1-based interior indices) and its cells relative
// to the centre.
template <int DIMS>
__device__ __forceinline__ void brick_home(const GridP &g, const Bricks &bk, int b, TileBox &tb, int home_lo[3],
                                           int home_hi[3])
{
    const int bx = b % bk.nb[0], byz = b / bk.nb[0], by = byz % bk.nb[1], bz = byz / bk.nb[1];
    const int n3[3] = {g.nx, g.ny, g.nz};
    const int bi[3] = {bx, by, bz};
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
}

// The boxes of brick b for this step (one CTA, ends with a barrier): the
// stored bounds widened by `margin` cells on each side (movers that gather a
// second time at the cell they move to), or the brick +- 1 cell when that is
// too large; strides and byte offsets; the fixed-point scale for the n
// particles of the brick, whose moves are below dmax cells per axis (current
// words of 32 bits, or 64 with WIDE); the
// memory offsets of the box cells along each axis (the periodic interior
// image, or along a non-periodic x axis (XPER false: the radius of the
// cylindrical form) the index itself); the current box zeroed and the
// node-averaged fields staged.
template <int DIMS, bool XPER, bool WIDE = false, bool PRE = false>
__device__ __forceinline__ void tile_setup(const GridP &g, const Bricks &bk, int b, uint32_t n, int margin, float dmax,
                                           float *sm, TileShared &ts, TileBox &tb, const int home_lo[3],
                                           const int home_hi[3], const float *__restrict__ Ex,
                                           const float *__restrict__ Ey, const float *__restrict__ Ez,
                                           const float *__restrict__ Bx, const float *__restrict__ By,
                                           const float *__restrict__ Bz)
{
    const int tid = threadIdx.x;
    const int n3[3] = {g.nx, g.ny, g.nz};
    const int *sb = bk.box + 8 * (size_t)b;
    int lo[3] = {ldco(sb) - margin, ldco(sb + 1) - margin, DIMS == 3 ? ldco(sb + 2) - margin : 0};
    int hi[3] = {ldco(sb + 3) + margin, ldco(sb + 4) + margin, DIMS == 3 ? ldco(sb + 5) + margin : 0};
    if (hi[0] < lo[0] || hi[1] < lo[1] || hi[2] < lo[2] || hi[0] - lo[0] >= kBoxAxisMax ||
        hi[1] - lo[1] >= kBoxAxisMax || hi[2] - lo[2] >= kBoxAxisMax ||
        box_floats(DIMS, hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1, WIDE ? 2 : 1) > bk.smem_floats) {
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
    const int NXn = tb.C[0] + 1, NY = tb.C[1] + 1, NZ = DIMS == 3 ? tb.C[2] + 1 : 1;
    const int JX = tb.C[0] + 3, JY = tb.C[1] + 3, JZ = DIMS == 3 ? tb.C[2] + 3 : 1;
    // node rows padded to 8 mod 16 words of 16 / 8 bytes when the box still
    // fits: the quarter-warps of the 16-byte gathers and the half-warps of
    // the 8-byte ones then see the lanes of two y rows on disjoint banks (the
    // lanes of a warp hold neighbouring cells of 4 rows of an 8-wide brick)
    int NX = NXn;
    if (DIMS == 3) {
        const int NXp = NXn + ((8 - NXn) & 15);
        if (6ll * NXp * NY * NZ + (WIDE ? 6ll : 3ll) * JX * JY * JZ <= (long long)bk.smem_floats) NX = NXp;
    }
    const int nnode = NX * NY * NZ;
    tb.NX = NX;
    tb.NXY = NX * NY;
    tb.JX = JX;
    tb.JXY = JX * JY;
    tb.njc = JX * JY * JZ;
    tb.oY4 = 16u * (uint32_t)NX;
    tb.oZ4 = 16u * (uint32_t)(NX * NY);
    constexpr uint32_t wb = WIDE ? 8u : 4u;   // bytes per current word
    tb.jo.cy = wb * (uint32_t)tb.njc;
    tb.jo.cz = 2u * wb * (uint32_t)tb.njc;
    tb.jo.y = wb * (uint32_t)JX;
    tb.jo.z = wb * (uint32_t)tb.JXY;
    tb.jo.yz = tb.jo.y + tb.jo.z;
    float4 *nA = reinterpret_cast<float4 *>(sm);
    float2 *nB = reinterpret_cast<float2 *>(sm + 4 * nnode);
    int *sJ = reinterpret_cast<int *>(sm + 6 * nnode);
    tb.nA = smem_addr(nA);
    tb.nB = smem_addr(nB);
    tb.sJ = smem_addr(sJ);
    // fixed-point scale: a particle adds at most b = |w| qi dmax to any entry,
    // so with S = 2^30 / (N b) no sum of the N particles exceeds 2^30;
    // S <= 2^22 / b keeps each contribution below 2^22 (the range of
    // fixed_round).  64-bit words: S = 2^62 / (N b), each contribution an
    // FP32 value rounded to an integer of up to 2^54, the sums exact.
    {
        const float b1 = dmax * g.qi_f * __uint_as_float(ldco(bk.wmax_bits));
        const float nf = fmaxf((float)n, 256.f);
        tb.S = b1 > 0.f ? (WIDE ? 4.611686018427388e18f : 1073741824.f) / (b1 * nf) : 1.f;
    }
    // offsets of the box cells lo-1 .. lo+C+1 along each axis (memory offset
    // of the interior image, times the axis stride)
    {
        const int ext[3] = {JX, JY, JZ};
        const int str[3] = {1, (int)g.sy, (int)g.sz};
#pragma unroll
        for (int d = 0; d < DIMS; d++)
            for (int t = tid; t < ext[d]; t += kTileThreads) {
                const int a = tb.hc[d] + lo[d] - 1 + t;
                ts.s_off[d][t] = ((XPER || d > 0 ? interior_of(a, n3[d]) : a) - 1) * str[d];
            }
        if (DIMS == 2 && tid == 0) ts.s_off[2][0] = 0;
    }
    for (int q = tid; q < (WIDE ? 6 : 3) * tb.njc; q += kTileThreads) sJ[q] = 0;
    __syncthreads();
    // stage node-averaged fields: node q = xx + NX*(yy + NY*zz) over the
    // padded rows, the padding skipped (the threads of a warp then load one
    // or two rows of the box; walking the real nodes densely spread a warp
    // over three rows, its loads read 42 % more from L2 and the mover took
    // 23 % longer); q/NX and r/NY by multiply-high (exact for q < 2^16, NX,
    // NY < 2^16)
    {
        const int sy = (int)g.sy, sz = (int)g.sz;
        const uint32_t mX = 0xffffffffu / (uint32_t)NX + 1u, mY = 0xffffffffu / (uint32_t)NY + 1u;
        for (int q = tid; q < nnode; q += kTileThreads) {
            const int r = (int)__umulhi((uint32_t)q, mX), xx = q - r * NX;
            if (xx >= NXn) continue;   // row padding
            const int zz = (int)__umulhi((uint32_t)r, mY), yy = r - zz * NY;
            const int nd = ts.s_off[0][xx + 1] + ts.s_off[1][yy + 1] + (DIMS == 3 ? ts.s_off[2][zz + 1] : 0);
            float4 A;
            float2 Bv;
            if (PRE) {
                A = ldro(bk.nodeA + nd);
                Bv = ldro(bk.nodeB + nd);
            } else {
                node_avg<DIMS>(Ex, Ey, Ez, Bx, By, Bz, nd, sy, sz, g.bext_f[0], g.bext_f[1], g.bext_f[2], A, Bv);
            }
            nA[q] = A;
            nB[q] = Bv;
        }
    }
    __syncthreads();
}

// After the brick's particles moved (and a barrier): the box current added
// to global J at the offsets of tile_setup (FP32 reductions), and the bounds
// of the particles' new cells stored as the box of the next step (the brick
// itself if no particle is left).
template <int DIMS, bool XPER, bool WIDE = false>
__device__ __forceinline__ void tile_finish(const GridP &g, const Bricks &bk, int b, const TileBox &tb, float *sm,
                                            TileShared &ts, const Bounds &bd, const int home_lo[3],
                                            const int home_hi[3], float *Jx, float *Jy, float *Jz)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nnode = tb.NXY * (DIMS == 3 ? tb.C[2] + 1 : 1);
    {
        const int JX = tb.JX, JY = tb.C[1] + 3;
        const uint32_t mX = 0xffffffffu / (uint32_t)JX + 1u, mY = 0xffffffffu / (uint32_t)JY + 1u;
        const int *sJ = reinterpret_cast<const int *>(sm + 6 * nnode);
        const long long *sJ8 = reinterpret_cast<const long long *>(sm + 6 * nnode);
        const float inv = 1.f / tb.S;
        const double inv8 = 1.0 / (double)tb.S;
        for (int q = tid; q < tb.njc; q += kTileThreads) {
            const int r = (int)__umulhi((uint32_t)q, mX), xx = q - r * JX;
            const int zz = (int)__umulhi((uint32_t)r, mY), yy = r - zz * JY;
            const int off = ts.s_off[0][xx] + ts.s_off[1][yy] + (DIMS == 3 ? ts.s_off[2][zz] : 0);
            if (WIDE) {
                const long long vx = sJ8[q], vy = sJ8[tb.njc + q], vz = sJ8[2 * tb.njc + q];
                if (vx != 0) atomicAdd(Jx + off, (float)((double)vx * inv8));
                if (vy != 0) atomicAdd(Jy + off, (float)((double)vy * inv8));
                if (vz != 0) atomicAdd(Jz + off, (float)((double)vz * inv8));
            } else {
                const int vx = sJ[q], vy = sJ[tb.njc + q], vz = sJ[2 * tb.njc + q];
                if (vx != 0) atomicAdd(Jx + off, (float)vx * inv);
                if (vy != 0) atomicAdd(Jy + off, (float)vy * inv);
                if (vz != 0) atomicAdd(Jz + off, (float)vz * inv);
            }
        }
    }
    int v[6] = {bd.lo[0], bd.lo[1], bd.lo[2], -bd.hi[0], -bd.hi[1], -bd.hi[2]};
#pragma unroll
    for (int e = 0; e < 6; e++) v[e] = __reduce_min_sync(0xffffffffu, v[e]);
    if (lane == 0)
#pragma unroll
        for (int e = 0; e < 6; e++) ts.red[warp][e] = v[e];
    __syncthreads();
    if (tid == 0) {
        int m[6];
        for (int e = 0; e < 6; e++) {
            m[e] = ts.red[0][e];
            for (int w2 = 1; w2 < kTileWarps; w2++) m[e] = min(m[e], ts.red[w2][e]);
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

// E and B interpolated with weights wt from the node box at box cell nb
// (movdep.F90:116-129 on the staged nodes), added to pE, pB: the corner rows
// (y, z) by register offsets, the x neighbour by an immediate.
template <int DIMS>
__device__ __forceinline__ void gather_box(const TileBox &tb, int nb, const float wt[8], float pE[3], float pB[3])
{
    const uint32_t a0 = tb.nA + 16u * (uint32_t)nb, b0 = tb.nB + 8u * (uint32_t)nb;
    const uint32_t a1 = a0 + tb.oY4, b1 = b0 + (tb.oY4 >> 1);
    accum(wt[0], lds4i<0>(a0), lds2i<0>(b0), pE, pB);
    accum(wt[1], lds4i<16>(a0), lds2i<8>(b0), pE, pB);
    accum(wt[2], lds4i<0>(a1), lds2i<0>(b1), pE, pB);
    accum(wt[3], lds4i<16>(a1), lds2i<8>(b1), pE, pB);
    if (DIMS == 3) {
        const uint32_t a2 = a0 + tb.oZ4, b2 = b0 + (tb.oZ4 >> 1);
        const uint32_t a3 = a1 + tb.oZ4, b3 = b1 + (tb.oZ4 >> 1);
        accum(wt[4], lds4i<0>(a2), lds2i<0>(b2), pE, pB);
        accum(wt[5], lds4i<16>(a2), lds2i<8>(b2), pE, pB);
        accum(wt[6], lds4i<0>(a3), lds2i<0>(b3), pE, pB);
        accum(wt[7], lds4i<16>(a3), lds2i<8>(b3), pE, pB);
    }
}

// The 12 VecJ entries v of a 3D cell (in fixed-point units, FP32) into a
// current box of 64-bit words at byte address a, each rounded to the nearest
// integer (the layout of red_entries_box).
__device__ __forceinline__ void red_entries_box_wide(uint32_t a, const JOff &o, const float v[12])
{
    red_shared_l<0>(a, __float2ll_rn(v[0]));
    red_shared_l<0>(a + o.y, __float2ll_rn(v[1]));
    red_shared_l<0>(a + o.z, __float2ll_rn(v[2]));
    red_shared_l<0>(a + o.yz, __float2ll_rn(v[3]));
    const uint32_t b = a + o.cy;
    red_shared_l<0>(b, __float2ll_rn(v[4]));
    red_shared_l<8>(b, __float2ll_rn(v[5]));
    const uint32_t bz = b + o.z;
    red_shared_l<0>(bz, __float2ll_rn(v[6]));
    red_shared_l<8>(bz, __float2ll_rn(v[7]));
    const uint32_t c = a + o.cz;
    red_shared_l<0>(c, __float2ll_rn(v[8]));
    red_shared_l<8>(c, __float2ll_rn(v[9]));
    const uint32_t cy = c + o.y;
    red_shared_l<0>(cy, __float2ll_rn(v[10]));
    red_shared_l<8>(cy, __float2ll_rn(v[11]));
}

// VecJ entries v (already in fixed-point units, FP32) into the current box
// at byte address a (the cell's Jx word): 3D 0..3 Jx at (y,z) corners, 4..7
// Jy at (x,z), 8..11 Jz at (x,y); 2D 0..1 Jx, 2..3 Jy, 4..7 Jz.
template <int DIMS>
__device__ __forceinline__ void red_entries_box(uint32_t a, const JOff &o, const float v[12])
{
    if (DIMS == 3) {
        const int2 r01 = fixed_round2(v[0], v[1]), r23 = fixed_round2(v[2], v[3]);
        const int2 r45 = fixed_round2(v[4], v[5]), r67 = fixed_round2(v[6], v[7]);
        const int2 r89 = fixed_round2(v[8], v[9]), rab = fixed_round2(v[10], v[11]);
        red_shared_i<0>(a, r01.x);
        red_shared_i<0>(a + o.y, r01.y);
        red_shared_i<0>(a + o.z, r23.x);
        red_shared_i<0>(a + o.yz, r23.y);
        const uint32_t b = a + o.cy;
        red_shared_i<0>(b, r45.x);
        red_shared_i<4>(b, r45.y);
        const uint32_t bz = b + o.z;
        red_shared_i<0>(bz, r67.x);
        red_shared_i<4>(bz, r67.y);
        const uint32_t c = a + o.cz;
        red_shared_i<0>(c, r89.x);
        red_shared_i<4>(c, r89.y);
        const uint32_t cy = c + o.y;
        red_shared_i<0>(cy, rab.x);
        red_shared_i<4>(cy, rab.y);
    } else {
        red_shared_i<0>(a, fixed_round(v[0]));
        red_shared_i<0>(a + o.y, fixed_round(v[1]));
        const uint32_t b = a + o.cy;
        red_shared_i<0>(b, fixed_round(v[2]));
        red_shared_i<4>(b, fixed_round(v[3]));
        const uint32_t c = a + o.cz;
        red_shared_i<0>(c, fixed_round(v[4]));
        red_shared_i<4>(c, fixed_round(v[5]));
        const uint32_t cy = c + o.y;
        red_shared_i<0>(cy, fixed_round(v[6]));
        red_shared_i<4>(cy, fixed_round(v[7]));
    }
}

}  // namespace pic
