// tile64.cuh -- one CTA per tile of cells for the FP64 movers in the
// reference layout (Cartesian: mover_f64_tiled.cu; cylindrical: cyl.cu),
// for the steps after a reorder.
//
// After the FP64 reorder (ReorderPrtlArr, mem_prtl.F90:166-301) the
// particles are in cell order, so the particles of W consecutive cells of
// one row occupy one contiguous slot range.  A tile is H such row segments
// (x in [1 + sx W, 1 + (sx+1) W), rows j0 .. j0 + H - 1 of one plane k, over
// the whole ghosted grid): H slot ranges.  move_tile64 is the CTA's part
// that does not depend on the geometry:
//   * it stages the node-averaged E and B (the values of GatherVecEfld /
//     GatherVecBfld, movdep_routines.F90:6-223, in the expressions and order
//     of the per-particle gathers, so interpolated fields, and with them
//     positions and momenta, equal the per-particle movers' bit for bit) of
//     the box of cells the tile's particles occupy, widened by MARGIN cells,
//     in shared memory;
//   * it sums the tile's current in a 64-bit fixed-point box in shared memory
//     and adds the box to J once with FP64 atomics, instead of 16 / 24
//     global FP64 atomics per particle;
//   * it hands every particle to the geometry's body, with the boxes, and
//     records the cells its particles move to, which bound the box of the
//     next step (the particles drift out of their tile between reorders).
// The current differs from a per-particle mover's only in the order of its
// sums and the fixed-point rounding of each contribution.  A tile whose box
// does not fit in shared memory takes its own cells plus one on each side;
// a particle whose cells lie outside the box gathers and deposits through
// global memory with the same arithmetic.
#pragma once

#include "common.cuh"
#include "kernels.cuh"
#include "particle_math.cuh"

namespace pic {

constexpr int kT64Threads = 256;   // 8 warps: the item order below covers 256 items

// Tile t -> its row segments: cells x0 .. x1 - 1 (1-based) of rows j0 ..
// j0 + nrow - 1 in planes k0 .. k0 + nk - 1 (segment p H + r: row j0 + r of
// plane k0 + p).  The tiles cover every cell of the ghosted
// grid, not only the interior: the exchange sends a particle that left
// through an edge or a corner through one face per step (the diagonal-face
// rule of LoadPrtlOutliers), so a reorder can find it in a ghost cell, and
// it must still belong to a tile (the range check of the move raises
// PIC_ERR_RANGE for a cell outside the ghost frame, before any access).
__host__ __device__ inline int tile_row_groups(const GridP &g, const Tiles64 &T)
{
    return 1 + (g.my - T.jfirst + T.H - 1) / T.H;
}
__device__ __forceinline__ void tile_cells(const GridP &g, const Tiles64 &T, int t, int &x0, int &x1, int &j0,
                                           int &nrow, int &k0, int &nk)
{
    const int sx = t % T.nsx, r = t / T.nsx;
    const int nry = tile_row_groups(g, T);
    x0 = 1 + sx * T.W;
    x1 = min(x0 + T.W, g.mx + 1);
    const int ry = r % nry;
    j0 = ry == 0 ? 1 : 1 + T.jfirst + (ry - 1) * T.H;
    nrow = max(0, min(ry == 0 ? T.jfirst : T.H, g.my + 1 - j0));
    if (g.dims == 3) {
        k0 = 1 + (r / nry) * T.D;
        nk = min(T.D, g.mz + 1 - k0);
    } else {
        k0 = 1;
        nk = 1;
    }
}

struct Box64 {
    int lo[3], C[3];      // node box cells: lo .. lo + C - 1 per axis (z: 1 cell in 2D)
    int NX, NXY;          // node strides (C + 1 per axis)
    int jlo[3], jC[3];    // current box cells jlo .. jlo + jC - 1: the node box without its margin
    int JX, JXY, nj;      // current strides (jC + 3 per axis) and words per component
};

template <int DIMS>
__device__ __forceinline__ bool in_box(const Box64 &bx, int i, int j, int k, int &nb)
{
    const int a = i - bx.lo[0], b = j - bx.lo[1], c = DIMS == 3 ? k - bx.lo[2] : 0;
    nb = a + bx.NX * b + bx.NXY * c;
    return (unsigned)a < (unsigned)bx.C[0] && (unsigned)b < (unsigned)bx.C[1] && (DIMS == 2 || (unsigned)c < (unsigned)bx.C[2]);
}

// gather() on the staged nodes: node q of the box holds the 6 node values of
// GatherVecEfld / GatherVecBfld; the corner sums run in the same order.
template <int DIMS>
__device__ __forceinline__ void gather_box64(const Box64 &bx, const double *sN, int nb, const double *wt, double pE[3],
                                             double pB[3])
{
    pE[0] = pE[1] = pE[2] = pB[0] = pB[1] = pB[2] = 0.0;
#pragma unroll
    for (int nn = 0; nn < (DIMS == 3 ? 8 : 4); nn++) {
        const int q = nb + (nn & 1) + ((nn >> 1) & 1) * bx.NX + ((nn >> 2) & 1) * bx.NXY;
        const double2 a = *reinterpret_cast<const double2 *>(sN + 6 * q);
        const double2 b = *reinterpret_cast<const double2 *>(sN + 6 * q + 2);
        const double2 c = *reinterpret_cast<const double2 *>(sN + 6 * q + 4);
        pE[0] = pE[0] + wt[nn] * a.x;
        pE[1] = pE[1] + wt[nn] * a.y;
        pE[2] = pE[2] + wt[nn] * b.x;
        pB[0] = pB[0] + wt[nn] * b.y;
        pB[1] = pB[1] + wt[nn] * c.x;
        pB[2] = pB[2] + wt[nn] * c.y;
    }
}

// An FP64 value already multiplied by the box's scale, rounded to the
// nearest integer: adding 1.5 * 2^52 leaves it in the low mantissa bits
// (exact for |v| < 2^51).
__device__ __forceinline__ long long fixed64(double v)
{
    return __double_as_longlong(v + 6755399441055744.0) - 0x4338000000000000ll;
}

// q added to the 64-bit word w of the fixed-point box with two native 32-bit
// shared-memory atomics: the low halves, then the high halves with the carry
// out of the low word, which the add that wrapped it sees in the old value
// it gets back.  The word then holds the exact sum of every q added (mod 2^64;
// the scale keeps the sums far inside the signed range).
__device__ __forceinline__ void add_fixed64(unsigned long long *w, long long q)
{
    unsigned *p = reinterpret_cast<unsigned *>(w);
    const unsigned lo = (unsigned)(unsigned long long)q, hi = (unsigned)((unsigned long long)q >> 32);
    const unsigned old = atomicAdd(p, lo);
    const unsigned h = hi + (old + lo < old ? 1u : 0u);
    if (h) atomicAdd(p + 1, h);
}

// The VecJ entries o of a cell whose box current cell is jb, added into the
// fixed-point box (the scatter offsets of movdep_routines.F90:276-303): each
// entry times the scale S rounded to an integer.
template <int DIMS>
__device__ __forceinline__ void deposit_box64(const Box64 &bx, unsigned long long *sJ, int jb, const double *o,
                                              double S)
{
    unsigned long long *jx = sJ + jb, *jy = sJ + bx.nj + jb, *jz = sJ + 2 * bx.nj + jb;
    const int oy = bx.JX, oz = bx.JXY;
    auto add = [&](unsigned long long *a, double v) { add_fixed64(a, fixed64(v * S)); };
    if (DIMS == 2) {
        add(jx, o[0]);
        add(jx + oy, o[1]);
        add(jy, o[2]);
        add(jy + 1, o[3]);
        add(jz, o[4]);
        add(jz + 1, o[5]);
        add(jz + oy, o[6]);
        add(jz + 1 + oy, o[7]);
    } else {
        add(jx, o[0]);
        add(jx + oy, o[1]);
        add(jx + oz, o[2]);
        add(jx + oy + oz, o[3]);
        add(jy, o[4]);
        add(jy + 1, o[5]);
        add(jy + oz, o[6]);
        add(jy + 1 + oz, o[7]);
        add(jz, o[8]);
        add(jz + 1, o[9]);
        add(jz + oy, o[10]);
        add(jz + 1 + oy, o[11]);
    }
}

// One particle's state in the reference layout.
struct P64 {
    double q, x, y, z, u, v, w;
    int flv;
};
__device__ __forceinline__ P64 load_p64(const PartF64 &p, uint32_t n)
{
    P64 s;
    s.flv = p.flv[n];
    s.q = p.q[n];
    s.x = p.x[n];
    s.y = p.y[n];
    s.z = p.z[n];
    s.u = p.u[n];
    s.v = p.v[n];
    s.w = p.w[n];
    return s;
}

// The boxes of a tile as the per-particle body sees them.
struct Tile64Ctx {
    Box64 bx;
    const double *sN;        // 6 node values per box node
    unsigned long long *sJ;  // fixed-point current, 3 components of bx.nj words
    double S;                // fixed-point scale
    bool use_box;
    // box current cell of cell (i, j, k) of the current box
    template <int DIMS>
    __device__ __forceinline__ int jcell(int i, int j, int k) const
    {
        return (i - bx.jlo[0] + 1) + bx.JX * (j - bx.jlo[1] + 1) + (DIMS == 3 ? bx.JXY * (k - bx.jlo[2] + 1) : 0);
    }
    // cell (i, j, k) lies in the current box (its deposit's words then do)
    template <int DIMS>
    __device__ __forceinline__ bool in_jbox(int i, int j, int k) const
    {
        return (unsigned)(i - bx.jlo[0]) < (unsigned)bx.jC[0] && (unsigned)(j - bx.jlo[1]) < (unsigned)bx.jC[1] &&
               (DIMS == 2 || (unsigned)(k - bx.jlo[2]) < (unsigned)bx.jC[2]);
    }
};

// The CTA's work on tile blockIdx.x (see the file comment).  body(s, n, ctx,
// nc) moves the particle s of slot n and returns true with its new cell in
// nc when that cell bounds the next box.  MARGIN widens the staged box by
// cells on each side (a body that gathers at the moved position too); bound
// is the largest VecJ entry a particle of charge q adds to one word, over
// q qi.  The current box covers the cells of the box without MARGIN (the
// start cells; a deposit beyond them by one cell lands in its +-1 frame).
// Shared memory: T.smem_bytes dynamic; smem64 the dynamic array.
template <int DIMS, int MARGIN, class Body>
__device__ __forceinline__ void move_tile64(const GridP &g, const PartF64 &p, const Tiles64 &T,
                                            const double *__restrict__ Ex, const double *__restrict__ Ey,
                                            const double *__restrict__ Ez, const double *__restrict__ Bx,
                                            const double *__restrict__ By, const double *__restrict__ Bz,
                                            double *Jx, double *Jy, double *Jz, double bound, double *smem64,
                                            Body &&body)
{
    __shared__ int s_red[kT64Threads / 32][6];
    __shared__ uint32_t s_rg[2 * kTile64MaxRows];
    const int t = blockIdx.x, tid = threadIdx.x;
    const int nseg = T.H * T.D;
    if (tid < 2 * nseg) s_rg[tid] = T.range[2 * (size_t)nseg * t + tid];
    __syncthreads();
    // the tile's particles: item i -> slot, over the H D ranges in order
    uint32_t total = 0;
    for (int r = 0; r < nseg; r++) total += s_rg[2 * r + 1] - s_rg[2 * r];
    if (total == 0) return;   // uniform across the CTA
    int *gbox = T.box + 8 * (size_t)t;
    Tile64Ctx ctx;
    Box64 &bx = ctx.bx;
    int lo[3] = {gbox[0] - MARGIN, gbox[1] - MARGIN, DIMS == 3 ? gbox[2] - MARGIN : 1};
    int hi[3] = {gbox[3] + MARGIN, gbox[4] + MARGIN, DIMS == 3 ? gbox[5] + MARGIN : 1};
    int margin = MARGIN;
    auto set_box = [&]() {
        for (int d = 0; d < 3; d++) {
            const int m = (DIMS == 2 && d == 2) ? 0 : margin;
            bx.lo[d] = lo[d];
            bx.C[d] = hi[d] - lo[d] + 1;
            bx.jlo[d] = lo[d] + m;
            bx.jC[d] = bx.C[d] - 2 * m;
        }
        bx.NX = bx.C[0] + 1;
        bx.NXY = bx.NX * (bx.C[1] + 1);
        bx.JX = bx.jC[0] + 3;
        bx.JXY = bx.JX * (bx.jC[1] + 3);
        bx.nj = bx.JXY * (DIMS == 3 ? bx.jC[2] + 3 : 1);
        return bx.NXY * (DIMS == 3 ? bx.C[2] + 1 : 1);
    };
    auto fits = [&](int nn) {
        return bx.jC[0] >= 1 && bx.jC[1] >= 1 && bx.jC[2] >= 1 && lo[0] >= 2 && hi[0] <= g.mx - 2 && lo[1] >= 2 &&
               hi[1] <= g.my - 2 && (DIMS == 2 || (lo[2] >= 2 && hi[2] <= g.mz - 2)) &&
               8ll * (6ll * nn + 3ll * bx.nj) <= (long long)T.smem_bytes;
    };
    int nnode = set_box();
    if (!fits(nnode)) {
        // the particles spread further than shared memory holds: the tile's
        // own cells plus one on each side (clamped to the ghost frame), the
        // particles beyond it through global memory
        int x0, x1, j0, nrow, k0, nk;
        tile_cells(g, T, t, x0, x1, j0, nrow, k0, nk);
        lo[0] = max(x0 - 1, 2); hi[0] = min(x1, g.mx - 2);
        lo[1] = max(j0 - 1, 2); hi[1] = min(j0 + nrow, g.my - 2);
        if (DIMS == 3) { lo[2] = max(k0 - 1, 2); hi[2] = min(k0 + nk, g.mz - 2); }
        margin = 0;   // the current box is the node box here
        nnode = set_box();
    }
    // the box fits (and lies where the kernel may read and write) or the
    // tile's particles all take the global path
    ctx.use_box = fits(nnode);
    double *sN = smem64;
    unsigned long long *sJ = reinterpret_cast<unsigned long long *>(smem64 + 6 * (ctx.use_box ? nnode : 0));
    ctx.sN = sN;
    ctx.sJ = sJ;
    // fixed-point scale of the current box: a particle adds at most
    // b = max|q| qi bound to a word, so with S <= 2^62 / (N b) no sum of
    // the tile's N particles leaves the signed range, and S <= 2^50 / b
    // keeps every product within the range of fixed64; one unit is then at
    // most 2^-50 of b (and N 2^-62 of it for N > 4096), far below the FP64
    // rounding of J
    ctx.S = 1.0;
    {
        const double b = __longlong_as_double((long long)*T.qmax) * g.qi * bound;
        if (b > 0.0) ctx.S = 1125899906842624.0 / b * (total > 4096u ? 4096.0 / (double)total : 1.0);
    }
    if (ctx.use_box) {
        const long long sy = g.sy, sz = g.sz;
        for (int q = tid; q < 3 * bx.nj; q += kT64Threads) sJ[q] = 0ull;
        for (int q = tid; q < nnode; q += kT64Threads) {
            const int a = q % bx.NX, r = q / bx.NX, b = r % (bx.C[1] + 1), c = r / (bx.C[1] + 1);
            const long long nd = cidx(g, lo[0] + a, lo[1] + b, DIMS == 3 ? lo[2] + c : 1);
            double *v = sN + 6 * q;
            // the node values of gather() (GatherVecEfld / GatherVecBfld)
            v[0] = (__ldg(Ex + nd - 1) + __ldg(Ex + nd)) * 0.5;
            v[1] = (__ldg(Ey + nd - sy) + __ldg(Ey + nd)) * 0.5;
            if (DIMS == 3) {
                v[2] = (__ldg(Ez + nd - sz) + __ldg(Ez + nd)) * 0.5;
                v[3] = (((__ldg(Bx + nd - sy - sz) + __ldg(Bx + nd - sz)) + __ldg(Bx + nd - sy)) + __ldg(Bx + nd)) * 0.25 + g.bext[0];
                v[4] = (((__ldg(By + nd - 1 - sz) + __ldg(By + nd - 1)) + __ldg(By + nd - sz)) + __ldg(By + nd)) * 0.25 + g.bext[1];
            } else {
                v[2] = __ldg(Ez + nd);
                v[3] = (__ldg(Bx + nd - sy) + __ldg(Bx + nd)) * 0.5 + g.bext[0];
                v[4] = (__ldg(By + nd - 1) + __ldg(By + nd)) * 0.5 + g.bext[1];
            }
            v[5] = (((__ldg(Bz + nd - 1 - sy) + __ldg(Bz + nd - 1)) + __ldg(Bz + nd - sy)) + __ldg(Bz + nd)) * 0.25 + g.bext[2];
        }
    }
    __syncthreads();
    int blo[3] = {0x3fffffff, 0x3fffffff, 0x3fffffff}, bhi[3] = {-0x3fffffff, -0x3fffffff, -0x3fffffff};
    auto slot_of = [&](uint32_t i) {
        for (int r = 0; r < nseg; r++) {
            const uint32_t len = s_rg[2 * r + 1] - s_rg[2 * r];
            if (i < len) return s_rg[2 * r] + i;
            i -= len;
        }
        return 0u;   // not reached for i < total
    };
    // Item order of the threads: in each chunk of 256 items, lane l of warp
    // w takes item 32 (l / 4) + 4 w + l % 4.  The four lanes of a quad read
    // four consecutive slots (one 32-byte sector of each array), and the
    // eight quads of a warp lie 32 items apart, in different cells at the
    // usual fill: lanes whose atomics meet at an address serialise, and this
    // order puts at most four lanes of a warp on one cell, where the 32
    // consecutive items of a plain grid stride share one or two cells.
    const uint32_t lane = tid & 31;
    const uint32_t perm = (lane >> 2) * 32 + (uint32_t)(tid >> 5) * 4 + (lane & 3);
    P64 cur;
    cur.flv = 0;
    uint32_t ncur = 0;
    if (perm < total) {
        ncur = slot_of(perm);
        cur = load_p64(p, ncur);
    }
    for (uint32_t i = perm; i < total; i += kT64Threads) {
        // the next particle loads while this one moves
        P64 nxt;
        nxt.flv = 0;
        uint32_t nn = 0;
        if (i + kT64Threads < total) {
            nn = slot_of(i + kT64Threads);
            nxt = load_p64(p, nn);
        }
        const uint32_t n = ncur;
        const P64 s = cur;
        cur = nxt;
        ncur = nn;
        if (s.flv == 0) continue;
        int nc[3];
        if (body(s, n, ctx, nc)) {
            blo[0] = min(blo[0], nc[0]); bhi[0] = max(bhi[0], nc[0]);
            blo[1] = min(blo[1], nc[1]); bhi[1] = max(bhi[1], nc[1]);
            blo[2] = min(blo[2], nc[2]); bhi[2] = max(bhi[2], nc[2]);
        }
    }
    __syncthreads();
    if (ctx.use_box) {
        // the box current onto J (one FP64 atomic per nonzero word)
        const int JY = bx.jC[1] + 3;
        const double inv = 1.0 / ctx.S;
        for (int q = tid; q < bx.nj; q += kT64Threads) {
            const long long ix = (long long)sJ[q], iy = (long long)sJ[bx.nj + q], iz = (long long)sJ[2 * bx.nj + q];
            if (ix == 0 && iy == 0 && iz == 0) continue;
            const double vx = (double)ix * inv, vy = (double)iy * inv, vz = (double)iz * inv;
            const int a = q % bx.JX, r = q / bx.JX, b = r % JY, cc = r / JY;
            const long long off = cidx(g, bx.jlo[0] - 1 + a, bx.jlo[1] - 1 + b, DIMS == 3 ? bx.jlo[2] - 1 + cc : 1);
            if (vx != 0.0) atomicAdd(Jx + off, vx);
            if (vy != 0.0) atomicAdd(Jy + off, vy);
            if (vz != 0.0) atomicAdd(Jz + off, vz);
        }
    }
    // the bounds of the next box (block reduction)
    int vred[6] = {blo[0], blo[1], blo[2], -bhi[0], -bhi[1], -bhi[2]};
#pragma unroll
    for (int e = 0; e < 6; e++) vred[e] = __reduce_min_sync(0xffffffffu, vred[e]);
    if ((tid & 31) == 0)
        for (int e = 0; e < 6; e++) s_red[tid >> 5][e] = vred[e];
    __syncthreads();
    if (tid == 0) {
        int m[6];
        for (int e = 0; e < 6; e++) {
            m[e] = s_red[0][e];
            for (int w2 = 1; w2 < kT64Threads / 32; w2++) m[e] = min(m[e], s_red[w2][e]);
        }
        if (m[0] != 0x3fffffff) {   // else keep the box (every particle left or is a hole)
            gbox[0] = m[0]; gbox[1] = m[1]; gbox[2] = m[2];
            gbox[3] = -m[3]; gbox[4] = -m[4]; gbox[5] = -m[5];
        }
    }
}

}  // namespace pic
