// mover_f64_tiled.cu -- the FP64 Cartesian mover in the reference layout,
// one CTA per tile of cells, for the steps after a reorder.
//
// Reference: src/movdep/movdep.F90:62-249 (the per-particle algorithm),
// src/movdep/movdep_routines.F90:6-223 (node-averaged fields VecE/VecB, which
// the reference computes once per cell before the particle loop) and
// :243-311 (the per-cell current VecJ it scatters onto the edges afterwards).
//
// The tiles, the staged node box and the fixed-point current box are
// tile64.cuh's; this file gives them the Cartesian particle: gather at the
// start position, Boris push, the two zigzag segments (a particle that stays
// in its cell adds them in registers first, so most particles make 8 / 12
// shared atomics instead of 16 / 24), positions and momenta bit for bit the
// per-particle mover's and the serial CPU build's.  A particle that leaves
// the interior is wrapped by the exchange and appended after the sorted
// range; those are moved by the per-particle kernel (k_move_f64).
#include "common.cuh"
#include "kernels.cuh"
#include "particle_math.cuh"
#include "tile64.cuh"

namespace pic {

namespace {

__device__ __forceinline__ uint32_t lower_bound_key(const uint32_t *__restrict__ keys, long long np, uint32_t c)
{
    long long lo = 0, hi = np;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (keys[mid] < c) lo = mid + 1;
        else hi = mid;
    }
    return (uint32_t)lo;
}

// The slot range of every row segment of every tile (lower bounds of the
// segment's first and past-the-end cells in the sorted keys) and the boxes of
// the next move: the tile's own cells.
__global__ void k_tile_starts(GridP g, Tiles64 T, const uint32_t *__restrict__ keys, const Counters *__restrict__ cnt)
{
    const long long np = cnt->np;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T.ntiles; t += gridDim.x * blockDim.x) {
        if (t == 0) *T.np = np;
        int x0, x1, j0, nrow, k0, nk;
        tile_cells(g, T, t, x0, x1, j0, nrow, k0, nk);
        uint32_t *rg = T.range + 2 * (size_t)T.H * T.D * t;
        for (int q = 0; q < T.D; q++)
            for (int r = 0; r < T.H; r++) {
                uint32_t b = 0, e = 0;
                if (r < nrow && q < nk) {
                    b = lower_bound_key(keys, np, (uint32_t)cidx(g, x0, j0 + r, k0 + q));
                    e = lower_bound_key(keys, np, (uint32_t)cidx(g, x1, j0 + r, k0 + q));
                }
                rg[2 * (q * T.H + r)] = b;
                rg[2 * (q * T.H + r) + 1] = e;
            }
        // the box of the first move: the tile's interior cells (a tile of
        // ghost cells only gets an empty box: its rare particles take the
        // global path)
        int *bx = T.box + 8 * (size_t)t;
        bx[0] = max(x0, 3); bx[1] = max(j0, 3); bx[2] = g.dims == 3 ? max(k0, 3) : 1;
        bx[3] = min(x1 - 1, g.mx - 3); bx[4] = min(j0 + nrow - 1, g.my - 3);
        bx[5] = g.dims == 3 ? min(k0 + nk - 1, g.mz - 3) : 1;
    }
}

template <int DIMS>
__global__ void __launch_bounds__(kT64Threads, 2) k_move_f64_tiled(GridP g, PartF64 p, Tiles64 T,
                                                                   const double *__restrict__ Ex,
                                                                   const double *__restrict__ Ey,
                                                                   const double *__restrict__ Ez,
                                                                   const double *__restrict__ Bx,
                                                                   const double *__restrict__ By,
                                                                   const double *__restrict__ Bz, double *Jx,
                                                                   double *Jy, double *Jz, int *err)
{
    extern __shared__ __align__(16) double smem64[];
    const double c = g.c, sqc = g.sqc, cinv = g.cinv, qi = g.qi;
    // a particle moves less than c per axis, so its two segments add at most
    // q qi c to a word
    move_tile64<DIMS, 0>(g, p, T, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, c, smem64,
                         [&](const P64 &s, uint32_t n, const Tile64Ctx &ctx, int *nc) {
        const Box64 &bx = ctx.bx;
        const int flv = s.flv;
        const double x0 = s.x, y0 = s.y, z0 = s.z;
        if (flv < 0 || flv > PIC_MAX_FLVR || !(x0 >= 2.0 && x0 < (double)(g.mx - 1)) ||
            !(y0 >= 2.0 && y0 < (double)(g.my - 1)) || (DIMS == 3 && !(z0 >= 2.0 && z0 < (double)(g.mz - 1)))) {
            raise_error(err, PIC_DEVERR_RANGE);
            return false;
        }
        const double qm = g.qm[flv] * 0.5;
        const int ip0 = (int)x0, jp0 = (int)y0, kz0 = (int)z0, kp0 = DIMS == 3 ? kz0 : 1;
        double wt[8];
        weights<double, DIMS>(x0 - ip0, y0 - jp0, z0 - kz0, wt);
        double pE[3], pB[3];
        int nb = 0;
        const bool inside = ctx.use_box && in_box<DIMS>(bx, ip0, jp0, kp0, nb);
        if (inside) gather_box64<DIMS>(bx, ctx.sN, nb, wt, pE, pB);
        else gather<double, DIMS>(g, Ex, Ey, Ez, Bx, By, Bz, cidx(g, ip0, jp0, kp0), wt, pE, pB);
        for (int d = 0; d < 3; d++) {
            pE[d] = pE[d] * qm;
            pB[d] = pB[d] * qm;
        }
        double u = s.u, v = s.v, w = s.w, gg;
        boris<double>(c, sqc, cinv, pE, pB, u, v, w, gg);
        if (!finite3(u, v, w)) {
            raise_error(err, PIC_DEVERR_NAN);
            return false;
        }
        const double x1 = x0 + (u * gg) * 1.0, y1 = y0 + (v * gg) * 1.0, z1 = z0 + (w * gg) * 1.0;
        const int ip = (int)x1, jp = (int)y1, kp = (int)z1;
        const double xr = fmin((double)(min(ip0, ip) + 1), fmax((double)max(ip0, ip), 0.5 * (x0 + x1)));
        const double yr = fmin((double)(min(jp0, jp) + 1), fmax((double)max(jp0, jp), 0.5 * (y0 + y1)));
        const double zr = fmin((double)(min(kz0, kp) + 1), fmax((double)max(kz0, kp), 0.5 * (z0 + z1)));
        const double qthis = s.q * qi;
        double o[12], o2[12];
        segment<double, DIMS>(qthis * (xr - x0), qthis * (yr - y0), qthis * (zr - z0), 0.5 * (x0 + xr) - ip0,
                              0.5 * (y0 + yr) - jp0, DIMS == 3 ? 0.5 * (z0 + zr) - kp0 : 0.0, o);
        segment<double, DIMS>(qthis * (x1 - xr), qthis * (y1 - yr), qthis * (z1 - zr), 0.5 * (x1 + xr) - ip,
                              0.5 * (y1 + yr) - jp, DIMS == 3 ? 0.5 * (z1 + zr) - kp : 0.0, o2);
        const int nk = DIMS == 3 ? kp : 1;
        const bool same = ip == ip0 && jp == jp0 && nk == kp0;
        if (inside) {
            const int jb0 = ctx.jcell<DIMS>(ip0, jp0, kp0);
            if (same) {
#pragma unroll
                for (int e = 0; e < (DIMS == 3 ? 12 : 8); e++) o[e] = o[e] + o2[e];
                deposit_box64<DIMS>(bx, ctx.sJ, jb0, o, ctx.S);
            } else {
                deposit_box64<DIMS>(bx, ctx.sJ, jb0, o, ctx.S);
                deposit_box64<DIMS>(bx, ctx.sJ,
                                    jb0 + (ip - ip0) + bx.JX * (jp - jp0) + (DIMS == 3 ? bx.JXY * (kp - kp0) : 0), o2,
                                    ctx.S);
            }
        } else {
            scatter<double, DIMS>(g, Jx, Jy, Jz, cidx(g, ip0, jp0, kp0), o);
            scatter<double, DIMS>(g, Jx, Jy, Jz, cidx(g, ip, jp, nk), o2);
        }
        p.u[n] = u;
        p.v[n] = v;
        p.w[n] = w;
        p.x[n] = x1;
        p.y[n] = y1;
        double zn = z1;
        if (DIMS == 2) {  // movdep.F90:241-249
            if (zn > 2.0) zn = zn - 1.0;
            else if (zn < 1.0) zn = 1.0 + zn;
        }
        p.z[n] = zn;
        // the particles that stay in the interior bound the next box (the
        // others are wrapped by the exchange and leave the tile's ranges)
        nc[0] = ip; nc[1] = jp; nc[2] = nk;
        return ip >= 3 && ip <= g.mx - 3 && jp >= 3 && jp <= g.my - 3 && (DIMS == 2 || (nk >= 3 && nk <= g.mz - 3));
    });
}

}  // namespace

void choose_tiles64(const GridP &g, Tiles64 &T)
{
    T.W = g.dims == 3 ? 32 : 64;
    if (T.W > g.mx) T.W = g.mx;
    T.H = g.dims == 3 ? 4 : 2;
    if (T.H > g.my) T.H = g.my;
    T.D = 1;
    T.jfirst = T.H;
    if (g.geom == PIC_GEOM_CYLINDRICAL) {
        // a theta grid of a few cells: row groups aligned to the interior
        // rows (the two low ghost rows alone) and two z planes per tile, so
        // that a tile stages fewer nodes per particle
        T.D = 2;
        T.jfirst = 2;
    }
    T.nsx = (g.mx + T.W - 1) / T.W;
    const int nry = tile_row_groups(g, T);
    T.ntiles = T.nsx * nry * (g.dims == 3 ? (g.mz + T.D - 1) / T.D : 1);
    T.smem_bytes = kTile64SmemBytes;
}

void launch_tiles64_after_reorder(const GridP &g, const uint32_t *keys, const Counters *cnt, Tiles64 &T,
                                  cudaStream_t s)
{
    const int b = (T.ntiles + kThreads - 1) / kThreads;
    k_tile_starts<<<b < kSMs * 8 ? (b > 0 ? b : 1) : kSMs * 8, kThreads, 0, s>>>(g, T, keys, cnt);
    count_launches(1);
}

void launch_move_deposit_f64_tiled(const GridP &g, const PartF64 &p, const Counters *cnt, const Tiles64 &T,
                                   double *const E[3], double *const B[3], double *const J[3], int *err, cudaStream_t s)
{
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_move_f64_tiled<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTile64SmemBytes);
        cudaFuncSetAttribute(k_move_f64_tiled<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTile64SmemBytes);
        attr_set = true;
    }
    if (g.dims == 3)
        k_move_f64_tiled<3><<<T.ntiles, kT64Threads, T.smem_bytes, s>>>(g, p, T, E[0], E[1], E[2], B[0], B[1], B[2],
                                                                       J[0], J[1], J[2], err);
    else
        k_move_f64_tiled<2><<<T.ntiles, kT64Threads, T.smem_bytes, s>>>(g, p, T, E[0], E[1], E[2], B[0], B[1], B[2],
                                                                       J[0], J[1], J[2], err);
    count_launches(1);
    // the particles appended by the wraps since the reorder, per particle
    launch_move_deposit_f64(g, p, cnt, E, B, J, err, s, nullptr, T.np);
}

}  // namespace pic
