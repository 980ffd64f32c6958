// mover.cu -- fused gather / relativistic Boris push / zigzag current deposit.
//
// Reference: src/movdep/movdep.F90:12-258 (CPU loop the FP64 path restates),
// src/movdep/movdep_routines.F90:6-223 (node-averaged fields),
// src/movdep/movdep_gpu.F90:56-334 (the reference's own CUDA Fortran kernel),
// weight tables vars.F90:322-356.
//
// FP64 path: the reference layout and arithmetic.  The node averages that the
// reference stages in VecE*/VecB* are recomputed per particle from the field
// arrays with the same expressions, so interpolated fields, momenta and
// positions equal the serial CPU build bit for bit.  Currents go to J with
// FP64 atomics (order-dependent in the last bits only).
//
// FP32 path: cell-relative positions (cell index + offset in [0,1)) so FP32
// keeps full sub-cell resolution anywhere in the box; the periodic wrap is an
// integer update of the cell index inside the kernel (no holes, no append).
#include "common.cuh"
#include "kernels.cuh"
#include "particle_math.cuh"

namespace pic {

// ---------------------------------------------------------------------------
// FP64, reference layout
// ---------------------------------------------------------------------------
template <int DIMS>
__global__ void __launch_bounds__(kThreads) k_move_f64(GridP g, PartF64 p, const Counters *__restrict__ cnt,
                                                       const double *__restrict__ Ex, const double *__restrict__ Ey,
                                                       const double *__restrict__ Ez, const double *__restrict__ Bx,
                                                       const double *__restrict__ By, const double *__restrict__ Bz,
                                                       double *Jx, double *Jy, double *Jz, int *err)
{
    const long long used = cnt->used;
    const double c = g.c, sqc = g.sqc, cinv = g.cinv, qi = g.qi;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < used; n += (long long)gridDim.x * blockDim.x) {
        const int flv = p.flv[n];
        if (flv == 0) continue;  // hole: moves nothing, deposits zero
        const double x0 = p.x[n], y0 = p.y[n], z0 = p.z[n];
        if (flv < 0 || flv > PIC_MAX_FLVR || !(x0 >= 2.0 && x0 < (double)(g.mx - 1)) ||
            !(y0 >= 2.0 && y0 < (double)(g.my - 1)) || (DIMS == 3 && !(z0 >= 2.0 && z0 < (double)(g.mz - 1)))) {
            raise_error(err, PIC_DEVERR_RANGE);
            continue;
        }
        const double qm = g.qm[flv] * 0.5;                                      // movdep.F90:78
        const int ip0 = (int)x0, jp0 = (int)y0, kp0 = (int)z0;                  // :89-91
        double wt[8];
        weights<double, DIMS>(x0 - ip0, y0 - jp0, z0 - kp0, wt);
        double pE[3], pB[3];
        gather<double, DIMS>(g, Ex, Ey, Ez, Bx, By, Bz, cidx(g, ip0, jp0, DIMS == 3 ? kp0 : 1), wt, pE, pB);
        for (int d = 0; d < 3; d++) {                                           // :134-139
            pE[d] = pE[d] * qm;
            pB[d] = pB[d] * qm;
        }
        double u = p.u[n], v = p.v[n], w = p.w[n], gg;
        boris<double>(c, sqc, cinv, pE, pB, u, v, w, gg);
        const double x1 = x0 + (u * gg) * 1.0, y1 = y0 + (v * gg) * 1.0, z1 = z0 + (w * gg) * 1.0; // :169-171
        // zigzag deposit, movdep.F90:177-237
        const int ip = (int)x1, jp = (int)y1, kp = (int)z1;
        const double xr = fmin((double)(min(ip0, ip) + 1), fmax((double)max(ip0, ip), 0.5 * (x0 + x1)));
        const double yr = fmin((double)(min(jp0, jp) + 1), fmax((double)max(jp0, jp), 0.5 * (y0 + y1)));
        const double zr = fmin((double)(min(kp0, kp) + 1), fmax((double)max(kp0, kp), 0.5 * (z0 + z1)));
        const double qthis = p.q[n] * qi;
        double o[12];
        segment<double, DIMS>(qthis * (xr - x0), qthis * (yr - y0), qthis * (zr - z0), 0.5 * (x0 + xr) - ip0,
                              0.5 * (y0 + yr) - jp0, DIMS == 3 ? 0.5 * (z0 + zr) - kp0 : 0.0, o);
        scatter<double, DIMS>(g, Jx, Jy, Jz, cidx(g, ip0, jp0, DIMS == 3 ? kp0 : 1), o);
        segment<double, DIMS>(qthis * (x1 - xr), qthis * (y1 - yr), qthis * (z1 - zr), 0.5 * (x1 + xr) - ip,
                              0.5 * (y1 + yr) - jp, DIMS == 3 ? 0.5 * (z1 + zr) - kp : 0.0, o);
        scatter<double, DIMS>(g, Jx, Jy, Jz, cidx(g, ip, jp, DIMS == 3 ? kp : 1), o);
        p.u[n] = u;
        p.v[n] = v;
        p.w[n] = w;
        p.x[n] = x1;
        p.y[n] = y1;
        double zn = z1;
        if (DIMS == 2) {  // movdep.F90:241-249 (zmin=1, zmax=2, zlen=1)
            if (zn > 2.0) zn = zn - 1.0;
            else if (zn < 1.0) zn = 1.0 + zn;
        }
        p.z[n] = zn;
    }
}

void launch_move_deposit_f64(const GridP &g, const PartF64 &p, const Counters *cnt, double *const E[3],
                             double *const B[3], double *const J[3], int *err, cudaStream_t s)
{
    const int grid = kSMs * 16;
    if (g.dims == 3)
        k_move_f64<3><<<grid, kThreads, 0, s>>>(g, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2], err);
    else
        k_move_f64<2><<<grid, kThreads, 0, s>>>(g, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2], err);
    count_launches(1);
}

// ---------------------------------------------------------------------------
// FP32, cell-relative
// ---------------------------------------------------------------------------
// One particle of the FP32 form with global gathers and global atomics.
template <int DIMS>
__device__ __forceinline__ void move_one_f32_global(const GridP &g, const PartF32 &p, long long n,
                                                    const float *__restrict__ Ex, const float *__restrict__ Ey,
                                                    const float *__restrict__ Ez, const float *__restrict__ Bx,
                                                    const float *__restrict__ By, const float *__restrict__ Bz,
                                                    float *Jx, float *Jy, float *Jz, int *err)
{
    const float c = (float)g.c, sqc = (float)g.sqc, cinv = (float)g.cinv, qi = (float)g.qi;
    const int mx = g.mx, my = g.my, mz = g.mz;
    const uint32_t key = p.key[n];
    const int flv = (int)(key >> kFlvShift);
    if (flv == 0) return;
    const int cell = (int)(key & kCellMask);
    int i, j, k;
        decode_cell(g, cell, i, j, k);
    if (i < 3 || i > mx - 3 || j < 3 || j > my - 3 || (DIMS == 3 && (k < 3 || k > mz - 3)) || (DIMS == 2 && k != 1)) {
        raise_error(err, PIC_DEVERR_RANGE);
        return;
    }
    const float dx = p.dx[n], dy = p.dy[n], dz = DIMS == 3 ? p.dz[n] : 0.f;
    const float qm = (float)g.qm[flv] * 0.5f;
    float wt[8];
    weights<float, DIMS>(dx, dy, dz, wt);
    float pE[3], pB[3];
    gather<float, DIMS>(g, Ex, Ey, Ez, Bx, By, Bz, (long long)cell, wt, pE, pB);
    for (int d = 0; d < 3; d++) {
        pE[d] = pE[d] * qm;
        pB[d] = pB[d] * qm;
    }
    float u = p.ux[n], v = p.uy[n], w = p.uz[n], gg;
    boris<float>(c, sqc, cinv, pE, pB, u, v, w, gg);
    // displacement in cell units; positions relative to this cell's corner
    const float x1 = dx + u * gg, y1 = dy + v * gg, z1 = dz + w * gg;
    const int sx = (int)floorf(x1), sy = (int)floorf(y1), sz = DIMS == 3 ? (int)floorf(z1) : 0;
    // zigzag relay point with ip0 = 0, ip = s (movdep.F90:183-185)
    const float xr = fminf((float)(min(0, sx) + 1), fmaxf((float)max(0, sx), 0.5f * (dx + x1)));
    const float yr = fminf((float)(min(0, sy) + 1), fmaxf((float)max(0, sy), 0.5f * (dy + y1)));
    const float qthis = p.w[n] * qi;
    float o[12];
    float Fz1, Fz2, Wz1 = 0.f, Wz2 = 0.f;
    if (DIMS == 3) {
        const float zr = fminf((float)(min(0, sz) + 1), fmaxf((float)max(0, sz), 0.5f * (dz + z1)));
        Fz1 = qthis * (zr - dz);
        Fz2 = qthis * (z1 - zr);
        Wz1 = 0.5f * (dz + zr);
        Wz2 = 0.5f * (z1 + zr) - (float)sz;
    } else {
        // out-of-plane motion: no cell crossing, the relay point is the midpoint
        Fz1 = qthis * (0.5f * (w * gg));
        Fz2 = Fz1;
    }
    segment<float, DIMS>(qthis * (xr - dx), qthis * (yr - dy), Fz1, 0.5f * (dx + xr), 0.5f * (dy + yr), Wz1, o);
    scatter<float, DIMS>(g, Jx, Jy, Jz, (long long)cell, o);
    const long long c1 = (long long)cell + sx + (long long)sy * g.sy + (long long)sz * g.sz;
    segment<float, DIMS>(qthis * (x1 - xr), qthis * (y1 - yr), Fz2, 0.5f * (x1 + xr) - (float)sx,
                         0.5f * (y1 + yr) - (float)sy, Wz2, o);
    scatter<float, DIMS>(g, Jx, Jy, Jz, c1, o);
    // new offsets and periodic cell index
    float nx = x1 - (float)sx, ny = y1 - (float)sy, nz = z1 - (float)sz;
    int ni = i + sx, nj = j + sy, nk = k + sz;
    if (nx >= 1.f) { nx -= 1.f; ni += 1; }
    if (ny >= 1.f) { ny -= 1.f; nj += 1; }
    if (DIMS == 3 && nz >= 1.f) { nz -= 1.f; nk += 1; }
    ni = wrap_index(ni, mx);
    nj = wrap_index(nj, my);
    if (DIMS == 3) nk = wrap_index(nk, mz);
    const uint32_t ncell = (uint32_t)((ni - 1) + mx * ((nj - 1) + my * (nk - 1)));
    p.key[n] = ((uint32_t)flv << kFlvShift) | ncell;
    p.dx[n] = nx;
    p.dy[n] = ny;
    if (DIMS == 3) p.dz[n] = nz;
    p.ux[n] = u;
    p.uy[n] = v;
    p.uz[n] = w;
}

template <int DIMS>
__global__ void __launch_bounds__(kThreads) k_move_f32(GridP g, PartF32 p, const Counters *__restrict__ cnt,
                                                       const float *__restrict__ Ex, const float *__restrict__ Ey,
                                                       const float *__restrict__ Ez, const float *__restrict__ Bx,
                                                       const float *__restrict__ By, const float *__restrict__ Bz,
                                                       float *Jx, float *Jy, float *Jz, int *err)
{
    const long long used = cnt->used;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < used; n += (long long)gridDim.x * blockDim.x)
        move_one_f32_global<DIMS>(g, p, n, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, err);
}

// ---------------------------------------------------------------------------
// FP32, cell-relative, tiled: one CTA per spatial tile.
//
// After a reorder the particles of a tile (a segment of W cells of one (j,k)
// row at sort time) are contiguous.  The CTA finds the bounding box of the
// cells its particles occupy now, stages the node-averaged E and B of that box
// in shared memory (each node value computed once per tile instead of once per
// particle), accumulates the tile's current in shared memory and adds it to
// the global J once per tile.  Tiles whose box does not fit take the global
// path of k_move_f32.
// ---------------------------------------------------------------------------
constexpr int kTileThreads = 256;

template <int DIMS>
__global__ void __launch_bounds__(kTileThreads, 2)
    k_move_f32_tiled(GridP g, PartF32 p, const uint32_t *__restrict__ tile_start, const float *__restrict__ Ex,
                     const float *__restrict__ Ey, const float *__restrict__ Ez, const float *__restrict__ Bx,
                     const float *__restrict__ By, const float *__restrict__ Bz, float *Jx, float *Jy, float *Jz,
                     int *err, int smem_floats)
{
    extern __shared__ __align__(16) float sm[];
    __shared__ int bb[6];
    const uint32_t p0 = tile_start[blockIdx.x], p1 = tile_start[blockIdx.x + 1];
    if (p0 >= p1) return;
    const int tid = threadIdx.x;
    const int mx = g.mx, my = g.my, mz = g.mz;
    if (tid < 3) {
        bb[tid] = 0x7fffffff;
        bb[tid + 3] = -0x7fffffff;
    }
    __syncthreads();
    {
        int lo0 = 0x7fffffff, lo1 = 0x7fffffff, lo2 = 0x7fffffff, hi0 = -0x7fffffff, hi1 = -0x7fffffff, hi2 = -0x7fffffff;
        for (uint32_t n = p0 + tid; n < p1; n += kTileThreads) {
            const uint32_t key = p.key[n];
            if ((key >> kFlvShift) == 0) continue;
            const int cell = (int)(key & kCellMask);
            int i, j, k;
        decode_cell(g, cell, i, j, k);
            lo0 = min(lo0, i); hi0 = max(hi0, i);
            lo1 = min(lo1, j); hi1 = max(hi1, j);
            lo2 = min(lo2, k); hi2 = max(hi2, k);
        }
        lo0 = __reduce_min_sync(0xffffffffu, lo0); hi0 = __reduce_max_sync(0xffffffffu, hi0);
        lo1 = __reduce_min_sync(0xffffffffu, lo1); hi1 = __reduce_max_sync(0xffffffffu, hi1);
        lo2 = __reduce_min_sync(0xffffffffu, lo2); hi2 = __reduce_max_sync(0xffffffffu, hi2);
        if ((tid & 31) == 0) {
            atomicMin(&bb[0], lo0); atomicMin(&bb[1], lo1); atomicMin(&bb[2], lo2);
            atomicMax(&bb[3], hi0); atomicMax(&bb[4], hi1); atomicMax(&bb[5], hi2);
        }
    }
    __syncthreads();
    const int ilo = bb[0], jlo = bb[1], klo = bb[2], ihi = bb[3], jhi = bb[4], khi = bb[5];
    if (ilo > ihi) return;  // only holes
    // node box [lo, hi+1], current box [lo-1, hi+2] per axis
    const int NX = ihi - ilo + 2, NY = jhi - jlo + 2, NZ = DIMS == 3 ? khi - klo + 2 : 1;
    const int JX = ihi - ilo + 4, JY = jhi - jlo + 4, JZ = DIMS == 3 ? khi - klo + 4 : 1;
    const int nnode = NX * NY * NZ, njc = JX * JY * JZ;
    const bool fits = (long long)nnode * 6 + (long long)njc * 3 <= smem_floats &&
                      ilo >= 3 && ihi <= mx - 3 && jlo >= 3 && jhi <= my - 3 &&
                      (DIMS == 2 || (klo >= 3 && khi <= mz - 3));
    const uint32_t ntile = p1 - p0;
    const uint32_t per = (ntile + kTileThreads - 1) / kTileThreads;
    const uint32_t b0 = p0 + tid * per, b1 = min(b0 + per, p1);
    if (!fits) {
        for (uint32_t n = b0; n < b1; n++) move_one_f32_global<DIMS>(g, p, n, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, err);
        return;
    }
    float4 *nA = reinterpret_cast<float4 *>(sm);
    float2 *nB = reinterpret_cast<float2 *>(sm + 4 * nnode);
    float *sJ = sm + 6 * nnode;
    const long long sy = g.sy, sz = g.sz;
    const float b0f = (float)g.bext[0], b1f = (float)g.bext[1], b2f = (float)g.bext[2];
    for (int q = tid; q < nnode; q += kTileThreads) {
        const int a = ilo + q % NX, r = q / NX, b = jlo + r % NY, c = DIMS == 3 ? klo + r / NY : 1;
        const long long nd = cidx(g, a, b, c);
        const float vex = (__ldg(Ex + nd - 1) + __ldg(Ex + nd)) * 0.5f;
        const float vey = (__ldg(Ey + nd - sy) + __ldg(Ey + nd)) * 0.5f;
        float vez, vbx, vby;
        if (DIMS == 3) {
            vez = (__ldg(Ez + nd - sz) + __ldg(Ez + nd)) * 0.5f;
            vbx = (((__ldg(Bx + nd - sy - sz) + __ldg(Bx + nd - sz)) + __ldg(Bx + nd - sy)) + __ldg(Bx + nd)) * 0.25f + b0f;
            vby = (((__ldg(By + nd - 1 - sz) + __ldg(By + nd - 1)) + __ldg(By + nd - sz)) + __ldg(By + nd)) * 0.25f + b1f;
        } else {
            vez = __ldg(Ez + nd);
            vbx = (__ldg(Bx + nd - sy) + __ldg(Bx + nd)) * 0.5f + b0f;
            vby = (__ldg(By + nd - 1) + __ldg(By + nd)) * 0.5f + b1f;
        }
        const float vbz = (((__ldg(Bz + nd - 1 - sy) + __ldg(Bz + nd - 1)) + __ldg(Bz + nd - sy)) + __ldg(Bz + nd)) * 0.25f + b2f;
        nA[q] = make_float4(vex, vey, vez, vbx);
        nB[q] = make_float2(vby, vbz);
    }
    for (int q = tid; q < 3 * njc; q += kTileThreads) sJ[q] = 0.f;
    __syncthreads();

    const float c = (float)g.c, sqc = (float)g.sqc, cinv = (float)g.cinv, qi = (float)g.qi;
    const int NXY = NX * NY, JXY = JX * JY;
    float *sJx = sJ, *sJy = sJ + njc, *sJz = sJ + 2 * njc;
    for (uint32_t n = b0; n < b1; n++) {
        const uint32_t key = p.key[n];
        const int flv = (int)(key >> kFlvShift);
        if (flv == 0) continue;
        const int cell = (int)(key & kCellMask);
        int i, j, k;
        decode_cell(g, cell, i, j, k);
        const float dx = p.dx[n], dy = p.dy[n], dz = DIMS == 3 ? p.dz[n] : 0.f;
        float wt[8];
        weights<float, DIMS>(dx, dy, dz, wt);
        const int nb = (i - ilo) + NX * ((j - jlo) + NY * (DIMS == 3 ? k - klo : 0));
        float pE[3] = {0.f, 0.f, 0.f}, pB[3] = {0.f, 0.f, 0.f};
#pragma unroll
        for (int c8 = 0; c8 < (DIMS == 3 ? 8 : 4); c8++) {
            const int q = nb + (c8 & 1) + ((c8 >> 1) & 1) * NX + ((c8 >> 2) & 1) * NXY;
            const float4 A = nA[q];
            const float2 Bv = nB[q];
            pE[0] = pE[0] + wt[c8] * A.x;
            pE[1] = pE[1] + wt[c8] * A.y;
            pE[2] = pE[2] + wt[c8] * A.z;
            pB[0] = pB[0] + wt[c8] * A.w;
            pB[1] = pB[1] + wt[c8] * Bv.x;
            pB[2] = pB[2] + wt[c8] * Bv.y;
        }
        const float qm = (float)g.qm[flv] * 0.5f;
        for (int d = 0; d < 3; d++) {
            pE[d] = pE[d] * qm;
            pB[d] = pB[d] * qm;
        }
        float u = p.ux[n], v = p.uy[n], w = p.uz[n], gg;
        boris<float>(c, sqc, cinv, pE, pB, u, v, w, gg);
        const float x1 = dx + u * gg, y1 = dy + v * gg, z1 = dz + w * gg;
        const int sxx = (int)floorf(x1), syy = (int)floorf(y1), szz = DIMS == 3 ? (int)floorf(z1) : 0;
        const float xr = fminf((float)(min(0, sxx) + 1), fmaxf((float)max(0, sxx), 0.5f * (dx + x1)));
        const float yr = fminf((float)(min(0, syy) + 1), fmaxf((float)max(0, syy), 0.5f * (dy + y1)));
        const float qthis = p.w[n] * qi;
        float o1[12], o2[12];
        float Fz1, Fz2, Wz1 = 0.f, Wz2 = 0.f;
        if (DIMS == 3) {
            const float zr = fminf((float)(min(0, szz) + 1), fmaxf((float)max(0, szz), 0.5f * (dz + z1)));
            Fz1 = qthis * (zr - dz);
            Fz2 = qthis * (z1 - zr);
            Wz1 = 0.5f * (dz + zr);
            Wz2 = 0.5f * (z1 + zr) - (float)szz;
        } else {
            Fz1 = qthis * (0.5f * (w * gg));
            Fz2 = Fz1;
        }
        segment<float, DIMS>(qthis * (xr - dx), qthis * (yr - dy), Fz1, 0.5f * (dx + xr), 0.5f * (dy + yr), Wz1, o1);
        segment<float, DIMS>(qthis * (x1 - xr), qthis * (y1 - yr), Fz2, 0.5f * (x1 + xr) - (float)sxx,
                             0.5f * (y1 + yr) - (float)syy, Wz2, o2);
        const int jb = (i - ilo + 1) + JX * ((j - jlo + 1) + JY * (DIMS == 3 ? k - klo + 1 : 0));
        const bool same = (sxx | syy | szz) == 0;
        if (same) {
#pragma unroll
            for (int e = 0; e < (DIMS == 3 ? 12 : 8); e++) o1[e] = o1[e] + o2[e];
        }
        if (DIMS == 3) {
            atomicAdd(sJx + jb, o1[0]); atomicAdd(sJx + jb + JX, o1[1]);
            atomicAdd(sJx + jb + JXY, o1[2]); atomicAdd(sJx + jb + JX + JXY, o1[3]);
            atomicAdd(sJy + jb, o1[4]); atomicAdd(sJy + jb + 1, o1[5]);
            atomicAdd(sJy + jb + JXY, o1[6]); atomicAdd(sJy + jb + 1 + JXY, o1[7]);
            atomicAdd(sJz + jb, o1[8]); atomicAdd(sJz + jb + 1, o1[9]);
            atomicAdd(sJz + jb + JX, o1[10]); atomicAdd(sJz + jb + 1 + JX, o1[11]);
            if (!same) {
                const int j2 = jb + sxx + syy * JX + szz * JXY;
                atomicAdd(sJx + j2, o2[0]); atomicAdd(sJx + j2 + JX, o2[1]);
                atomicAdd(sJx + j2 + JXY, o2[2]); atomicAdd(sJx + j2 + JX + JXY, o2[3]);
                atomicAdd(sJy + j2, o2[4]); atomicAdd(sJy + j2 + 1, o2[5]);
                atomicAdd(sJy + j2 + JXY, o2[6]); atomicAdd(sJy + j2 + 1 + JXY, o2[7]);
                atomicAdd(sJz + j2, o2[8]); atomicAdd(sJz + j2 + 1, o2[9]);
                atomicAdd(sJz + j2 + JX, o2[10]); atomicAdd(sJz + j2 + 1 + JX, o2[11]);
            }
        } else {
            atomicAdd(sJx + jb, o1[0]); atomicAdd(sJx + jb + JX, o1[1]);
            atomicAdd(sJy + jb, o1[2]); atomicAdd(sJy + jb + 1, o1[3]);
            atomicAdd(sJz + jb, o1[4]); atomicAdd(sJz + jb + 1, o1[5]);
            atomicAdd(sJz + jb + JX, o1[6]); atomicAdd(sJz + jb + 1 + JX, o1[7]);
            if (!same) {
                const int j2 = jb + sxx + syy * JX;
                atomicAdd(sJx + j2, o2[0]); atomicAdd(sJx + j2 + JX, o2[1]);
                atomicAdd(sJy + j2, o2[2]); atomicAdd(sJy + j2 + 1, o2[3]);
                atomicAdd(sJz + j2, o2[4]); atomicAdd(sJz + j2 + 1, o2[5]);
                atomicAdd(sJz + j2 + JX, o2[6]); atomicAdd(sJz + j2 + 1 + JX, o2[7]);
            }
        }
        // new offsets and periodic cell index
        float nx = x1 - (float)sxx, ny = y1 - (float)syy, nz = z1 - (float)szz;
        int ni = i + sxx, nj = j + syy, nk = k + szz;
        if (nx >= 1.f) { nx -= 1.f; ni += 1; }
        if (ny >= 1.f) { ny -= 1.f; nj += 1; }
        if (DIMS == 3 && nz >= 1.f) { nz -= 1.f; nk += 1; }
        ni = wrap_index(ni, mx);
        nj = wrap_index(nj, my);
        if (DIMS == 3) nk = wrap_index(nk, mz);
        p.key[n] = ((uint32_t)flv << kFlvShift) | (uint32_t)((ni - 1) + mx * ((nj - 1) + my * (nk - 1)));
        p.dx[n] = nx;
        p.dy[n] = ny;
        if (DIMS == 3) p.dz[n] = nz;
        p.ux[n] = u;
        p.uy[n] = v;
        p.uz[n] = w;
    }
    __syncthreads();
    // add the tile's current to the global arrays (cells of the box, ghosts included)
    for (int q = tid; q < 3 * njc; q += kTileThreads) {
        const float val = sJ[q];
        if (val == 0.f) continue;
        const int comp = q / njc, r = q - comp * njc;
        const int a = ilo - 1 + r % JX, r2 = r / JX, b = jlo - 1 + r2 % JY, cz = DIMS == 3 ? klo - 1 + r2 / JY : 1;
        float *J = comp == 0 ? Jx : comp == 1 ? Jy : Jz;
        atomicAdd(J + cidx(g, a, b, cz), val);
    }
}

constexpr int kTileSmemBytes = 100 * 1024;

void launch_move_deposit_f32_tiled(const GridP &g, const PartF32 &p, const uint32_t *tile_start, int ntiles,
                                   float *const E[3], float *const B[3], float *const J[3], int *err, cudaStream_t s)
{
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_move_f32_tiled<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmemBytes);
        cudaFuncSetAttribute(k_move_f32_tiled<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmemBytes);
        attr_set = true;
    }
    const int nf = kTileSmemBytes / 4;
    if (g.dims == 3)
        k_move_f32_tiled<3><<<ntiles, kTileThreads, kTileSmemBytes, s>>>(g, p, tile_start, E[0], E[1], E[2], B[0], B[1],
                                                                         B[2], J[0], J[1], J[2], err, nf);
    else
        k_move_f32_tiled<2><<<ntiles, kTileThreads, kTileSmemBytes, s>>>(g, p, tile_start, E[0], E[1], E[2], B[0], B[1],
                                                                         B[2], J[0], J[1], J[2], err, nf);
    count_launches(1);
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

}  // namespace pic
