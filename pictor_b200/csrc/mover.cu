// mover.cu -- fused gather / relativistic Boris push / zigzag current deposit,
// FP64 reference layout.
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
// FP64 atomics (order-dependent in the last bits only), or, with
// pic_config.exact_current, are summed in the serial build's order: each
// cell's VecJ entries in particle order (segment 1 before segment 2), then
// the VecJ entries onto the edges in the loop order of ReduceCurrentMatrix
// (movdep_routines.F90:262-308), which makes J, and with it the whole step,
// equal to the serial CPU build bit for bit and independent of the launch.
//
// The FP32 cell-relative movers are in mover_f32.cu.
#include "common.cuh"
#include "kernels.cuh"
#include "particle_math.cuh"

namespace pic {

// ---------------------------------------------------------------------------
// FP64, reference layout
// ---------------------------------------------------------------------------
// Records of the exact-order deposit (see SegRecords): key and values of
// record r, or key ncell for a record that carries nothing.
struct RecOut {
    uint32_t *key;
    double *val;
    long long n2;
};

template <int DIMS>
__device__ __forceinline__ void put_record(const GridP &g, const RecOut &ro, long long r, long long cell,
                                           const double *o)
{
    constexpr int NE = DIMS == 3 ? 12 : 8;
    ro.key[r] = (uint32_t)cell;
#pragma unroll
    for (int e = 0; e < NE; e++) ro.val[e * ro.n2 + r] = o[e];
}

template <int DIMS, bool RECORD>
__global__ void __launch_bounds__(kThreads) k_move_f64(GridP g, PartF64 p, const Counters *__restrict__ cnt,
                                                       const double *__restrict__ Ex, const double *__restrict__ Ey,
                                                       const double *__restrict__ Ez, const double *__restrict__ Bx,
                                                       const double *__restrict__ By, const double *__restrict__ Bz,
                                                       double *Jx, double *Jy, double *Jz, int *err, RecOut ro,
                                                       const long long *__restrict__ first)
{
    const long long used = cnt->used;
    const long long n0 = first ? *first : 0;
    const double c = g.c, sqc = g.sqc, cinv = g.cinv, qi = g.qi;
    for (long long n = n0 + (long long)blockIdx.x * blockDim.x + threadIdx.x; n < used;
         n += (long long)gridDim.x * blockDim.x) {
        if (RECORD) {   // nothing recorded unless the particle deposits below
            ro.key[2 * n] = (uint32_t)g.ncell;
            ro.key[2 * n + 1] = (uint32_t)g.ncell;
        }
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
        if (!finite3(u, v, w)) {
            raise_error(err, PIC_DEVERR_NAN);
            continue;
        }
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
        if (RECORD) put_record<DIMS>(g, ro, 2 * n, cidx(g, ip0, jp0, DIMS == 3 ? kp0 : 1), o);
        else scatter<double, DIMS>(g, Jx, Jy, Jz, cidx(g, ip0, jp0, DIMS == 3 ? kp0 : 1), o);
        segment<double, DIMS>(qthis * (x1 - xr), qthis * (y1 - yr), qthis * (z1 - zr), 0.5 * (x1 + xr) - ip,
                              0.5 * (y1 + yr) - jp, DIMS == 3 ? 0.5 * (z1 + zr) - kp : 0.0, o);
        if (RECORD) put_record<DIMS>(g, ro, 2 * n + 1, cidx(g, ip, jp, DIMS == 3 ? kp : 1), o);
        else scatter<double, DIMS>(g, Jx, Jy, Jz, cidx(g, ip, jp, DIMS == 3 ? kp : 1), o);
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

// The records' count: two per particle slot.
__global__ void k_record_count(const Counters *__restrict__ cnt, long long *count) { *count = 2 * cnt->used; }

// VecJ of every cell that has records: the thread at the first sorted record
// of a cell sums the cell's records in sorted order (particle order, segment
// 1 before 2) from +0, as the serial build adds to its zeroed VecJ
// (movdep.F90:209,233).  Cells without records keep the zeros of the memset.
template <int DIMS>
__global__ void __launch_bounds__(kThreads) k_vecj_sum(GridP g, const uint32_t *__restrict__ key,
                                                       const uint32_t *__restrict__ idx, const long long *__restrict__ count,
                                                       const double *__restrict__ val, long long n2, double *vecj)
{
    constexpr int NE = DIMS == 3 ? 12 : 8;
    const long long n = *count;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const uint32_t k = key[q];
        if (k >= (uint32_t)g.ncell || (q > 0 && key[q - 1] == k)) continue;
        double acc[NE];
#pragma unroll
        for (int e = 0; e < NE; e++) acc[e] = 0.0;
        for (long long t = q; t < n && key[t] == k; t++) {
            const long long r = idx[t];
#pragma unroll
            for (int e = 0; e < NE; e++) acc[e] = acc[e] + val[e * n2 + r];
        }
#pragma unroll
        for (int e = 0; e < NE; e++) vecj[e * g.ncell + k] = acc[e];
    }
}

// J from VecJ in the loop order of ReduceCurrentMatrix (movdep_routines.F90:
// 262-308: cells i = 1..mx-1, j = 1..my-1, k = 1..mz-1 in column-major order,
// entries 0..NE-1 within a cell, added onto J zeroed by ResetCurrent).  An
// edge receives the entries of up to 4 cells; they are added in the order
// the loop visits those cells (increasing linear index).
template <int DIMS>
__global__ void __launch_bounds__(kThreads) k_assemble_j(GridP g, const double *__restrict__ vecj, double *Jx,
                                                         double *Jy, double *Jz)
{
    const long long N = g.ncell;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        decode_cell(g, (int)c, i, j, k);
        // source cell (a, b, d) = (i - da, j - db, k - dd) takes part if inside the loop range
        auto V = [&](int e, int da, int db, int dd) -> double {
            const int a = i - da, b = j - db, d = k - dd;
            if (a < 1 || a > g.mx - 1 || b < 1 || b > g.my - 1) return 0.0;
            if (DIMS == 3 && (d < 1 || d > g.mz - 1)) return 0.0;
            return vecj[e * N + (c - da - db * g.sy - dd * g.sz)];
        };
        if (DIMS == 3) {
            Jx[c] = (((0.0 + V(3, 0, 1, 1)) + V(2, 0, 0, 1)) + V(1, 0, 1, 0)) + V(0, 0, 0, 0);
            Jy[c] = (((0.0 + V(7, 1, 0, 1)) + V(6, 0, 0, 1)) + V(5, 1, 0, 0)) + V(4, 0, 0, 0);
            Jz[c] = (((0.0 + V(11, 1, 1, 0)) + V(10, 0, 1, 0)) + V(9, 1, 0, 0)) + V(8, 0, 0, 0);
        } else {
            Jx[c] = (0.0 + V(1, 0, 1, 0)) + V(0, 0, 0, 0);
            Jy[c] = (0.0 + V(3, 1, 0, 0)) + V(2, 0, 0, 0);
            Jz[c] = (((0.0 + V(7, 1, 1, 0)) + V(6, 0, 1, 0)) + V(5, 1, 0, 0)) + V(4, 0, 0, 0);
        }
    }
}

static unsigned grid_for(long long n)
{
    long long b = (n + kThreads - 1) / kThreads;
    if (b > (long long)kSMs * 32) b = (long long)kSMs * 32;
    return (unsigned)(b < 1 ? 1 : b);
}

void launch_move_deposit_f64(const GridP &g, const PartF64 &p, const Counters *cnt, double *const E[3],
                             double *const B[3], double *const J[3], int *err, cudaStream_t s, SegRecords *rec,
                             const long long *first)
{
    const int grid = kSMs * 16;
    if (!rec) {
        const RecOut ro = {nullptr, nullptr, 0};
        if (g.dims == 3)
            k_move_f64<3, false><<<grid, kThreads, 0, s>>>(g, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1],
                                                          J[2], err, ro, first);
        else
            k_move_f64<2, false><<<grid, kThreads, 0, s>>>(g, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1],
                                                          J[2], err, ro, first);
        count_launches(1);
        return;
    }
    const RecOut ro = {rec->sc.key[0], rec->val, rec->n2};
    const int NE = g.dims == 3 ? 12 : 8;
    if (g.dims == 3)
        k_move_f64<3, true><<<grid, kThreads, 0, s>>>(g, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2],
                                                     err, ro, nullptr);
    else
        k_move_f64<2, true><<<grid, kThreads, 0, s>>>(g, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2],
                                                     err, ro, nullptr);
    k_record_count<<<1, 1, 0, s>>>(cnt, rec->count);
    count_launches(2);
    const int r = radix_sort_keys(rec->sc, rec->count, sort_key_bits(g.ncell), s);
    cudaMemsetAsync(rec->vecj, 0, (size_t)NE * (size_t)g.ncell * sizeof(double), s);
    const unsigned gq = grid_for(rec->n2);
    if (g.dims == 3)
        k_vecj_sum<3><<<gq, kThreads, 0, s>>>(g, rec->sc.key[r], rec->sc.idx[r], rec->count, rec->val, rec->n2,
                                              rec->vecj);
    else
        k_vecj_sum<2><<<gq, kThreads, 0, s>>>(g, rec->sc.key[r], rec->sc.idx[r], rec->count, rec->val, rec->n2,
                                              rec->vecj);
    if (g.dims == 3) k_assemble_j<3><<<grid_for(g.ncell), kThreads, 0, s>>>(g, rec->vecj, J[0], J[1], J[2]);
    else k_assemble_j<2><<<grid_for(g.ncell), kThreads, 0, s>>>(g, rec->vecj, J[0], J[1], J[2]);
    count_launches(2);
}

}  // namespace pic
