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
// FP64 atomics (order-dependent in the last bits only).
//
// The FP32 cell-relative movers are in mover_f32.cu.
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

}  // namespace pic
