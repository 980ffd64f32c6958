// bc.cu -- walls along x on one rank (src/bc/bc_reflect.F90 with
// xborders(procxind) = 0), for setups whose EnforceBC_PostMovDep
// (MAIN.F90:77) and EnforceBC_Final (:209) put reflecting particle walls and
// conducting field walls on the x faces (bc_face(1), bc_face(2)).  FP64
// reference layout, the same arithmetic as the reference's CPU routines.
#include "common.cuh"
#include "kernels.cuh"

namespace pic {

namespace {

// RefPrtlLeft / RefPrtlRight (bc_reflect.F90:164-190): a particle beyond the
// wall xw (x < xw on the left, x > xw on the right) is mirrored and its u
// reversed.
__global__ void k_refl_prtl(PartF64 p, const Counters *__restrict__ cnt, double xw, int side)
{
    const long long used = cnt->used;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < used;
         n += (long long)gridDim.x * blockDim.x) {
        if (p.flv[n] == 0) continue;
        const double x = p.x[n];
        if (side == 0 ? x < xw : x > xw) {
            p.u[n] = -p.u[n];
            p.x[n] = 2.0 * xw - x;
        }
    }
}

// ReflCurrentLeft / Right (bc_reflect.F90:195-237): F(to,:,:) = F(to,:,:) +-
// F(from,:,:), then F(from,:,:) = 0, over every (j, k).
__global__ void k_fold_x_layer(GridP g, double *F, int to, int from, double sign)
{
    const long long n = (long long)g.my * g.mz;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const long long ct = (long long)(to - 1) + g.mx * q, cf = (long long)(from - 1) + g.mx * q;
        F[ct] = sign > 0.0 ? F[ct] + F[cf] : F[ct] - F[cf];
        F[cf] = 0.0;
    }
}

// CondBC_Fld_Left / Right (bc_reflect.F90:43-72): Ey, Ez = 0 on x layers x0..x1.
__global__ void k_zero_x_layers(GridP g, double *Ey, double *Ez, int x0, int x1)
{
    const int w = x1 - x0 + 1;
    const long long n = (long long)w * g.my * g.mz;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const long long jk = q / w;
        const long long c = (long long)(x0 - 1 + (int)(q - jk * w)) + g.mx * jk;
        Ey[c] = 0.0;
        Ez[c] = 0.0;
    }
}

int grid_for(long long n)
{
    const long long b = (n + kThreads - 1) / kThreads;
    return (int)(b < kSMs * 8 ? (b > 0 ? b : 1) : kSMs * 8);
}

}  // namespace

// RefBC_Prtl_Left (side 0, bc_reflect.F90:146-155) / RefBC_Prtl_Right
// (side 1, :135-144) at the wall `pos` (cells from the first interior cell).
void launch_wall_reflect(const GridP &g, PartF64 &p, const Counters *cnt, double *const J[3], int side, double pos,
                         long long capacity, cudaStream_t s)
{
    const double xw = pos - 0.0 + 3;
    if (side == 0 ? xw > 1 : xw < g.mx - 1) {
        k_refl_prtl<<<grid_for(capacity), kThreads, 0, s>>>(p, cnt, xw, side);
        count_launches(1);
    }
    const long long plane = (long long)g.my * g.mz;
    if (side == 0) {
        const int ind = (int)ceil(pos - 0.0 + 3), indx = (int)ceil(pos - 0.5 - 0.0 + 3);
        if (ind >= 2 && ind <= g.mx) {
            k_fold_x_layer<<<grid_for(plane), kThreads, 0, s>>>(g, J[1], ind, ind - 1, 1.0);
            k_fold_x_layer<<<grid_for(plane), kThreads, 0, s>>>(g, J[2], ind, ind - 1, 1.0);
            count_launches(2);
        }
        if (indx >= 2 && indx <= g.mx) {
            k_fold_x_layer<<<grid_for(plane), kThreads, 0, s>>>(g, J[0], indx, indx - 1, -1.0);
            count_launches(1);
        }
    } else {
        const int ind = (int)floor(pos - 0.0 + 3), indx = (int)floor(pos - 0.5 - 0.0 + 3);
        if (ind >= 1 && ind <= g.mx - 1) {
            k_fold_x_layer<<<grid_for(plane), kThreads, 0, s>>>(g, J[1], ind, ind + 1, 1.0);
            k_fold_x_layer<<<grid_for(plane), kThreads, 0, s>>>(g, J[2], ind, ind + 1, 1.0);
            count_launches(2);
        }
        if (indx >= 1 && indx <= g.mx - 1) {
            k_fold_x_layer<<<grid_for(plane), kThreads, 0, s>>>(g, J[0], indx, indx + 1, -1.0);
            count_launches(1);
        }
    }
}

// CondBC_Fld_Left (side 0) / CondBC_Fld_Right (side 1) at the wall `pos`.
void launch_wall_conducting(const GridP &g, double *const E[3], int side, double pos, cudaStream_t s)
{
    int x0, x1;
    if (side == 0) {
        x1 = (int)floor(pos - 0.0 + 3);
        if (x1 < 1) return;
        x1 = x1 < g.mx ? x1 : g.mx;
        x0 = 1;
    } else {
        x0 = (int)ceil(pos - 0.0 + 3);
        if (x0 > g.mx) return;
        x0 = x0 > 1 ? x0 : 1;
        x1 = g.mx;
    }
    k_zero_x_layers<<<grid_for((long long)(x1 - x0 + 1) * g.my * g.mz), kThreads, 0, s>>>(g, E[1], E[2], x0, x1);
    count_launches(1);
}

}  // namespace pic
