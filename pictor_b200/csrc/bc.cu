// bc.cu -- walls along x and y on one rank (src/bc/bc_reflect.F90 with
// xborders(procxind) = 0), for setups whose EnforceBC_PostMovDep
// (MAIN.F90:77) and EnforceBC_Final (:209) put reflecting particle walls and
// conducting field walls on the x faces (bc_face(1), bc_face(2)) or the y
// faces (bc_face(3), bc_face(4)).  FP64
// reference layout, the same arithmetic as the reference's CPU routines.
#include "common.cuh"
#include "kernels.cuh"

namespace pic {

namespace {

// RefPrtlLeft / RefPrtlRight (bc_reflect.F90:164-190): a particle beyond the
// wall xw (x < xw on the left, x > xw on the right) is mirrored and its u
// reversed.
__global__ void k_refl_prtl(const int *__restrict__ flv, double *X, double *U, const Counters *__restrict__ cnt,
                            double xw, int side)
{
    const long long used = cnt->used;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < used;
         n += (long long)gridDim.x * blockDim.x) {
        if (flv[n] == 0) continue;
        const double x = X[n];
        if (side == 0 ? x < xw : x > xw) {
            U[n] = -U[n];
            X[n] = 2.0 * xw - x;
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

// The y layer version (RefBC_Prtl_Top / Bottom, bc_reflect.F90:79-128).
__global__ void k_fold_y_layer(GridP g, double *F, int to, int from, double sign)
{
    const long long n = (long long)g.mx * g.mz;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const long long k = q / g.mx, i = q - k * g.mx;
        const long long ct = i + g.mx * ((to - 1) + g.my * k), cf = i + g.mx * ((from - 1) + g.my * k);
        F[ct] = sign > 0.0 ? F[ct] + F[cf] : F[ct] - F[cf];
        F[cf] = 0.0;
    }
}

// CondBC_Fld_Top / Bottom (bc_reflect.F90:11-41): Ex, Ez = 0 on y layers y0..y1.
__global__ void k_zero_y_layers(GridP g, double *Ex, double *Ez, int y0, int y1)
{
    const int h = y1 - y0 + 1;
    const long long n = (long long)g.mx * h * g.mz;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const long long r = q / g.mx, i = q - r * g.mx;
        const long long k = r / h, jj = r - k * h;
        const long long c = i + g.mx * ((y0 - 1 + jj) + g.my * k);
        Ex[c] = 0.0;
        Ez[c] = 0.0;
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

// RemovePrtl_Left / Right (bc_open.F90:8-62): a particle beyond the wall on
// the face's axis becomes a hole with RemovePrtl's values.
__global__ void k_remove_prtl(PartF64 p, const Counters *__restrict__ cnt, int axis, int low, double wall, double zhole)
{
    const long long used = cnt->used;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < used;
         n += (long long)gridDim.x * blockDim.x) {
        if (p.flv[n] == 0) continue;
        const double c = axis == 0 ? p.x[n] : axis == 1 ? p.y[n] : p.z[n];
        if (low ? c < wall : c > wall) {
            p.q[n] = 0.0;
            p.flv[n] = 0;
            p.u[n] = 0.0;
            p.v[n] = 0.0;
            p.w[n] = 0.0;
            p.x[n] = 3.8;
            p.y[n] = 3.8;
            p.z[n] = zhole;
        }
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
        k_refl_prtl<<<grid_for(capacity), kThreads, 0, s>>>(p.flv, p.x, p.u, cnt, xw, side);
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

// RefBC_Prtl_Bottom (side 0, bc_reflect.F90:106-128) / RefBC_Prtl_Top (side 1,
// :79-104): W = int(wall) is the first layer inside the wall.
void launch_wall_reflect_y(const GridP &g, PartF64 &p, const Counters *cnt, double *const J[3], int side, double pos,
                           long long capacity, cudaStream_t s)
{
    const double yw = pos - 0.0 + 3;
    const int W = (int)yw;
    if (side == 0 ? yw > 1 : yw < g.my - 1) {
        k_refl_prtl<<<grid_for(capacity), kThreads, 0, s>>>(p.flv, p.y, p.v, cnt, yw, side);
        count_launches(1);
    }
    const long long plane = (long long)g.mx * g.mz;
    if (side == 0 && W >= 3 && W <= g.my - 2) {
        k_fold_y_layer<<<grid_for(plane), kThreads, 0, s>>>(g, J[0], W, W - 1, 1.0);
        k_fold_y_layer<<<grid_for(plane), kThreads, 0, s>>>(g, J[1], W, W - 1, -1.0);
        k_fold_y_layer<<<grid_for(plane), kThreads, 0, s>>>(g, J[2], W, W - 1, 1.0);
        count_launches(3);
    } else if (side == 1 && W >= 2 && W <= g.my - 2) {
        k_fold_y_layer<<<grid_for(plane), kThreads, 0, s>>>(g, J[0], W, W + 1, 1.0);
        k_fold_y_layer<<<grid_for(plane), kThreads, 0, s>>>(g, J[1], W - 1, W, -1.0);
        k_fold_y_layer<<<grid_for(plane), kThreads, 0, s>>>(g, J[2], W, W + 1, 1.0);
        count_launches(3);
    }
}

// CondBC_Fld_Bottom (side 0) / CondBC_Fld_Top (side 1) at the wall `pos`.
void launch_wall_conducting_y(const GridP &g, double *const E[3], int side, double pos, cudaStream_t s)
{
    int y0, y1;
    if (side == 0) {
        y1 = (int)floor(pos - 0.0 + 3);
        if (y1 < 1) return;
        y1 = y1 < g.my ? y1 : g.my;
        y0 = 1;
    } else {
        y0 = (int)ceil(pos - 0.0 + 3);
        if (y0 > g.my) return;
        y0 = y0 > 1 ? y0 : 1;
        y1 = g.my;
    }
    k_zero_y_layers<<<grid_for((long long)g.mx * (y1 - y0 + 1) * g.mz), kThreads, 0, s>>>(g, E[0], E[2], y0, y1);
    count_launches(1);
}

// RemovePrtl at face 1..6 (x, y, z; low, high), wall at bc_pos_local = pos + 3.
void launch_wall_remove(const GridP &g, PartF64 &p, const Counters *cnt, int face, double pos, long long capacity,
                        cudaStream_t s)
{
    k_remove_prtl<<<grid_for(capacity), kThreads, 0, s>>>(p, cnt, (face - 1) / 2, face % 2, pos - 0.0 + 3,
                                                          g.dims == 3 ? 3.8 : 1.5);
    count_launches(1);
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
