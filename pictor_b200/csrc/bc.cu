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

// ---------------------------------------------------------------------------
// Field faces of EnforceBC_Final (bc.F90:292-340) other than 'cond'.
// Global positions on one rank: x0 = xborders(procxind) - 3 = -3 (likewise
// y0, z0; z0 = 0 in 2D); the staggered positions of the six components are
// those of bc_attenuate.F90:36-81 and :184-206.
// ---------------------------------------------------------------------------

// The cube of t as gfortran evaluates t**3 (t * t * t).
__device__ __forceinline__ double cube(double t) { return t * t * t; }

// AttenFactorVacuum (bc_attenuate.F90:222-290): the faces' attn_vac_pos p
// (+-huge for faces that are not 'attn') and attn_scale sc; the z faces only
// in 3D.  Later faces override earlier ones, as in the reference.
struct AttnVac {
    double p[6], sc[6];
    int ind[6];   // attn_vac_pos_ind
};
__device__ double atten_factor_vacuum(const AttnVac &a, bool three_d, double x, double y, double z)
{
    const double *p = a.p;
    double af = 0.0;
    if (x < p[0]) {
        if ((y <= (p[3] + p[0] - x)) && (y >= (p[2] - p[0] + x)))
            if (z <= (p[5] + p[0] - x) && (z >= (p[4] - p[0] + x))) af = cube(fabs(x - p[0]) / a.sc[0]);
    } else if (x > p[1]) {
        if ((y <= (p[3] - p[1] + x)) && (y >= (p[2] + p[1] - x)))
            if ((z <= (p[5] - p[1] + x)) && (z >= (p[4] + p[1] - x))) af = cube(fabs(x - p[1]) / a.sc[1]);
    }
    if (y < p[2]) {
        if ((y < (p[2] - p[0] + x)) && (y < (p[2] + p[1] - x)))
            if ((z >= (p[4] - p[2] + y)) && (z <= (p[5] + p[2] - y))) af = cube(fabs(y - p[2]) / a.sc[2]);
    } else if (y > p[3]) {
        if ((y > (p[3] + p[0] - x)) && (y > (p[3] - p[1] + x)))
            if ((z >= (p[4] + p[3] - y)) && (z <= (p[5] - p[3] + y))) af = cube(fabs(y - p[3]) / a.sc[3]);
    }
    if (three_d) {
        if (z < p[4]) {
            if ((z < (p[4] - p[0] + x)) && (z < (p[4] + p[1] - x)))
                if ((z < (p[4] - p[2] + y)) && (z < (p[4] + p[3] - y))) af = cube(fabs(z - p[4]) / a.sc[4]);
        } else if (z > p[5]) {
            if (z > (p[5] + p[0] - x) && (z > (p[5] - p[1] + x)))
                if ((z > (p[5] + p[2] - y)) && (z > (p[5] - p[3] + y))) af = cube(fabs(z - p[5]) / a.sc[5]);
        }
    }
    af = fmin(1.0, af);
    af = fmax(0.0, af);
    return 1.0 - af;
}

// Attenuate_EM_Vacuum (bc_attenuate.F90:151-220): every cell of the
// ghosted grid outside the box of attn_vac_pos_ind has its six components
// scaled by AttenFactorVacuum at their staggered positions.
__global__ void k_attn_vacuum(GridP g, AttnVac a, double *Ex, double *Ey, double *Ez, double *Bx, double *By,
                              double *Bz)
{
    const long long n = g.ncell;
    const bool three_d = g.dims == 3;
    const double x0 = -3.0, y0 = -3.0, z0 = three_d ? -3.0 : 0.0;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const long long jk = c / g.mx;
        const int i = (int)(c - jk * g.mx) + 1, j = (int)(jk % g.my) + 1, k = (int)(jk / g.my) + 1;
        const int ig = i - 3, jg = j - 3, kg = k - 3;
        const bool inside = ig > a.ind[0] && ig < a.ind[1] && jg > a.ind[2] && jg < a.ind[3] &&
                            (!three_d || (kg > a.ind[4] && kg < a.ind[5]));
        if (inside) continue;
        const double xi = (double)i + x0, yj = (double)j + y0, zk = (double)k + z0;
        const double xh = (double)i + 0.5 + x0, yh = (double)j + 0.5 + y0, zh = (double)k + 0.5 + z0;
        Ex[c] = Ex[c] * atten_factor_vacuum(a, three_d, xh, yj, zk);
        Ey[c] = Ey[c] * atten_factor_vacuum(a, three_d, xi, yh, zk);
        Ez[c] = Ez[c] * atten_factor_vacuum(a, three_d, xi, yj, zh);
        Bx[c] = Bx[c] * atten_factor_vacuum(a, three_d, xi, yh, zh);
        By[c] = By[c] * atten_factor_vacuum(a, three_d, xh, yj, zh);
        Bz[c] = Bz[c] * atten_factor_vacuum(a, three_d, xh, yh, zk);
    }
}

// Attenuate_EM_Flow (bc_attenuate.F90:16-98) for a uniform flow: MagFld and
// Drift of the face are the constants b and v.  atnn_domain (:117-131) on
// face side (1..4) with the thickness dl, AttenFactor (:102-115) with the
// scale length sc.
struct AttnFlow {
    double pos, dl, sc, b[3], v[3];
    int side;
};
__device__ __forceinline__ bool atnn_domain(const AttnFlow &a, double xg, double yg)
{
    switch (a.side) {
        case 1: return xg >= a.pos && xg <= a.pos + a.dl;
        case 2: return xg <= a.pos && xg >= a.pos - a.dl;
        case 3: return yg >= a.pos && yg <= a.pos + a.dl;
        default: return yg <= a.pos && yg >= a.pos - a.dl;
    }
}
__device__ __forceinline__ double atten_factor(const AttnFlow &a, double xg, double yg)
{
    const double t = a.side <= 2 ? fabs(xg - a.pos) / a.sc : fabs(yg - a.pos) / a.sc;
    double af = cube(t);
    af = fmin(1.0, af);
    af = fmax(0.0, af);
    return 1.0 - af;
}
__global__ void k_attn_flow(GridP g, AttnFlow a, double *Ex, double *Ey, double *Ez, double *Bx, double *By, double *Bz)
{
    const long long n = g.ncell;
    const double x0 = -3.0, y0 = -3.0;
    // the flow's motional field -v x B, as the reference forms it per component
    const double fx = a.v[2] * a.b[1] - a.v[1] * a.b[2];
    const double fy = a.v[0] * a.b[2] - a.v[2] * a.b[0];
    const double fz = a.v[1] * a.b[0] - a.v[0] * a.b[1];
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const long long jk = c / g.mx;
        const int i = (int)(c - jk * g.mx) + 1, j = (int)(jk % g.my) + 1;
        const double xi = (double)i + x0, yj = (double)j + y0;
        const double xh = (double)i + 0.5 + x0, yh = (double)j + 0.5 + y0;
        if (atnn_domain(a, xh, yj)) Ex[c] = (Ex[c] - fx) * atten_factor(a, xh, yj) + fx;
        if (atnn_domain(a, xi, yh)) Ey[c] = (Ey[c] - fy) * atten_factor(a, xi, yh) + fy;
        if (atnn_domain(a, xi, yj)) Ez[c] = (Ez[c] - fz) * atten_factor(a, xi, yj) + fz;
        if (atnn_domain(a, xi, yh)) Bx[c] = (Bx[c] - a.b[0]) * atten_factor(a, xi, yh) + a.b[0];
        if (atnn_domain(a, xh, yj)) By[c] = (By[c] - a.b[1]) * atten_factor(a, xh, yj) + a.b[1];
        if (atnn_domain(a, xh, yh)) Bz[c] = (Bz[c] - a.b[2]) * atten_factor(a, xh, yh) + a.b[2];
    }
}

// OpenBC_Fld_Right (side 1, bc.F90:411-440) / OpenBC_Fld_Left (side 0,
// :442-469) at the local layer xl: Ey, Ez halved and Bx copied from layer xl
// beyond it, Ex, By, Bz halved from xl on (right) or below xl (left).
__global__ void k_open_fld_x(GridP g, double *Ex, double *Ey, double *Ez, double *Bx, double *By, double *Bz, int xl,
                             int side)
{
    const long long n = g.ncell;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const long long jk = c / g.mx;
        const int i = (int)(c - jk * g.mx) + 1;
        const long long src = (long long)(xl - 1) + g.mx * jk;
        const bool a = side == 1 ? i >= xl + 1 : i <= xl - 1;   // Ey, Ez, Bx
        const bool b = side == 1 ? i >= xl : i <= xl - 1;       // Ex, By, Bz
        if (a) {
            Ey[c] = 0.5 * Ey[c];
            Ez[c] = 0.5 * Ez[c];
            Bx[c] = Bx[src];
        }
        if (b) {
            Ex[c] = 0.5 * Ex[c];
            By[c] = 0.5 * By[c];
            Bz[c] = 0.5 * Bz[c];
        }
    }
}

// ---------------------------------------------------------------------------
// 'open' particle faces along x: OpenBC_Prtl_Right / Left (bc.F90:478-621)
// with dx = 1 (EnforceBC_Final, :333-334).  The particles beyond the face
// become holes (DeletePrtl, mem_prtl.F90:7-22); each particle in the layer
// of width dx inside the face is mirrored across it and appended
// (InsertNewPrtl, mem_prtl.F90:120-133, in slot order), its u lowered by
// gamma v0 with v0 the mean x velocity of flavours 1, 2 in its (j, k)
// column of the layer (OpenBC_MeanPrtlSpeed, bc.F90:603-621; den starts at
// 1), clamped to <= 0 on the right face and >= 0 on the left one.
// ---------------------------------------------------------------------------

// den = 1, vel = 0 over the my * mz columns (col[c], col[ncol + c]).
__global__ void k_open_cols_init(double *col, int ncol)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncol; c += gridDim.x * blockDim.x) {
        col[c] = 1.0;
        col[ncol + c] = 0.0;
    }
}

// Holes beyond the face, layer flags, and the column sums (FP64 atomics: the
// sums' order, and with it the last bit of v0, follows the atomics).
__global__ void k_open_prtl_mark(GridP g, PartF64 p, const Counters *__restrict__ cnt, int side, double wall,
                                 double dx, uint32_t *flag, double *col, double zhole, int *err)
{
    const long long used = cnt->used;
    const int ncol = g.my * g.mz;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < used;
         n += (long long)gridDim.x * blockDim.x) {
        uint32_t f = 0;
        if (p.q[n] != 0.0) {
            const double x = p.x[n];
            if (side == 1 ? x > wall : x < wall) {
                p.q[n] = 0.0;
                p.x[n] = 3.8;
                p.y[n] = 3.8;
                p.z[n] = zhole;
                p.u[n] = 0.0;
                p.v[n] = 0.0;
                p.w[n] = 0.0;
                p.flv[n] = 0;
            } else if (side == 1 ? (x > wall - dx && x < wall) : (x < wall + dx && x > wall)) {
                const int j = (int)p.y[n], k = g.dims == 3 ? (int)p.z[n] : 1;
                if (j < 1 || j > g.my || k < 1 || k > g.mz) {
                    raise_error(err, PIC_DEVERR_RANGE);
                } else {
                    f = 1;
                    if (p.flv[n] <= 2) {
                        const double u = p.u[n], v = p.v[n], w = p.w[n];
                        const double invg = 1.0 / sqrt(1.0 + u * u + v * v + w * w);
                        const int c = (j - 1) + g.my * (k - 1);
                        atomicAdd(col + c, 1.0);
                        atomicAdd(col + ncol + c, u * invg);
                    }
                }
            }
        }
        flag[n] = f;
    }
}

// vel = vel / den per column.
__global__ void k_open_cols_mean(double *col, int ncol)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncol; c += gridDim.x * blockDim.x)
        col[ncol + c] = col[ncol + c] / col[c];
}

constexpr int kOpenTile = 4096;   // slots per block of the stable compaction

// Flagged slots per tile of kOpenTile slots below `used`.
__global__ void __launch_bounds__(256) k_open_tile_counts(const Counters *__restrict__ cnt,
                                                          const uint32_t *__restrict__ flag, uint32_t *counts)
{
    __shared__ uint32_t red[8];
    const long long used = cnt->used;
    const long long base = (long long)blockIdx.x * kOpenTile;
    uint32_t c = 0;
    for (int r = threadIdx.x; r < kOpenTile; r += 256) {
        const long long n = base + r;
        if (n < used) c += flag[n];
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < 8; w++) t += red[w];
        counts[blockIdx.x] = t;
    }
}

// The mirrored copies, appended at used + (rank of the particle among the
// layer's particles in slot order): block b ranks the flags of its tile
// from the tile's offset (stable: lanes, warps and chunks in slot order);
// nothing is written when the copies do not fit.
__global__ void __launch_bounds__(256) k_open_prtl_insert(GridP g, PartF64 p, const Counters *__restrict__ cnt,
                                                          int side, double wall, const uint32_t *__restrict__ flag,
                                                          const uint32_t *__restrict__ offs,
                                                          const uint32_t *__restrict__ total,
                                                          const double *__restrict__ col, long long capacity, int *err)
{
    __shared__ uint32_t wsum[8];
    const long long used = cnt->used;
    const long long m = (long long)*total;
    if (used + m > capacity) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_error(err, PIC_DEVERR_OVERFLOW);
        return;
    }
    const int ncol = g.my * g.mz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t run = offs[blockIdx.x];
    const long long base = (long long)blockIdx.x * kOpenTile;
    for (int r = 0; r < kOpenTile; r += 256) {
        const long long n = base + r + threadIdx.x;
        const bool f = n < used && flag[n] != 0;
        const uint32_t bal = __ballot_sync(0xffffffffu, f);
        if (lane == 0) wsum[warp] = __popc(bal);
        __syncthreads();
        uint32_t before = 0, chunk = 0;
        for (int w = 0; w < 8; w++) {
            if (w < warp) before += wsum[w];
            chunk += wsum[w];
        }
        if (f) {
            uint32_t lt;
            asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
            const long long d = used + (long long)(run + before + __popc(bal & lt));
            const double x = p.x[n], y = p.y[n], z = p.z[n], u = p.u[n], v = p.v[n], w = p.w[n];
            const int j = (int)y, k = g.dims == 3 ? (int)z : 1;
            double v0 = col[ncol + (j - 1) + g.my * (k - 1)];
            if (side == 1 ? v0 > 0.0 : v0 < 0.0) v0 = 0.0;
            const double gamma = sqrt(1.0 + u * u + v * v + w * w);
            p.x[d] = 2.0 * wall - x;
            p.y[d] = y;
            p.z[d] = z;
            p.u[d] = u - gamma * v0;
            p.v[d] = v;
            p.w[d] = w;
            p.q[d] = p.q[n];
            p.flv[d] = p.flv[n];
        }
        run += chunk;
        __syncthreads();
    }
}

__global__ void k_open_prtl_finish(Counters *cnt, const uint32_t *__restrict__ total, long long capacity)
{
    const long long m = (long long)*total;
    if (cnt->used + m <= capacity) cnt->used += m;
}

// ---------------------------------------------------------------------------
// RefPrtlFluidFrameRight (bc_inflow.F90:62-97) for a uniform drift vx: a
// particle beyond the drifted injector layer x1 = xinj + vx c is reflected in
// the frame moving with the flow (ReflectPrtlMovingFrameX, :100-121),
// mirrored to 2 x1 - x, and the current of that move deposited
// (DepositCurrentPIC, deposit.F90:11-103, FP64 atomics into J).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void add_j(double *F, long long c, double v) { atomicAdd(F + c, v); }

__global__ void k_refl_fluid_right(GridP g, PartF64 p, const Counters *__restrict__ cnt, double x1, double drift,
                                   double *Jx, double *Jy, double *Jz, int *err)
{
    const long long used = cnt->used;
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < used;
         n += (long long)gridDim.x * blockDim.x) {
        if (p.q[n] == 0.0) continue;
        const double x0 = p.x[n];
        if (!(x0 > x1)) continue;
        const double y0 = p.y[n], z0 = p.z[n];
        // ReflectPrtlMovingFrameX
        double db, dg;
        if (fabs(drift) < 1.0) {
            db = drift;
            dg = 1.0 / sqrt((1.0 - drift) * (1.0 + drift));
        } else {
            dg = fabs(drift);
            db = sqrt((drift - 1.0) * (drift + 1.0)) / drift;
        }
        double u = p.u[n];
        const double v = p.v[n], w = p.w[n];
        double gamma = sqrt(1.0 + u * u + v * v + w * w);
        db = -db;
        u = dg * u + dg * db * gamma;
        u = -u;
        gamma = sqrt(1.0 + u * u + v * v + w * w);
        db = -db;
        u = dg * u + dg * db * gamma;
        const double x = 2.0 * x1 - x0, y = y0, z = z0;
        // DepositCurrentPIC
        const int i1 = (int)floor(x0), i2 = (int)floor(x), j1 = (int)floor(y0), j2 = (int)floor(y);
        int k1 = (int)floor(z0), k2 = (int)floor(z);
        const bool three = g.dims == 3;
        if (i1 < 1 || i1 > g.mx - 1 || i2 < 1 || i2 > g.mx - 1 || j1 < 1 || j1 > g.my - 1 ||
            (three && (k1 < 1 || k1 > g.mz - 1))) {
            raise_error(err, PIC_DEVERR_RANGE);
            continue;
        }
        p.u[n] = u;
        p.x[n] = x;
        const double qthis = p.q[n] * g.qi;
        const double xr = fmin((double)(min(i1, i2) + 1), fmax((double)max(i1, i2), 0.5 * (x0 + x)));
        const double yr = fmin((double)(min(j1, j2) + 1), fmax((double)max(j1, j2), 0.5 * (y0 + y)));
        const double zr = fmin((double)(min(k1, k2) + 1), fmax((double)max(k1, k2), 0.5 * (z0 + z)));
        const double Fx1 = qthis * (xr - x0), Fy1 = qthis * (yr - y0), Fz1 = qthis * (zr - z0);
        const double Wx1 = 0.5 * (x0 + xr) - i1, Wy1 = 0.5 * (y0 + yr) - j1;
        const double Wx2 = 0.5 * (x + xr) - i2, Wy2 = 0.5 * (y + yr) - j2;
        double Wz1, Wz2;
        if (!three) {
            k1 = 1;
            k2 = 1;
            Wz1 = 0.0;
            Wz2 = 0.0;
        } else {
            Wz1 = 0.5 * (z0 + zr) - k1;
            Wz2 = 0.5 * (z + zr) - k2;
        }
        const double Fx2 = qthis * (x - xr), Fy2 = qthis * (y - yr), Fz2 = qthis * (z - zr);
        auto C = [&](int i, int j, int k) { return cidx(g, i, j, k); };
        add_j(Jx, C(i1, j1, k1), Fx1 * (1.0 - Wy1) * (1.0 - Wz1));
        add_j(Jx, C(i1, j1 + 1, k1), Fx1 * Wy1 * (1.0 - Wz1));
        if (three) {
            add_j(Jx, C(i1, j1, k1 + 1), Fx1 * (1.0 - Wy1) * Wz1);
            add_j(Jx, C(i1, j1 + 1, k1 + 1), Fx1 * Wy1 * Wz1);
        }
        add_j(Jx, C(i2, j2, k2), Fx2 * (1.0 - Wy2) * (1.0 - Wz2));
        add_j(Jx, C(i2, j2 + 1, k2), Fx2 * Wy2 * (1.0 - Wz2));
        if (three) {
            add_j(Jx, C(i2, j2, k2 + 1), Fx2 * (1.0 - Wy2) * Wz2);
            add_j(Jx, C(i2, j2 + 1, k2 + 1), Fx2 * Wy2 * Wz2);
        }
        add_j(Jy, C(i1, j1, k1), Fy1 * (1.0 - Wx1) * (1.0 - Wz1));
        add_j(Jy, C(i1 + 1, j1, k1), Fy1 * Wx1 * (1.0 - Wz1));
        if (three) {
            add_j(Jy, C(i1, j1, k1 + 1), Fy1 * (1.0 - Wx1) * Wz1);
            add_j(Jy, C(i1 + 1, j1, k1 + 1), Fy1 * Wx1 * Wz1);
        }
        add_j(Jy, C(i2, j2, k2), Fy2 * (1.0 - Wx2) * (1.0 - Wz2));
        add_j(Jy, C(i2 + 1, j2, k2), Fy2 * Wx2 * (1.0 - Wz2));
        if (three) {
            add_j(Jy, C(i2, j2, k2 + 1), Fy2 * (1.0 - Wx2) * Wz2);
            add_j(Jy, C(i2 + 1, j2, k2 + 1), Fy2 * Wx2 * Wz2);
        }
        add_j(Jz, C(i1, j1, k1), Fz1 * (1.0 - Wx1) * (1.0 - Wy1));
        add_j(Jz, C(i1 + 1, j1, k1), Fz1 * Wx1 * (1.0 - Wy1));
        add_j(Jz, C(i1, j1 + 1, k1), Fz1 * (1.0 - Wx1) * Wy1);
        add_j(Jz, C(i1 + 1, j1 + 1, k1), Fz1 * Wx1 * Wy1);
        add_j(Jz, C(i2, j2, k2), Fz2 * (1.0 - Wx2) * (1.0 - Wy2));
        add_j(Jz, C(i2 + 1, j2, k2), Fz2 * Wx2 * (1.0 - Wy2));
        add_j(Jz, C(i2, j2 + 1, k2), Fz2 * (1.0 - Wx2) * Wy2);
        add_j(Jz, C(i2 + 1, j2 + 1, k2), Fz2 * Wx2 * Wy2);
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

// Attenuate_EM_Vacuum for the 'attn' faces in the bit mask `faces` (bit n-1
// = bc_face(n)) at pos[n-1] with attn_scale sc[n-1]; returns without a
// launch when the whole grid lies inside (bc_attenuate.F90:158-172).
void launch_bc_attenuate(const GridP &g, double *const E[3], double *const B[3], int faces, const double *pos,
                         const double *sc, cudaStream_t s)
{
    AttnVac a;
    for (int n = 0; n < 6; n++) {
        const bool on = (faces >> n) & 1;
        const bool upper = (n & 1) != 0;   // faces 2, 4, 6
        a.p[n] = on ? pos[n] : (upper ? 2147483647.0 : -2147483647.0);
        a.sc[n] = on ? sc[n] : 1.0;
        a.ind[n] = on ? (upper ? (int)ceil(a.p[n]) + 1 : (int)floor(a.p[n]) - 1) : (upper ? 2147483647 : -2147483647);
    }
    const bool inside = 1 - 3 > a.ind[0] && g.mx - 3 < a.ind[1] && 1 - 3 > a.ind[2] && g.my - 3 < a.ind[3] &&
                        (g.dims == 2 || (1 - 3 > a.ind[4] && g.mz - 3 < a.ind[5]));
    if (inside) return;
    k_attn_vacuum<<<grid_for(g.ncell), kThreads, 0, s>>>(g, a, E[0], E[1], E[2], B[0], B[1], B[2]);
    count_launches(1);
}

// Attenuate_EM_Flow on face `side` (1..4) with a uniform flow; nothing when
// the thickness is 0 or the layer lies outside the grid (:33-35).
void launch_bc_attenuate_flow(const GridP &g, double *const E[3], double *const B[3], int side, double pos, double dl,
                              double sc, const double *b, const double *v, cudaStream_t s)
{
    if (dl == 0.0) return;
    const double o = -3.0;   // x0 = y0
    if (side == 1 && (pos + dl) - o < 1) return;
    if (side == 3 && (pos + dl) - o < 1) return;
    if (side == 2 && (pos - dl) - o > g.mx) return;
    if (side == 4 && (pos - dl) - o > g.my) return;
    AttnFlow a;
    a.pos = pos;
    a.dl = dl;
    a.sc = sc;
    a.side = side;
    for (int d = 0; d < 3; d++) {
        a.b[d] = b[d];
        a.v[d] = v[d];
    }
    k_attn_flow<<<grid_for(g.ncell), kThreads, 0, s>>>(g, a, E[0], E[1], E[2], B[0], B[1], B[2]);
    count_launches(1);
}

// OpenBC_Fld_Left (side 0) / OpenBC_Fld_Right (side 1) at `pos`.
void launch_bc_open_fld_x(const GridP &g, double *const E[3], double *const B[3], int side, double pos, cudaStream_t s)
{
    const int xl = (int)ceil(pos - 0.0 + 3);
    if (side == 1 ? !(xl >= 1 && xl <= g.mx - 1) : !(xl >= 2 && xl <= g.mx)) return;
    k_open_fld_x<<<grid_for(g.ncell), kThreads, 0, s>>>(g, E[0], E[1], E[2], B[0], B[1], B[2], xl, side);
    count_launches(1);
}

// OpenBC_Prtl_Left (side 0) / OpenBC_Prtl_Right (side 1) at `pos` with
// dx = 1; col holds 2 my mz doubles; flag (capacity words), counts
// (capacity / 4096 + 1 words), scan_tmp and total are scratch (the
// radix-sort buffers, free between reorders).
void launch_bc_open_prtl_x(const GridP &g, PartF64 &p, Counters *cnt, int side, double pos, double *col,
                           uint32_t *flag, uint32_t *counts, uint32_t *scan_tmp, uint32_t *total, long long capacity,
                           int *err, cudaStream_t s)
{
    const double wall = pos - 0.0 + 3;
    if (side == 1 ? !(wall < g.mx - 1) : !(wall > 1)) return;
    const int ncol = g.my * g.mz;
    const unsigned tiles = (unsigned)((capacity + kOpenTile - 1) / kOpenTile);
    k_open_cols_init<<<grid_for(ncol), kThreads, 0, s>>>(col, ncol);
    k_open_prtl_mark<<<grid_for(capacity), kThreads, 0, s>>>(g, p, cnt, side, wall, 1.0, flag, col,
                                                             g.dims == 3 ? 3.8 : 1.5, err);
    k_open_cols_mean<<<grid_for(ncol), kThreads, 0, s>>>(col, ncol);
    k_open_tile_counts<<<tiles, 256, 0, s>>>(cnt, flag, counts);
    count_launches(4);
    scan_exclusive_u32(counts, counts, tiles, scan_tmp, total, s);
    k_open_prtl_insert<<<tiles, 256, 0, s>>>(g, p, cnt, side, wall, flag, counts, total, col, capacity, err);
    k_open_prtl_finish<<<1, 1, 0, s>>>(cnt, total, capacity);
    count_launches(2);
}

// RefPrtlFluidFrameRight at the right injector `pos` (bc_face(2)%pos_prtl)
// for the uniform drift vx; nothing when the injector lies at or beyond the
// grid's last layer (xinj_local > mx - 1).
void launch_bc_inflow_reflect(const GridP &g, PartF64 &p, const Counters *cnt, double *const J[3], double pos,
                              double drift, long long capacity, int *err, cudaStream_t s)
{
    const double xinj = pos - 0.0 + 3;
    if (xinj > g.mx - 1) return;
    k_refl_fluid_right<<<grid_for(capacity), kThreads, 0, s>>>(g, p, cnt, xinj + drift * g.c, drift, J[0], J[1], J[2],
                                                               err);
    count_launches(1);
}

}  // namespace pic
