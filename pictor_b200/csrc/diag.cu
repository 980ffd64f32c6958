// diag.cu -- FP64 diagnostics on the device.
//
// Reference: src/io/savedata_routines.F90:265-348 (CalcEnergy, CalcPrtlEnergy,
// CalcFldEnergy, CalcDivE).  Field energy is a deterministic two-level
// reduction (per-block partial sums in a scratch array, then one block adds
// them in block order); the Gauss residual deposits the CIC charge density of
// q*qi at nodes, folded periodically, and reports max |divE - rho| with divE
// the backward-difference node divergence of CalcDivE.
#include "common.cuh"
#include "kernels.cuh"

namespace pic {

constexpr int kDiagThreads = 256;

int field_energy_blocks(const GridP &g)
{
    const long long nint = (long long)g.nx * g.ny * (g.dims == 3 ? g.nz : 1);
    long long b = (nint + kDiagThreads * 8 - 1) / (kDiagThreads * 8);
    if (b > kSMs * 8) b = kSMs * 8;
    return (int)(b < 1 ? 1 : b);
}

__device__ __forceinline__ void interior_ijk(const GridP &g, long long t, int &i, int &j, int &k)
{
    i = 3 + (int)(t % g.nx);
    const long long r = t / g.nx;
    j = 3 + (int)(r % g.ny);
    k = g.dims == 3 ? 3 + (int)(r / g.ny) : 1;
}

__device__ __forceinline__ double block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kDiagThreads / 32; w++) t += red[w];
    return t;
}

template <typename T>
__global__ void __launch_bounds__(kDiagThreads) k_field_energy_partial(GridP g, const T *__restrict__ Ex, const T *__restrict__ Ey,
                                                                       const T *__restrict__ Ez, const T *__restrict__ Bx,
                                                                       const T *__restrict__ By, const T *__restrict__ Bz,
                                                                       double *partials)
{
    __shared__ double red[kDiagThreads / 32];
    const long long nint = (long long)g.nx * g.ny * (g.dims == 3 ? g.nz : 1);
    double eb = 0, ee = 0;
    const double dtheta = 2.0 * 3.14159265358979323846264 / g.ny;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        interior_ijk(g, t, i, j, k);
        const long long c = cidx(g, i, j, k);
        const double bx = Bx[c], by = By[c], bz = Bz[c], ex = Ex[c], ey = Ey[c], ez = Ez[c];
        if (g.geom == PIC_GEOM_CYLINDRICAL) {
            // CalcFldEnergy_cyl (cyl_savedata_routines.F90:8-31): r weights, axis cell excluded
            if (i < 4) continue;
            const double r = ((double)i - 3.0) + -0.5, rp = r + 0.5;
            eb += ((r * (bx * bx) + rp * (by * by)) + rp * (bz * bz)) * dtheta;
            ee += ((rp * (ex * ex) + r * (ey * ey)) + r * (ez * ez)) * dtheta;
        } else {
            eb += (bx * bx + by * by) + bz * bz;
            ee += (ex * ex + ey * ey) + ez * ez;
        }
    }
    const double sb = block_sum(eb, red);
    const double se = block_sum(ee, red);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = sb;
        partials[2 * blockIdx.x + 1] = se;
    }
}

__global__ void k_sum_partials(const double *__restrict__ partials, int nblocks, double *out2)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double sb = 0, se = 0;
    for (int b = 0; b < nblocks; b++) {
        sb += partials[2 * b];
        se += partials[2 * b + 1];
    }
    out2[0] = sb;
    out2[1] = se;
}

void launch_field_energy(const GridP &g, const void *const E[3], const void *const B[3], bool fp32, double *partials,
                         int nblocks, double *out2, cudaStream_t s)
{
    if (fp32)
        k_field_energy_partial<float><<<nblocks, kDiagThreads, 0, s>>>(
            g, (const float *)E[0], (const float *)E[1], (const float *)E[2], (const float *)B[0], (const float *)B[1],
            (const float *)B[2], partials);
    else
        k_field_energy_partial<double><<<nblocks, kDiagThreads, 0, s>>>(
            g, (const double *)E[0], (const double *)E[1], (const double *)E[2], (const double *)B[0],
            (const double *)B[1], (const double *)B[2], partials);
    k_sum_partials<<<1, 32, 0, s>>>(partials, nblocks, out2);
    count_launches(1);
    count_launches(1);
}

// ---------------------------------------------------------------------------
// Kinetic energy per species (CalcPrtlEnergy, savedata_routines.F90:283-308),
// with the particle weight wtp = |q| (charge = weight * FlvrCharge).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void add_species_energy(const GridP &g, double masse, int flv, double q, double u, double v,
                                                   double w, double *acc)
{
    const double c = g.c;
    const double gm = sqrt(((1.0 + u * u) + v * v) + w * w);
    const double wt = fabs(q);
    if (q > 0) acc[flv] += (((gm - 1.0) * wt) * (q * g.qi / g.qm[flv])) * c * c;
    if (q < 0) acc[flv] += ((gm - 1.0) * wt) * ((masse * c) * c);
}

__global__ void __launch_bounds__(kDiagThreads) k_pe_f64(GridP g, PartF64 p, const Counters *__restrict__ cnt, double masse,
                                                         double *out)
{
    double acc[PIC_MAX_FLVR + 1];
    for (int f = 0; f <= PIC_MAX_FLVR; f++) acc[f] = 0;
    const long long n = cnt->used;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int flv = p.flv[i];
        if (flv <= 0 || flv > PIC_MAX_FLVR) continue;
        add_species_energy(g, masse, flv, p.q[i], p.u[i], p.v[i], p.w[i], acc);
    }
    for (int f = 1; f <= PIC_MAX_FLVR; f++) {
        double v = acc[f];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(out + f - 1, v);
    }
}

__global__ void __launch_bounds__(kDiagThreads) k_pe_f32(GridP g, PartF32 p, const Counters *__restrict__ cnt, double masse,
                                                         double *out)
{
    double acc[PIC_MAX_FLVR + 1];
    for (int f = 0; f <= PIC_MAX_FLVR; f++) acc[f] = 0;
    const long long n = cnt->used;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int flv = (int)(p.key[i] >> kFlvShift);
        if (flv == 0) continue;
        add_species_energy(g, masse, flv, (double)p.w[i], (double)p.ux[i], (double)p.uy[i], (double)p.uz[i], acc);
    }
    for (int f = 1; f <= PIC_MAX_FLVR; f++) {
        double v = acc[f];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(out + f - 1, v);
    }
}

void launch_particle_energy_f64(const GridP &g, const PartF64 &p, const Counters *cnt, double masse, double *out,
                                cudaStream_t s)
{
    k_pe_f64<<<kSMs * 4, kDiagThreads, 0, s>>>(g, p, cnt, masse, out);
    count_launches(1);
}

void launch_particle_energy_f32(const GridP &g, const PartF32 &p, const Counters *cnt, double masse, double *out,
                                cudaStream_t s)
{
    k_pe_f32<<<kSMs * 4, kDiagThreads, 0, s>>>(g, p, cnt, masse, out);
    count_launches(1);
}

// ---------------------------------------------------------------------------
// Gauss residual
// ---------------------------------------------------------------------------
__device__ __forceinline__ void deposit_rho(const GridP &g, double *rho, double *rho_pos, int i, int j, int k, double dx,
                                            double dy, double dz, double q)
{
    for (int nn = 0; nn < (g.dims == 3 ? 8 : 4); nn++) {
        const double w = ((nn & 1) ? dx : 1.0 - dx) * ((nn & 2) ? dy : 1.0 - dy) * ((nn & 4) ? dz : 1.0 - dz);
        const int a = wrap_index(i + (nn & 1), g.mx), b = wrap_index(j + ((nn >> 1) & 1), g.my);
        const int c = g.dims == 3 ? wrap_index(k + ((nn >> 2) & 1), g.mz) : 1;
        const long long o = cidx(g, a, b, c);
        atomicAdd(rho + o, q * w);
        if (q > 0) atomicAdd(rho_pos + o, q * w);
    }
}

__global__ void k_rho_f64(GridP g, PartF64 p, const Counters *__restrict__ cnt, double *rho, double *rho_pos)
{
    const long long n = cnt->used;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        if (p.flv[t] == 0) continue;
        const double x = p.x[t], y = p.y[t], z = p.z[t];
        if (!(x >= 1.0 && x < g.mx && y >= 1.0 && y < g.my)) continue;
        const int i = (int)floor(x), j = (int)floor(y);
        const int k = g.dims == 3 ? (int)floor(z) : 1;
        if (g.dims == 3 && !(z >= 1.0 && z < g.mz)) continue;
        deposit_rho(g, rho, rho_pos, i, j, k, x - i, y - j, g.dims == 3 ? z - k : 0.0, p.q[t] * g.qi);
    }
}

__global__ void k_rho_f32(GridP g, PartF32 p, const Counters *__restrict__ cnt, double *rho, double *rho_pos)
{
    const long long n = cnt->used;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const uint32_t key = p.key[t];
        if ((key >> kFlvShift) == 0) continue;
        const int cell = (int)(key & kCellMask);
        const int i = cell % g.mx + 1, jk = cell / g.mx, j = jk % g.my + 1, k = jk / g.my + 1;
        deposit_rho(g, rho, rho_pos, i, j, k, (double)p.dx[t], (double)p.dy[t], g.dims == 3 ? (double)p.dz[t] : 0.0,
                    (double)p.w[t] * g.qi);
    }
}

template <typename T>
__global__ void __launch_bounds__(kDiagThreads) k_gauss_max(GridP g, const T *__restrict__ Ex, const T *__restrict__ Ey,
                                                            const T *__restrict__ Ez, const double *__restrict__ rho,
                                                            const double *__restrict__ rho_pos, double *out2)
{
    const long long nint = (long long)g.nx * g.ny * (g.dims == 3 ? g.nz : 1);
    double res = 0, rm = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nint; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        interior_ijk(g, t, i, j, k);
        const long long c = cidx(g, i, j, k);
        double div = ((double)Ex[c] - (double)Ex[c - 1]) + ((double)Ey[c] - (double)Ey[c - g.sy]);
        if (g.dims == 3) div = div + ((double)Ez[c] - (double)Ez[c - g.sz]);
        res = fmax(res, fabs(div - rho[c]));
        rm = fmax(rm, fabs(rho_pos[c]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        res = fmax(res, __shfl_down_sync(0xffffffffu, res, o));
        rm = fmax(rm, __shfl_down_sync(0xffffffffu, rm, o));
    }
    if ((threadIdx.x & 31) == 0) {
        // non-negative doubles order like their bit patterns
        atomicMax((unsigned long long *)out2, (unsigned long long)__double_as_longlong(res));
        atomicMax((unsigned long long *)(out2 + 1), (unsigned long long)__double_as_longlong(rm));
    }
}

// The CIC charge density alone (the initial Gauss solve, poisson.cu).
void launch_rho_f64(const GridP &g, const PartF64 &p, const Counters *cnt, double *rho, double *rho_pos, cudaStream_t s)
{
    cudaMemsetAsync(rho, 0, (size_t)g.ncell * sizeof(double), s);
    cudaMemsetAsync(rho_pos, 0, (size_t)g.ncell * sizeof(double), s);
    k_rho_f64<<<kSMs * 8, 256, 0, s>>>(g, p, cnt, rho, rho_pos);
    count_launches(1);
}

void launch_rho_f32(const GridP &g, const PartF32 &p, const Counters *cnt, double *rho, double *rho_pos, cudaStream_t s)
{
    cudaMemsetAsync(rho, 0, (size_t)g.ncell * sizeof(double), s);
    cudaMemsetAsync(rho_pos, 0, (size_t)g.ncell * sizeof(double), s);
    k_rho_f32<<<kSMs * 8, 256, 0, s>>>(g, p, cnt, rho, rho_pos);
    count_launches(1);
}

void launch_gauss_f64(const GridP &g, const PartF64 &p, const Counters *cnt, const double *const E[3], double *rho,
                      double *rho_pos, double *out2, cudaStream_t s)
{
    cudaMemsetAsync(rho, 0, (size_t)g.ncell * sizeof(double), s);
    cudaMemsetAsync(rho_pos, 0, (size_t)g.ncell * sizeof(double), s);
    cudaMemsetAsync(out2, 0, 2 * sizeof(double), s);
    k_rho_f64<<<kSMs * 8, 256, 0, s>>>(g, p, cnt, rho, rho_pos);
    count_launches(1);
    k_gauss_max<double><<<field_energy_blocks(g), kDiagThreads, 0, s>>>(g, E[0], E[1], E[2], rho, rho_pos, out2);
    count_launches(1);
}

void launch_gauss_f32(const GridP &g, const PartF32 &p, const Counters *cnt, const float *const E[3], double *rho,
                      double *rho_pos, double *out2, cudaStream_t s)
{
    cudaMemsetAsync(rho, 0, (size_t)g.ncell * sizeof(double), s);
    cudaMemsetAsync(rho_pos, 0, (size_t)g.ncell * sizeof(double), s);
    cudaMemsetAsync(out2, 0, 2 * sizeof(double), s);
    k_rho_f32<<<kSMs * 8, 256, 0, s>>>(g, p, cnt, rho, rho_pos);
    count_launches(1);
    k_gauss_max<float><<<field_energy_blocks(g), kDiagThreads, 0, s>>>(g, E[0], E[1], E[2], rho, rho_pos, out2);
    count_launches(1);
}

}  // namespace pic
