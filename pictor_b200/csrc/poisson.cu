// poisson.cu -- the initial electrostatic field of the Cartesian grid in FP64:
// E = -grad(phi) on the Yee grid with the discrete divergence of CalcDivE
// (src/io/savedata_routines.F90:310-348, the node divergence of the Gauss
// residual in diag.cu) equal to the CIC charge density of the particles.
//
// The reference has no field solver of this kind: its setups start from a
// neutral plasma with E = 0 or set the fields themselves.  The FP32 form keeps
// this one step in FP64 (with the charge-conservation check and the energy
// diagnostics), so that a run that does not start neutral starts with the
// field its charge implies.
//
// With Ex(i) = -(phi(i+1) - phi(i)) (Ex at i + 1/2) and likewise for y and z,
// the divergence at node i is -(L phi)(i), L the 7-point (5-point in 2D)
// periodic Laplacian on the interior nodes.  On a periodic grid L is
// singular with the constants as its null space, so the solve takes the
// density minus its mean (a uniform neutralising background, returned to
// the caller) and finds the phi of zero mean by conjugate gradients on -L,
// which is symmetric positive definite on the mean-free vectors.  Every
// scalar of the iteration stays on the device; the host looks at the residual
// every kCheck iterations.  Reductions are two-level in a fixed order, so the
// solve is deterministic.
#include "common.cuh"
#include "kernels.cuh"

namespace pic {

namespace {

constexpr int kPT = 256;
constexpr int kPBlocks = kSMs * 4;   // blocks of the grid-stride kernels (and partial sums)
constexpr int kCheck = 16;           // iterations between host checks of the residual

struct PGrid {
    int nx, ny, nz;   // interior nodes (nz = 1 in 2D)
    long long n;
    int dims;
};

struct CGScalars {
    double rr, rr_new, pAp, alpha, beta, bb, sum;
};

__device__ __forceinline__ void pijk(const PGrid &q, long long t, int &i, int &j, int &k)
{
    i = (int)(t % q.nx);
    const long long r = t / q.nx;
    j = (int)(r % q.ny);
    k = (int)(r / q.ny);
}
__device__ __forceinline__ long long plin(const PGrid &q, int i, int j, int k)
{
    return (long long)i + (long long)q.nx * ((long long)j + (long long)q.ny * k);
}
__device__ __forceinline__ int pwrap(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

__device__ __forceinline__ double block_reduce(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kPT / 32; w++) t += red[w];
    __syncthreads();
    return t;
}

// b = the interior nodes' density (the ghosted rho of the Gauss diagnostic at
// interior indices 3..n+2); partial sums of b.
__global__ void __launch_bounds__(kPT) k_rhs(GridP g, PGrid q, const double *__restrict__ rho, double *b,
                                             double *partial)
{
    __shared__ double red[kPT / 32];
    double acc = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < q.n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        pijk(q, t, i, j, k);
        const double v = rho[cidx(g, i + 3, j + 3, q.dims == 3 ? k + 3 : 1)];
        b[t] = v;
        acc += v;
    }
    const double s = block_reduce(acc, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// out = the sum of nb partials in a fixed order (one block).
__global__ void __launch_bounds__(kPT) k_sum(const double *__restrict__ partial, int nb, double *out)
{
    __shared__ double red[kPT / 32];
    double acc = 0;
    for (int b = threadIdx.x; b < nb; b += kPT) acc += partial[b];
    const double s = block_reduce(acc, red);
    if (threadIdx.x == 0) *out = s;
}

// b -= mean; x = 0; r = p = b; partial sums of r.r.
__global__ void __launch_bounds__(kPT) k_start(PGrid q, double *b, double *x, double *r, double *p,
                                               const CGScalars *__restrict__ sc, double *partial)
{
    __shared__ double red[kPT / 32];
    const double mean = sc->sum / (double)q.n;
    double acc = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < q.n; t += (long long)gridDim.x * blockDim.x) {
        const double v = b[t] - mean;
        b[t] = v;
        x[t] = 0.0;
        r[t] = v;
        p[t] = v;
        acc += v * v;
    }
    const double s = block_reduce(acc, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// Ap = -L p; partial sums of p.Ap.
__global__ void __launch_bounds__(kPT) k_apply(PGrid q, const double *__restrict__ p, double *Ap, double *partial)
{
    __shared__ double red[kPT / 32];
    double acc = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < q.n; t += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        pijk(q, t, i, j, k);
        const double c = p[t];
        double s = (p[plin(q, pwrap(i - 1, q.nx), j, k)] + p[plin(q, pwrap(i + 1, q.nx), j, k)]) +
                   (p[plin(q, i, pwrap(j - 1, q.ny), k)] + p[plin(q, i, pwrap(j + 1, q.ny), k)]);
        double d = 4.0 * c;
        if (q.dims == 3) {
            s = s + (p[plin(q, i, j, pwrap(k - 1, q.nz))] + p[plin(q, i, j, pwrap(k + 1, q.nz))]);
            d = 6.0 * c;
        }
        const double a = d - s;
        Ap[t] = a;
        acc += c * a;
    }
    const double s = block_reduce(acc, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// alpha = rr / pAp (pAp summed from the partials).
__global__ void __launch_bounds__(kPT) k_alpha(const double *__restrict__ partial, int nb, CGScalars *sc)
{
    __shared__ double red[kPT / 32];
    double acc = 0;
    for (int b = threadIdx.x; b < nb; b += kPT) acc += partial[b];
    const double s = block_reduce(acc, red);
    if (threadIdx.x == 0) {
        sc->pAp = s;
        sc->alpha = s > 0.0 ? sc->rr / s : 0.0;
    }
}

// x += alpha p; r -= alpha Ap; partial sums of r.r.
__global__ void __launch_bounds__(kPT) k_update(PGrid q, double *x, double *r, const double *__restrict__ p,
                                                const double *__restrict__ Ap, const CGScalars *__restrict__ sc,
                                                double *partial)
{
    __shared__ double red[kPT / 32];
    const double alpha = sc->alpha;
    double acc = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < q.n; t += (long long)gridDim.x * blockDim.x) {
        x[t] = x[t] + alpha * p[t];
        const double v = r[t] - alpha * Ap[t];
        r[t] = v;
        acc += v * v;
    }
    const double s = block_reduce(acc, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// beta = rr_new / rr; rr = rr_new.
__global__ void __launch_bounds__(kPT) k_beta(const double *__restrict__ partial, int nb, CGScalars *sc)
{
    __shared__ double red[kPT / 32];
    double acc = 0;
    for (int b = threadIdx.x; b < nb; b += kPT) acc += partial[b];
    const double s = block_reduce(acc, red);
    if (threadIdx.x == 0) {
        sc->beta = sc->rr > 0.0 ? s / sc->rr : 0.0;
        sc->rr = s;
    }
}

// p = r + beta p.
__global__ void __launch_bounds__(kPT) k_direction(PGrid q, const double *__restrict__ r, double *p,
                                                   const CGScalars *__restrict__ sc)
{
    const double beta = sc->beta;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < q.n; t += (long long)gridDim.x * blockDim.x)
        p[t] = r[t] + beta * p[t];
}

// E = -grad(phi) on every cell of the ghosted grid (a ghost cell takes the
// value of its periodic interior image, as the field kernels' halo does);
// 2D: Ez = 0.
template <typename T>
__global__ void __launch_bounds__(kPT) k_efield_from_phi(GridP g, PGrid q, const double *__restrict__ phi, T *Ex, T *Ey,
                                                         T *Ez)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < g.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        const long long jk = c / g.mx;
        const int a = (int)(c - jk * g.mx) + 1, bb = (int)(jk % g.my) + 1, cc = (int)(jk / g.my) + 1;
        const int i = wrap_index(a, g.mx) - 3, j = wrap_index(bb, g.my) - 3;
        const int k = q.dims == 3 ? wrap_index(cc, g.mz) - 3 : 0;
        const double f = phi[plin(q, i, j, k)];
        Ex[c] = (T)(-(phi[plin(q, pwrap(i + 1, q.nx), j, k)] - f));
        Ey[c] = (T)(-(phi[plin(q, i, pwrap(j + 1, q.ny), k)] - f));
        Ez[c] = q.dims == 3 ? (T)(-(phi[plin(q, i, j, pwrap(k + 1, q.nz))] - f)) : (T)0;
    }
}

}  // namespace

int solve_gauss(const GridP &g, void *const E[3], bool fp32, const double *rho, double tol, int max_iter,
                cudaStream_t s, int *iters, double *rel_res, double *rho_mean)
{
    PGrid q;
    q.nx = g.nx;
    q.ny = g.ny;
    q.nz = g.dims == 3 ? g.nz : 1;
    q.dims = g.dims;
    q.n = (long long)q.nx * q.ny * q.nz;
    double *buf = nullptr;
    CGScalars *sc = nullptr;
    cudaError_t e = cudaMalloc(&buf, (4 * (size_t)q.n + kPBlocks) * sizeof(double));
    if (e != cudaSuccess) return PIC_ERR_OOM;
    e = cudaMalloc(&sc, sizeof(CGScalars));
    if (e != cudaSuccess) {
        cudaFree(buf);
        return PIC_ERR_OOM;
    }
    double *x = buf, *r = buf + q.n, *p = buf + 2 * q.n, *Ap = buf + 3 * q.n, *partial = buf + 4 * q.n;
    cudaMemsetAsync(sc, 0, sizeof(CGScalars), s);
    // b in Ap (the right-hand side is not needed after the start)
    k_rhs<<<kPBlocks, kPT, 0, s>>>(g, q, rho, Ap, partial);
    k_sum<<<1, kPT, 0, s>>>(partial, kPBlocks, &sc->sum);
    k_start<<<kPBlocks, kPT, 0, s>>>(q, Ap, x, r, p, sc, partial);
    k_sum<<<1, kPT, 0, s>>>(partial, kPBlocks, &sc->rr);
    cudaMemcpyAsync(&sc->bb, &sc->rr, sizeof(double), cudaMemcpyDeviceToDevice, s);
    count_launches(4);
    CGScalars hs;
    int it = 0;
    int rc = PIC_OK;
    e = cudaMemcpyAsync(&hs, sc, sizeof(hs), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = PIC_ERR_CUDA;
    const double bb = hs.bb;
    double rr = hs.rr;
    while (rc == PIC_OK && bb > 0.0 && it < max_iter && !(rr <= tol * tol * bb)) {
        const int n = max_iter - it < kCheck ? max_iter - it : kCheck;
        for (int m = 0; m < n; m++) {
            k_apply<<<kPBlocks, kPT, 0, s>>>(q, p, Ap, partial);
            k_alpha<<<1, kPT, 0, s>>>(partial, kPBlocks, sc);
            k_update<<<kPBlocks, kPT, 0, s>>>(q, x, r, p, Ap, sc, partial);
            k_beta<<<1, kPT, 0, s>>>(partial, kPBlocks, sc);
            k_direction<<<kPBlocks, kPT, 0, s>>>(q, r, p, sc);
            count_launches(5);
        }
        it += n;
        e = cudaMemcpyAsync(&hs, sc, sizeof(hs), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = PIC_ERR_CUDA;
        rr = hs.rr;
    }
    if (rc == PIC_OK) {
        if (fp32)
            k_efield_from_phi<float><<<kPBlocks, kPT, 0, s>>>(g, q, x, (float *)E[0], (float *)E[1], (float *)E[2]);
        else
            k_efield_from_phi<double><<<kPBlocks, kPT, 0, s>>>(g, q, x, (double *)E[0], (double *)E[1], (double *)E[2]);
        count_launches(1);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = PIC_ERR_CUDA;
    }
    if (iters) *iters = it;
    if (rel_res) *rel_res = bb > 0.0 ? sqrt(rr / bb) : 0.0;
    if (rho_mean) *rho_mean = hs.sum / (double)q.n;
    cudaFree(sc);
    cudaFree(buf);
    if (rc == PIC_OK && bb > 0.0 && !(rr <= tol * tol * bb)) rc = PIC_ERR_TIMEOUT;
    return rc;
}

}  // namespace pic
