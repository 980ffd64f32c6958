// fields.cu -- stencil kernels of the field solver (Yee and Lehe FDTD),
// the periodic halo, the current fold, AddCurrent and the current filter.
//
// Reference: src/maxwell/em_update.F90 (Yee), src/maxwell/em_update_lehe.F90
// (Lehe), src/comm/comm_fld.F90 (halo copy / current fold on one periodic
// rank), src/maxwell/current.F90 (ResetCurrent, moving-average filter).
//
// Design: one thread per interior cell.  A thread computes the new value of
// its cell and also writes every periodic ghost image of that cell, so the
// halo copy that follows each update in the reference (SendRecvFlds) costs no
// extra pass and no extra read.  The same trick folds the current: every ghost
// J cell has exactly one periodic image, so the thread of that image reads it,
// adds it in the order of the reference's x-, y-, z-fold, and zeroes it
// (ResetCurrent fused into the consumer).
//
// The FP64 instantiations keep the reference's operation order and this file
// is compiled without FMA contraction, so the FP64 results equal the serial
// CPU build bit for bit.
#include "common.cuh"
#include "field_math.cuh"
#include "kernels.cuh"

namespace pic {

template <typename T, int DIMS, int FDTD>
__global__ void __launch_bounds__(256) k_bhalf(GridP g, const T *__restrict__ Ex, const T *__restrict__ Ey,
                                               const T *__restrict__ Ez, T *Bx, T *By, T *Bz)
{
    bhalf_at<T, DIMS, FDTD>(g, interior_cell<DIMS>(g), Ex, Ey, Ez, Bx, By, Bz);
}

template <typename T, int DIMS, int MODE>
__global__ void __launch_bounds__(256) k_efield(GridP g, T *__restrict__ Ex, T *__restrict__ Ey, T *__restrict__ Ez,
                                                const T *__restrict__ Bx, const T *__restrict__ By,
                                                const T *__restrict__ Bz, T *__restrict__ Jx, T *__restrict__ Jy,
                                                T *__restrict__ Jz)
{
    efield_at<T, DIMS, MODE>(g, interior_cell<DIMS>(g), Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz);
}

// UpdateCurrentAllFaces as a separate phase: J(interior) <- fold(J).  Each J
// cell is read by exactly one thread, so the in-place update is race free.
template <typename T, int DIMS>
__global__ void __launch_bounds__(256) k_fold(GridP g, T *Jx, T *Jy, T *Jz)
{
    const CellIter it = interior_cell<DIMS>(g);
    if (!it.ok) return;
    const long long c0 = cidx(g, it.i, it.j, it.k);
    const T fx = fold_cell<T, DIMS>(g, Jx, it.i, it.j, it.k);
    const T fy = fold_cell<T, DIMS>(g, Jy, it.i, it.j, it.k);
    const T fz = fold_cell<T, DIMS>(g, Jz, it.i, it.j, it.k);
    Jx[c0] = fx;
    Jy[c0] = fy;
    Jz[c0] = fz;
}

// One pass of the (1/4,1/2,1/4) moving average along `axis` on the interior
// with periodic neighbours (current.F90:55-163 on one periodic rank, where the
// halo refresh before each axis makes the ghost neighbours the periodic
// images).  out and in are distinct buffers.
template <typename T, int DIMS>
__global__ void __launch_bounds__(256) k_filter_axis(GridP g, int axis, const T *__restrict__ in, T *out)
{
    const CellIter it = interior_cell<DIMS>(g);
    if (!it.ok) return;
    int lo[3] = {it.i, it.j, it.k}, hi[3] = {it.i, it.j, it.k};
    const int m = axis == 0 ? g.mx : axis == 1 ? g.my : g.mz;
    lo[axis] = wrap_index(lo[axis] - 1, m);
    hi[axis] = wrap_index(hi[axis] + 1, m);
    const long long c0 = cidx(g, it.i, it.j, it.k);
    const T v = ((T)0.25 * in[cidx(g, lo[0], lo[1], lo[2])] + (T)0.5 * in[c0]) + (T)0.25 * in[cidx(g, hi[0], hi[1], hi[2])];
    out[c0] = v;
}

// ---------------------------------------------------------------------------
// Host launchers.
// ---------------------------------------------------------------------------
static dim3 interior_grid(const GridP &g)
{
    return dim3((unsigned)((g.nx + 31) / 32), (unsigned)((g.ny + 7) / 8), (unsigned)(g.dims == 3 ? g.nz : 1));
}

// ---------------------------------------------------------------------------
// Batched field phases: one persistent launch for all runs of a batch.  A
// CTA takes work items (a (32, 8) block of one run's interior) in turn; the
// run's grid description is copied into shared memory for the item.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int batch_run_of(const int *__restrict__ start, int n, int item)
{
    int lo = 0, hi = n;   // start[lo] <= item < start[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (start[mid] <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Copy the words of *src into *dst with the threads of the block.
template <typename S>
__device__ __forceinline__ void block_copy(S *dst, const S *src)
{
    static_assert(sizeof(S) % 4 == 0, "word copy");
    const int *a = reinterpret_cast<const int *>(src);
    int *b = reinterpret_cast<int *>(dst);
    const int nt = blockDim.x * blockDim.y;
    for (int w = threadIdx.y * blockDim.x + threadIdx.x; w < (int)(sizeof(S) / 4); w += nt) b[w] = a[w];
}

template <int DIMS, int FDTD, int PHASE>   // PHASE 0: B half step, 1: E update + fold + AddCurrent + zero J
__global__ void __launch_bounds__(256) k_field_batch(const BatchRun *__restrict__ runs, const int *__restrict__ start,
                                                     int n, int total)
{
    __shared__ BatchRun sr;
    for (int item = blockIdx.x; item < total; item += gridDim.x) {
        const int r = batch_run_of(start, n, item);
        __syncthreads();   // the previous item is done with sr
        block_copy(&sr, &runs[r]);
        __syncthreads();
        const int local = item - start[r];
        const int bx = local % sr.fb[0], byz = local / sr.fb[0], by = byz % sr.fb[1], bz = byz / sr.fb[1];
        const CellIter it = interior_cell_at<DIMS>(sr.g, bx, by, bz);
        if (PHASE == 0)
            bhalf_at<float, DIMS, FDTD>(sr.g, it, sr.E[0], sr.E[1], sr.E[2], sr.B[0], sr.B[1], sr.B[2]);
        else
            efield_at<float, DIMS, 1>(sr.g, it, sr.E[0], sr.E[1], sr.E[2], sr.B[0], sr.B[1], sr.B[2], sr.J[0], sr.J[1],
                                      sr.J[2]);
    }
}

static unsigned batch_grid(int total)
{
    const int cap = kSMs * 8;
    return (unsigned)(total < cap ? (total > 0 ? total : 1) : cap);
}

void launch_batch_bhalf(int dims, int fdtd, const BatchRun *runs, const int *fstart, int n, int total, cudaStream_t s)
{
    const dim3 block(32, 8, 1);
    const unsigned grid = batch_grid(total);
    if (dims == 3) {
        if (fdtd == PIC_FDTD_YEE) k_field_batch<3, PIC_FDTD_YEE, 0><<<grid, block, 0, s>>>(runs, fstart, n, total);
        else k_field_batch<3, PIC_FDTD_LEHE, 0><<<grid, block, 0, s>>>(runs, fstart, n, total);
    } else {
        if (fdtd == PIC_FDTD_YEE) k_field_batch<2, PIC_FDTD_YEE, 0><<<grid, block, 0, s>>>(runs, fstart, n, total);
        else k_field_batch<2, PIC_FDTD_LEHE, 0><<<grid, block, 0, s>>>(runs, fstart, n, total);
    }
    count_launches(1);
}

void launch_batch_efield(int dims, const BatchRun *runs, const int *fstart, int n, int total, cudaStream_t s)
{
    const dim3 block(32, 8, 1);
    const unsigned grid = batch_grid(total);
    if (dims == 3) k_field_batch<3, PIC_FDTD_YEE, 1><<<grid, block, 0, s>>>(runs, fstart, n, total);
    else k_field_batch<2, PIC_FDTD_YEE, 1><<<grid, block, 0, s>>>(runs, fstart, n, total);
    count_launches(1);
}

__global__ void k_batch_flip(BatchRun *runs, int r) { runs[r].cur ^= 1; }

void launch_batch_flip(BatchRun *runs, int r, cudaStream_t s)
{
    k_batch_flip<<<1, 1, 0, s>>>(runs, r);
    count_launches(1);
}

template <typename T>
void launch_bhalf(const GridP &g, T *const E[3], T *const B[3], cudaStream_t s)
{
    const dim3 grid = interior_grid(g), block(32, 8, 1);
    if (g.dims == 3) {
        if (g.fdtd == PIC_FDTD_YEE) k_bhalf<T, 3, PIC_FDTD_YEE><<<grid, block, 0, s>>>(g, E[0], E[1], E[2], B[0], B[1], B[2]);
        else k_bhalf<T, 3, PIC_FDTD_LEHE><<<grid, block, 0, s>>>(g, E[0], E[1], E[2], B[0], B[1], B[2]);
    } else {
        if (g.fdtd == PIC_FDTD_YEE) k_bhalf<T, 2, PIC_FDTD_YEE><<<grid, block, 0, s>>>(g, E[0], E[1], E[2], B[0], B[1], B[2]);
        else k_bhalf<T, 2, PIC_FDTD_LEHE><<<grid, block, 0, s>>>(g, E[0], E[1], E[2], B[0], B[1], B[2]);
    }
    count_launches(1);
}

template <typename T>
void launch_efield(const GridP &g, int mode, T *const E[3], T *const B[3], T *const J[3], cudaStream_t s)
{
    const dim3 grid = interior_grid(g), block(32, 8, 1);
#define LE(D, M) k_efield<T, D, M><<<grid, block, 0, s>>>(g, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2])
    if (g.dims == 3) {
        if (mode == 0) LE(3, 0);
        else if (mode == 1) LE(3, 1);
        else if (mode == 2) LE(3, 2);
        else LE(3, 3);
    } else {
        if (mode == 0) LE(2, 0);
        else if (mode == 1) LE(2, 1);
        else if (mode == 2) LE(2, 2);
        else LE(2, 3);
    }
#undef LE
    count_launches(1);
}

template <typename T>
void launch_fold(const GridP &g, T *const J[3], cudaStream_t s)
{
    const dim3 grid = interior_grid(g), block(32, 8, 1);
    if (g.dims == 3) k_fold<T, 3><<<grid, block, 0, s>>>(g, J[0], J[1], J[2]);
    else k_fold<T, 2><<<grid, block, 0, s>>>(g, J[0], J[1], J[2]);
    count_launches(1);
}

template <typename T>
void launch_filter(const GridP &g, T *const J[3], T *tmp, cudaStream_t s)
{
    const dim3 grid = interior_grid(g), block(32, 8, 1);
    const size_t bytes = (size_t)g.ncell * sizeof(T);
    for (int c = 0; c < 3; c++) {
        for (int axis = 0; axis < g.dims; axis++) {
            if (g.dims == 3) k_filter_axis<T, 3><<<grid, block, 0, s>>>(g, axis, J[c], tmp);
            else k_filter_axis<T, 2><<<grid, block, 0, s>>>(g, axis, J[c], tmp);
            cudaMemcpyAsync(J[c], tmp, bytes, cudaMemcpyDeviceToDevice, s);
        }
    }
    count_launches(3 * g.dims);
}

template void launch_bhalf<double>(const GridP &, double *const[3], double *const[3], cudaStream_t);
template void launch_bhalf<float>(const GridP &, float *const[3], float *const[3], cudaStream_t);
template void launch_efield<double>(const GridP &, int, double *const[3], double *const[3], double *const[3], cudaStream_t);
template void launch_efield<float>(const GridP &, int, float *const[3], float *const[3], float *const[3], cudaStream_t);
template void launch_fold<double>(const GridP &, double *const[3], cudaStream_t);
template void launch_fold<float>(const GridP &, float *const[3], cudaStream_t);
template void launch_filter<double>(const GridP &, double *const[3], double *, cudaStream_t);
template void launch_filter<float>(const GridP &, float *const[3], float *, cudaStream_t);

}  // namespace pic
