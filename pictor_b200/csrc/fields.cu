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
#include "kernels.cuh"

namespace pic {

template <typename T>
struct Coef {
    T h, fc;
    T L[12];
    __host__ __device__ Coef() {}
    __host__ __device__ explicit Coef(const GridP &g) : h((T)g.h), fc((T)g.fc)
    {
        for (int i = 0; i < 12; i++) L[i] = (T)g.lehe[i];
    }
};

// Ghost image along one axis of an interior index a (0 = none).
__device__ __forceinline__ int image_of(int a, int m)
{
    const int n = m - 5;
    if (a <= 5) return a + n;      // 3..5 -> m-2..m
    if (a >= m - 4) return a - n;  // m-4..m-3 -> 1..2
    return 0;
}

// Image along x: none in the slab form, whose x ghosts the neighbouring
// slabs fill (SendRecvFlds / UpdateCurrentAllFaces across ranks).
__device__ __forceinline__ int image_x(const GridP &g, int i) { return g.x_external ? 0 : image_of(i, g.mx); }

// Write v to interior cell (i,j,k) and all of its periodic ghost images.
template <typename T, int DIMS>
__device__ __forceinline__ void store_with_images(const GridP &g, T *F, int i, int j, int k, T v)
{
    const int ii[2] = {i, image_x(g, i)};
    const int jj[2] = {j, image_of(j, g.my)};
    const int kk[2] = {k, DIMS == 3 ? image_of(k, g.mz) : 0};
#pragma unroll
    for (int c = 0; c < (DIMS == 3 ? 2 : 1); c++) {
        if (kk[c] == 0) continue;
#pragma unroll
        for (int b = 0; b < 2; b++) {
            if (jj[b] == 0) continue;
#pragma unroll
            for (int a = 0; a < 2; a++) {
                if (ii[a] == 0) continue;
                F[cidx(g, ii[a], jj[b], kk[c])] = v;
            }
        }
    }
}

template <typename T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }

// ---------------------------------------------------------------------------
// Lehe directional differences, em_update_lehe.F90:223-258 (inv_d = 1).
// ---------------------------------------------------------------------------
template <typename T, int DIMS>
__device__ __forceinline__ T gradX(const GridP &g, const Coef<T> &C, const T *F, long long c0)
{
    const long long sy = g.sy, sz = g.sz;
    T r = C.L[0] * (ld(F + c0 + 1) - ld(F + c0));
    r = r + C.L[3] * (ld(F + c0 + 1 + sy) - ld(F + c0 + sy));
    r = r + C.L[3] * (ld(F + c0 + 1 - sy) - ld(F + c0 - sy));
    if (DIMS == 3) {
        r = r + C.L[4] * (ld(F + c0 + 1 + sz) - ld(F + c0 + sz));
        r = r + C.L[4] * (ld(F + c0 + 1 - sz) - ld(F + c0 - sz));
    }
    r = r + C.L[9] * (ld(F + c0 + 2) - ld(F + c0 - 1));
    return r;
}

template <typename T, int DIMS>
__device__ __forceinline__ T gradY(const GridP &g, const Coef<T> &C, const T *F, long long c0)
{
    const long long sy = g.sy, sz = g.sz;
    T r = C.L[1] * (ld(F + c0 + sy) - ld(F + c0));
    r = r + C.L[5] * (ld(F + c0 + 1 + sy) - ld(F + c0 + 1));
    r = r + C.L[5] * (ld(F + c0 - 1 + sy) - ld(F + c0 - 1));
    if (DIMS == 3) {
        r = r + C.L[6] * (ld(F + c0 + sy + sz) - ld(F + c0 + sz));
        r = r + C.L[6] * (ld(F + c0 + sy - sz) - ld(F + c0 - sz));
    }
    r = r + C.L[10] * (ld(F + c0 + 2 * sy) - ld(F + c0 - sy));
    return r;
}

template <typename T>
__device__ __forceinline__ T gradZ(const GridP &g, const Coef<T> &C, const T *F, long long c0)
{
    const long long sy = g.sy, sz = g.sz;
    T r = C.L[2] * (ld(F + c0 + sz) - ld(F + c0));
    r = r + C.L[7] * (ld(F + c0 + 1 + sz) - ld(F + c0 + 1));
    r = r + C.L[7] * (ld(F + c0 - 1 + sz) - ld(F + c0 - 1));
    r = r + C.L[8] * (ld(F + c0 + sy + sz) - ld(F + c0 + sy));
    r = r + C.L[8] * (ld(F + c0 - sy + sz) - ld(F + c0 - sy));
    r = r + C.L[11] * (ld(F + c0 + 2 * sz) - ld(F + c0 - sz));
    return r;
}

struct CellIter {
    int i, j, k;
    bool ok;
};

// Interior cell of thread (threadIdx.x, threadIdx.y) in block (bx, by, bz)
// of the (32, 8) tiling of the interior.
template <int DIMS>
__device__ __forceinline__ CellIter interior_cell_at(const GridP &g, int bx, int by, int bz)
{
    CellIter it;
    it.i = 3 + bx * blockDim.x + threadIdx.x;
    it.j = 3 + by * blockDim.y + threadIdx.y;
    it.k = DIMS == 3 ? 3 + bz : 1;
    it.ok = it.i <= g.mx - 3 && it.j <= g.my - 3;
    return it;
}
template <int DIMS>
__device__ __forceinline__ CellIter interior_cell(const GridP &g)
{
    return interior_cell_at<DIMS>(g, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// B <- B - (c/2) curl E (UpdateBfieldHalf) + halo (SendRecvFlds(B)).
// ---------------------------------------------------------------------------
template <typename T, int DIMS, int FDTD>
__device__ __forceinline__ void bhalf_at(const GridP &g, const CellIter &it, const T *__restrict__ Ex,
                                         const T *__restrict__ Ey, const T *__restrict__ Ez, T *Bx, T *By, T *Bz)
{
    if (!it.ok) return;
    const Coef<T> C(g);
    const T h = C.h;
    const long long c0 = cidx(g, it.i, it.j, it.k);
    const long long sy = g.sy, sz = g.sz;
    T bx, by, bz;
    if (FDTD == PIC_FDTD_YEE) {  // em_update.F90:65-72
        if (DIMS == 3) {
            bx = (Bx[c0] - h * (ld(Ez + c0 + sy) - ld(Ez + c0))) + h * (ld(Ey + c0 + sz) - ld(Ey + c0));
            by = (By[c0] - h * (ld(Ex + c0 + sz) - ld(Ex + c0))) + h * (ld(Ez + c0 + 1) - ld(Ez + c0));
            bz = (Bz[c0] - h * (ld(Ey + c0 + 1) - ld(Ey + c0))) + h * (ld(Ex + c0 + sy) - ld(Ex + c0));
        } else {
            bx = Bx[c0] - h * (ld(Ez + c0 + sy) - ld(Ez + c0));
            by = By[c0] + h * (ld(Ez + c0 + 1) - ld(Ez + c0));
            bz = (Bz[c0] - h * (ld(Ey + c0 + 1) - ld(Ey + c0))) + h * (ld(Ex + c0 + sy) - ld(Ex + c0));
        }
    } else {  // em_update_lehe.F90:209-216
        if (DIMS == 3) {
            bx = (Bx[c0] - h * gradY<T, 3>(g, C, Ez, c0)) + h * gradZ<T>(g, C, Ey, c0);
            by = (By[c0] - h * gradZ<T>(g, C, Ex, c0)) + h * gradX<T, 3>(g, C, Ez, c0);
            bz = (Bz[c0] - h * gradX<T, 3>(g, C, Ey, c0)) + h * gradY<T, 3>(g, C, Ex, c0);
        } else {
            bx = Bx[c0] - h * gradY<T, 2>(g, C, Ez, c0);
            by = By[c0] + h * gradX<T, 2>(g, C, Ez, c0);
            bz = (Bz[c0] - h * gradX<T, 2>(g, C, Ey, c0)) + h * gradY<T, 2>(g, C, Ex, c0);
        }
    }
    store_with_images<T, DIMS>(g, Bx, it.i, it.j, it.k, bx);
    store_with_images<T, DIMS>(g, By, it.i, it.j, it.k, by);
    store_with_images<T, DIMS>(g, Bz, it.i, it.j, it.k, bz);
}

template <typename T, int DIMS, int FDTD>
__global__ void __launch_bounds__(256) k_bhalf(GridP g, const T *__restrict__ Ex, const T *__restrict__ Ey,
                                               const T *__restrict__ Ez, T *Bx, T *By, T *Bz)
{
    bhalf_at<T, DIMS, FDTD>(g, interior_cell<DIMS>(g), Ex, Ey, Ez, Bx, By, Bz);
}

// Yee E update of one cell (em_update.F90:27-34; Lehe keeps it, em_update_lehe.F90:174-181).
template <typename T, int DIMS>
__device__ __forceinline__ void e_curl(const GridP &g, T fc, const T *Ex, const T *Ey, const T *Ez, const T *Bx,
                                       const T *By, const T *Bz, long long c0, T &ex, T &ey, T &ez)
{
    const long long sy = g.sy, sz = g.sz;
    if (DIMS == 3) {
        ex = (Ex[c0] + fc * (ld(Bz + c0) - ld(Bz + c0 - sy))) - fc * (ld(By + c0) - ld(By + c0 - sz));
        ey = (Ey[c0] + fc * (ld(Bx + c0) - ld(Bx + c0 - sz))) - fc * (ld(Bz + c0) - ld(Bz + c0 - 1));
        ez = (Ez[c0] + fc * (ld(By + c0) - ld(By + c0 - 1))) - fc * (ld(Bx + c0) - ld(Bx + c0 - sy));
    } else {
        ex = Ex[c0] + fc * (ld(Bz + c0) - ld(Bz + c0 - sy));
        ey = Ey[c0] - fc * (ld(Bz + c0) - ld(Bz + c0 - 1));
        ez = (Ez[c0] + fc * (ld(By + c0) - ld(By + c0 - 1))) - fc * (ld(Bx + c0) - ld(Bx + c0 - sy));
    }
}

// Fold partner along one axis of an interior index a (0 = none), see image_of.
// J1 = J + J(x-partner); J2 = J1 + J1(y-partner); J3 = J2 + J2(z-partner):
// the order of comm_fld.F90:15-33 (x faces, then y, then z).  Loads only.
template <typename T, int DIMS>
__device__ __forceinline__ T fold_cell(const GridP &g, const T *__restrict__ J, int i, int j, int k)
{
    const int pi = image_x(g, i), pj = image_of(j, g.my);
    const int pk = DIMS == 3 ? image_of(k, g.mz) : 0;
    auto J1 = [&](int b, int c) -> T {
        T v = J[cidx(g, i, b, c)];
        if (pi) v = v + J[cidx(g, pi, b, c)];
        return v;
    };
    auto J2 = [&](int c) -> T {
        T v = J1(j, c);
        if (pj) v = v + J1(pj, c);
        return v;
    };
    T v = J2(k);
    if (DIMS == 3 && pk) v = v + J2(pk);
    return v;
}

// Zero the J cells fold_cell read (ResetCurrent of the consumed current).
template <typename T, int DIMS>
__device__ __forceinline__ void zero_fold_cells(const GridP &g, T *__restrict__ J, int i, int j, int k)
{
    const int ii[2] = {i, image_x(g, i)};
    const int jj[2] = {j, image_of(j, g.my)};
    const int kk[2] = {k, DIMS == 3 ? image_of(k, g.mz) : 0};
#pragma unroll
    for (int c = 0; c < (DIMS == 3 ? 2 : 1); c++) {
        if (kk[c] == 0) continue;
#pragma unroll
        for (int b = 0; b < 2; b++) {
            if (jj[b] == 0) continue;
#pragma unroll
            for (int a = 0; a < 2; a++) {
                if (ii[a] == 0) continue;
                J[cidx(g, ii[a], jj[b], kk[c])] = (T)0;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// E <- E + c curl B (UpdateEfield) [- fold(J) (AddCurrent)] + halo.
// MODE 0: curl only; 1: curl + fold + AddCurrent, zeroing J; 2: AddCurrent of
// an already folded J alone (phase API); 3: curl + AddCurrent of an already
// folded (and filtered) J.  Every load of a thread precedes its stores, so
// the loads of a thread are in flight together (an interleaved load, zero,
// load sequence on J serialised the memory latency).
// ---------------------------------------------------------------------------
template <typename T, int DIMS, int MODE>
__device__ __forceinline__ void efield_at(const GridP &g, const CellIter &it, T *__restrict__ Ex, T *__restrict__ Ey,
                                          T *__restrict__ Ez, const T *__restrict__ Bx, const T *__restrict__ By,
                                          const T *__restrict__ Bz, T *__restrict__ Jx, T *__restrict__ Jy,
                                          T *__restrict__ Jz)
{
    if (!it.ok) return;
    const long long c0 = cidx(g, it.i, it.j, it.k);
    T ex, ey, ez, jx = (T)0, jy = (T)0, jz = (T)0;
    if (MODE == 2) {
        ex = Ex[c0];
        ey = Ey[c0];
        ez = Ez[c0];
    } else {
        e_curl<T, DIMS>(g, (T)g.fc, Ex, Ey, Ez, Bx, By, Bz, c0, ex, ey, ez);
    }
    if (MODE == 1) {
        jx = fold_cell<T, DIMS>(g, Jx, it.i, it.j, it.k);
        jy = fold_cell<T, DIMS>(g, Jy, it.i, it.j, it.k);
        jz = fold_cell<T, DIMS>(g, Jz, it.i, it.j, it.k);
    } else if (MODE == 2 || MODE == 3) {
        jx = Jx[c0];
        jy = Jy[c0];
        jz = Jz[c0];
    }
    if (MODE != 0) {  // em_update.F90:96-98 with grid_inv_d = 1
        ex = ex - (jx * (T)1) * (T)1;
        ey = ey - (jy * (T)1) * (T)1;
        ez = ez - (jz * (T)1) * (T)1;
    }
    store_with_images<T, DIMS>(g, Ex, it.i, it.j, it.k, ex);
    store_with_images<T, DIMS>(g, Ey, it.i, it.j, it.k, ey);
    store_with_images<T, DIMS>(g, Ez, it.i, it.j, it.k, ez);
    if (MODE == 1) {
        zero_fold_cells<T, DIMS>(g, Jx, it.i, it.j, it.k);
        zero_fold_cells<T, DIMS>(g, Jy, it.i, it.j, it.k);
        zero_fold_cells<T, DIMS>(g, Jz, it.i, it.j, it.k);
    }
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
