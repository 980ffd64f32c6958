// mover_f32.cu -- the FP32 cell-relative mover's kernels and launchers: the
// per-particle form (before the first reorder), the tiled form (one CTA per
// brick) and the batched form (all runs of an ensemble in one launch).  The
// algorithm and its design are described in mover_f32.cuh.
#include "mover_f32.cuh"

namespace pic {

// ---------------------------------------------------------------------------
// Per-particle form (before the first reorder): grid-stride over the array.
// ---------------------------------------------------------------------------
// Slots [*first, used) (every slot when first is null): a slab moves the
// particles it received since its last reorder here, after the tiled launch.
template <int DIMS, bool XC, bool XS>
__global__ void __launch_bounds__(kThreads) k_move_f32(GridP g, PartF32 p, const Counters *__restrict__ cnt,
                                                       const float *__restrict__ Ex, const float *__restrict__ Ey,
                                                       const float *__restrict__ Ez, const float *__restrict__ Bx,
                                                       const float *__restrict__ By, const float *__restrict__ Bz,
                                                       float *Jx, float *Jy, float *Jz, int *err,
                                                       const uint32_t *__restrict__ first)
{
    TileBox tb = {};
    PackedBounds bd;
    const uint32_t step = gridDim.x * blockDim.x;
    const uint32_t n0 = first ? *first : 0u;
    push_range<DIMS, XC, XS>(g, p, n0 + blockIdx.x * blockDim.x + threadIdx.x, (uint32_t)cnt->used, step, Ex, Ey, Ez,
                             Bx, By, Bz, Jx, Jy, Jz, err, tb, bd);
}

void launch_move_deposit_f32(const GridP &g, const PartF32 &p, const Counters *cnt, float *const E[3],
                             float *const B[3], float *const J[3], int *err, cudaStream_t s)
{
    const int grid = kSMs * 16;
#define PIC_MOVE_PP(D, X, S)                                                                                         \
    k_move_f32<D, X, S><<<grid, kThreads, 0, s>>>(g, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2], err, \
                                                   nullptr)
    const bool xs = g.x_external != 0;
    if (g.dims == 3 && g.exact_charge) {
        if (xs) PIC_MOVE_PP(3, true, true); else PIC_MOVE_PP(3, true, false);
    } else if (g.dims == 3) {
        if (xs) PIC_MOVE_PP(3, false, true); else PIC_MOVE_PP(3, false, false);
    } else {
        if (xs) PIC_MOVE_PP(2, false, true); else PIC_MOVE_PP(2, false, false);
    }
#undef PIC_MOVE_PP
    count_launches(1);
}

// ---------------------------------------------------------------------------
// Tiled form: one CTA per brick.
// ---------------------------------------------------------------------------

template <int DIMS, bool XC, bool PRE, bool XS = false>
__global__ void __launch_bounds__(kTileThreads, 3)
    k_move_f32_tiled(GridP g, PartF32 p, Bricks bk, const float *__restrict__ Ex, const float *__restrict__ Ey,
                     const float *__restrict__ Ez, const float *__restrict__ Bx, const float *__restrict__ By,
                     const float *__restrict__ Bz, float *Jx, float *Jy, float *Jz, int *err)
{
    extern __shared__ __align__(16) float sm[];
    __shared__ TileShared ts;
    move_brick<DIMS, XC, PRE, XS>(g, p, bk, blockIdx.x, sm, ts, Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz, err);
}

// The node averages of every interior node (node_avg, the same expressions
// as the bricks' own staging), for the tiled mover's boxes.  A (32, 8) block
// covers 32 x 8 nodes of kNodeKz consecutive z planes (3D).
constexpr int kNodeKz = 4;
template <int DIMS>
__global__ void __launch_bounds__(kThreads) k_node_avg(GridP g, const float *__restrict__ Ex, const float *__restrict__ Ey,
                                                       const float *__restrict__ Ez, const float *__restrict__ Bx,
                                                       const float *__restrict__ By, const float *__restrict__ Bz,
                                                       float4 *nodeA, float2 *nodeB)
{
    const int sy = (int)g.sy, sz = (int)g.sz;
    const int i = 3 + blockIdx.x * 32 + threadIdx.x, j = 3 + blockIdx.y * 8 + threadIdx.y;
    if (i > g.nx + 2 || j > g.ny + 2) return;
    for (int z = 0; z < (DIMS == 3 ? kNodeKz : 1); z++) {
        const int k = DIMS == 3 ? 3 + blockIdx.z * kNodeKz + z : 1;
        if (DIMS == 3 && k > g.nz + 2) break;
        const int nd = (int)cidx(g, i, j, k);
        float4 A;
        float2 Bv;
        node_avg<DIMS>(Ex, Ey, Ez, Bx, By, Bz, nd, sy, sz, g.bext_f[0], g.bext_f[1], g.bext_f[2], A, Bv);
        nodeA[nd] = A;
        nodeB[nd] = Bv;
    }
}

// The tiled mover for all runs of a batch in one launch: CTA b takes brick b
// of the concatenated brick list (the run's description copied into shared
// memory).
__device__ __forceinline__ int batch_run_of_m(const int *__restrict__ start, int n, int item)
{
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (start[mid] <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <int DIMS, bool XC>
__global__ void __launch_bounds__(kTileThreads, 3)
    k_move_f32_batch(const BatchRun *__restrict__ runs, const int *__restrict__ start, int n)
{
    extern __shared__ __align__(16) float sm[];
    __shared__ TileShared ts;
    __shared__ BatchRun sr;
    const int item = blockIdx.x;
    const int r = batch_run_of_m(start, n, item);
    {
        const int *a = reinterpret_cast<const int *>(&runs[r]);
        int *d = reinterpret_cast<int *>(&sr);
        for (int w = threadIdx.x; w < (int)(sizeof(BatchRun) / 4); w += kTileThreads) d[w] = a[w];
    }
    __syncthreads();
    move_brick<DIMS, XC>(sr.g, sr.p[sr.cur], sr.bk, item - start[r], sm, ts, sr.E[0], sr.E[1], sr.E[2], sr.B[0], sr.B[1],
                     sr.B[2], sr.J[0], sr.J[1], sr.J[2], sr.err);
}

void launch_batch_move(int dims, bool exact_charge, const BatchRun *runs, const int *mstart, int n, int total,
                       cudaStream_t s)
{
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_move_f32_batch<3, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
        cudaFuncSetAttribute(k_move_f32_batch<3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
        cudaFuncSetAttribute(k_move_f32_batch<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
        attr_set = true;
    }
    if (total <= 0) return;
    if (dims == 3 && exact_charge) k_move_f32_batch<3, true><<<total, kTileThreads, kBrickSmemBytes, s>>>(runs, mstart, n);
    else if (dims == 3) k_move_f32_batch<3, false><<<total, kTileThreads, kBrickSmemBytes, s>>>(runs, mstart, n);
    else k_move_f32_batch<2, false><<<total, kTileThreads, kBrickSmemBytes, s>>>(runs, mstart, n);
    count_launches(1);
}

void launch_move_deposit_f32_tiled(const GridP &g, const PartF32 &p, const Bricks &bk, const Counters *cnt,
                                   float *const E[3], float *const B[3], float *const J[3], int *err, cudaStream_t s)
{
    static bool attr_set = false;
    const int bytes = bk.smem_floats * 4;
    if (!attr_set) {
        cudaFuncSetAttribute(k_move_f32_tiled<3, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
        cudaFuncSetAttribute(k_move_f32_tiled<3, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
        cudaFuncSetAttribute(k_move_f32_tiled<2, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
        cudaFuncSetAttribute(k_move_f32_tiled<3, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
        cudaFuncSetAttribute(k_move_f32_tiled<3, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
        cudaFuncSetAttribute(k_move_f32_tiled<2, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
        cudaFuncSetAttribute(k_move_f32_tiled<3, false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kBrickSmemBytes);
        cudaFuncSetAttribute(k_move_f32_tiled<3, true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kBrickSmemBytes);
        cudaFuncSetAttribute(k_move_f32_tiled<2, false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kBrickSmemBytes);
        attr_set = true;
    }
    if (g.x_external) {
        // a slab: the box's x cells include the ghost layers, which the node
        // arrays (interior nodes only) do not hold, so each brick averages
        // its own box
        if (g.dims == 3 && g.exact_charge)
            k_move_f32_tiled<3, true, false, true><<<bk.ntiles, kTileThreads, bytes, s>>>(
                g, p, bk, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2], err);
        else if (g.dims == 3)
            k_move_f32_tiled<3, false, false, true><<<bk.ntiles, kTileThreads, bytes, s>>>(
                g, p, bk, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2], err);
        else
            k_move_f32_tiled<2, false, false, true><<<bk.ntiles, kTileThreads, bytes, s>>>(
                g, p, bk, E[0], E[1], E[2], B[0], B[1], B[2], J[0], J[1], J[2], err);
        // the particles appended since the reorder (received from the
        // neighbours) are in no brick's range: moved one per thread
        const uint32_t *first = bk.tile_start + bk.ntiles;
        const int grid = kSMs * 4;
        if (g.dims == 3 && g.exact_charge)
            k_move_f32<3, true, true><<<grid, kThreads, 0, s>>>(g, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0],
                                                               J[1], J[2], err, first);
        else if (g.dims == 3)
            k_move_f32<3, false, true><<<grid, kThreads, 0, s>>>(g, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0],
                                                                J[1], J[2], err, first);
        else
            k_move_f32<2, false, true><<<grid, kThreads, 0, s>>>(g, p, cnt, E[0], E[1], E[2], B[0], B[1], B[2], J[0],
                                                                J[1], J[2], err, first);
        count_launches(2);
        return;
    }
    const bool pre = bk.nodeA != nullptr;
    if (pre) {
        const dim3 grid((unsigned)((g.nx + 31) / 32), (unsigned)((g.ny + 7) / 8),
                        (unsigned)(g.dims == 3 ? (g.nz + kNodeKz - 1) / kNodeKz : 1)),
            block(32, 8, 1);
        if (g.dims == 3)
            k_node_avg<3><<<grid, block, 0, s>>>(g, E[0], E[1], E[2], B[0], B[1], B[2], bk.nodeA, bk.nodeB);
        else
            k_node_avg<2><<<grid, block, 0, s>>>(g, E[0], E[1], E[2], B[0], B[1], B[2], bk.nodeA, bk.nodeB);
        count_launches(1);
    }
#define PIC_MOVE_TILED(D, X, P)                                                                                      \
    k_move_f32_tiled<D, X, P><<<bk.ntiles, kTileThreads, bytes, s>>>(g, p, bk, E[0], E[1], E[2], B[0], B[1], B[2], J[0], \
                                                                    J[1], J[2], err)
    if (g.dims == 3 && g.exact_charge) {
        if (pre) PIC_MOVE_TILED(3, true, true); else PIC_MOVE_TILED(3, true, false);
    } else if (g.dims == 3) {
        if (pre) PIC_MOVE_TILED(3, false, true); else PIC_MOVE_TILED(3, false, false);
    } else {
        if (pre) PIC_MOVE_TILED(2, false, true); else PIC_MOVE_TILED(2, false, false);
    }
#undef PIC_MOVE_TILED
    count_launches(1);
}

}  // namespace pic
