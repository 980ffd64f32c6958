// bricks.cu -- the reorder of the FP32 form: particles grouped by brick.
//
// The reference reorders its particle array every prtl_reorder_period steps
// by cell (ReorderPrtlArr, src/mem/mem_prtl.F90:166-301) so that the mover
// walks memory in cell order; holes are dropped.  The FP32 form keeps that
// role and cadence but groups by brick, a block of TX x TY x TZ interior
// cells, which is the unit the tiled mover (mover_f32.cu) gives one CTA:
//
//   1. brick id per particle; per-brick counts (warp-aggregated atomics),
//   2. exclusive scan of the counts -> tile_start (first particle of every
//      brick; the last entry is the live count),
//   3. each particle takes the next slot of its brick from an atomic cursor
//      (one atomic per run of equal bricks within a warp); the slot records
//      where the particle came from and its key,
//   4. the per-brick boxes the mover starts from (the bricks themselves),
//      and max |w| over the live particles (the mover's fixed-point scale),
//   5. one CTA per brick orders the brick's particles by cell (a counting
//      sort in shared memory) and lays them out transposed: the sorted list
//      is cut into R = cells-per-brick rows of about ppc particles and stored
//      column by column, so consecutive slots hold particles of consecutive
//      cells.  The mover gives consecutive slots to the lanes of a warp, so
//      its node gathers and current atomics in shared memory hit neighbouring
//      words (few bank conflicts) instead of random cells of the brick.  The
//      payload moves once, from the old slot straight to the final one.
//
// Holes are dropped, as in the reference.  The order of particles within a
// cell follows shared-memory atomics.  The FP32 step does not depend on the
// order beyond the rounding of its FP32 current sums, which is
// order-dependent in any case.
#include "common.cuh"
#include "kernels.cuh"

namespace pic {

__device__ __forceinline__ uint32_t lanemask_lt_b()
{
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// a / t[d] of a brick axis by multiply-shift (a < 2^28).
__device__ __forceinline__ uint32_t brick_axis(const Bricks &bk, int d, int a)
{
    return bk.t[d] == 1 ? (uint32_t)a : (uint32_t)fast_div((unsigned)a, bk.tmagic[d], bk.tshift[d]);
}

// Brick of an interior cell (1-based indices 3..n+2), x fastest.
__device__ __forceinline__ uint32_t brick_of(const Bricks &bk, int i, int j, int k)
{
    const uint32_t bx = brick_axis(bk, 0, i - 3), by = brick_axis(bk, 1, j - 3), bz = brick_axis(bk, 2, k - 3);
    return bx + (uint32_t)bk.nb[0] * (by + (uint32_t)bk.nb[1] * bz);
}

constexpr uint32_t kNoBrick = 0xffffffffu;

// Runs of 32 slots a warp loads before it works on them (count and slots
// passes): the loads of four runs are in flight at once.
constexpr int kRuns = 4;

// 1. brick id of every slot (kNoBrick for holes) and per-brick counts.
__global__ void __launch_bounds__(kThreads) k_brick_count(GridP g, Bricks bk, PartF32 p, const Counters *__restrict__ cnt,
                                                          uint32_t *bid, int *err)
{
    const long long used = cnt->used;
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x * kRuns;
    uint32_t wmax = 0;   // max |w| bits seen by this thread
    for (long long base = ((long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) * kRuns; base < used;
         base += stride) {
        uint32_t key[kRuns], wb[kRuns];
#pragma unroll
        for (int u = 0; u < kRuns; u++) {
            const long long n = base + 32 * u + lane;
            key[u] = n < used ? p.key[n] : 0u;
            wb[u] = n < used ? __float_as_uint(fabsf(p.w[n])) : 0u;
        }
#pragma unroll
        for (int u = 0; u < kRuns; u++) {
            const long long n = base + 32 * u + lane;
            uint32_t b = kNoBrick;
            if ((key[u] >> kFlvShift) != 0) {   // holes and slots past `used` have key 0
                int i, j, k;
                decode_cell(g, (int)(key[u] & kCellMask), i, j, k);
                if (i < 3 || i > g.mx - 3 || j < 3 || j > g.my - 3 ||
                    (g.dims == 3 ? (k < 3 || k > g.mz - 3) : k != 1)) {
                    raise_error(err, PIC_DEVERR_RANGE);  // dropped like a hole
                } else {
                    b = brick_of(bk, i, j, g.dims == 3 ? k : 3);
                }
                wmax = max(wmax, wb[u]);   // |w| bit patterns order as integers
            }
            if (n < used) bid[n] = b;
            const uint32_t peers = __match_any_sync(0xffffffffu, b);
            if (b != kNoBrick && (peers & lanemask_lt_b()) == 0) atomicAdd(&bk.count[b], (uint32_t)__popc(peers));
        }
    }
    // one atomic per block
    __shared__ uint32_t s_w[kThreads / 32];
    wmax = __reduce_max_sync(0xffffffffu, wmax);
    if (lane == 0) s_w[threadIdx.x >> 5] = wmax;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t m = 0;
        for (int w = 0; w < kThreads / 32; w++) m = max(m, s_w[w]);
        if (m) atomicMax(bk.wmax_bits, m);
    }
}

// 3. the next free slot of its brick for every live particle: the slot gets
//    the particle's source index (src) and key (out.key, read by step 5).
__global__ void __launch_bounds__(kThreads) k_brick_slots(Bricks bk, PartF32 in, PartF32 out,
                                                          const uint32_t *__restrict__ bid,
                                                          const Counters *__restrict__ cnt)
{
    const long long used = cnt->used;
    const int lane = threadIdx.x & 31;
    const long long stride = (long long)gridDim.x * blockDim.x * kRuns;
    for (long long base = ((long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) * kRuns; base < used;
         base += stride) {
        uint32_t bs[kRuns], key[kRuns];
#pragma unroll
        for (int u = 0; u < kRuns; u++) {
            const long long n = base + 32 * u + lane;
            bs[u] = n < used ? bid[n] : kNoBrick;
            key[u] = n < used ? in.key[n] : 0u;
        }
        // the cursor atomics of all runs issued before any result is used
        uint32_t peers[kRuns], slot[kRuns];
#pragma unroll
        for (int u = 0; u < kRuns; u++) {
            peers[u] = __match_any_sync(0xffffffffu, bs[u]);
            slot[u] = 0;
            if (bs[u] != kNoBrick && (peers[u] & lanemask_lt_b()) == 0)
                slot[u] = atomicAdd(&bk.cursor[bs[u]], (uint32_t)__popc(peers[u]));
        }
#pragma unroll
        for (int u = 0; u < kRuns; u++) {
            const long long n = base + 32 * u + lane;
            const int leader = __ffs(peers[u]) - 1;
            const uint32_t at = __shfl_sync(0xffffffffu, slot[u], leader) + (uint32_t)__popc(peers[u] & lanemask_lt_b());
            if (bs[u] != kNoBrick) {
                out.key[at] = key[u];
                bk.src[at] = (uint32_t)n;
            }
        }
    }
}

// Slot of sorted position s in the transposed layout of N particles over R
// rows: row r holds sorted positions [r (C-1) + min(r, L), ...) with C =
// ceil(N / R) columns and L = N - R (C - 1) rows of length C (the rest have
// C - 1); slots run down the rows of column 0, then column 1, ...
__host__ __device__ inline uint32_t transposed_slot(uint32_t s, uint32_t N, uint32_t R)
{
    const uint32_t C = (N + R - 1) / R;
    const uint32_t L = N - R * (C - 1);
    uint32_t row, col;
    if (s < L * C) {
        row = s / C;
        col = s - row * C;
    } else {
        const uint32_t t = s - L * C;
        row = L + t / (C - 1);
        col = t - (row - L) * (C - 1);
    }
    return col * R + row;
}

// Payload array a of the FP32 particle record as 32-bit words: key, dx, dy,
// dz, ux, uy, uz, w.
__device__ __forceinline__ uint32_t *payload_words(const PartF32 &p, int a)
{
    switch (a) {
        case 0: return p.key;
        case 1: return reinterpret_cast<uint32_t *>(p.dx);
        case 2: return reinterpret_cast<uint32_t *>(p.dy);
        case 3: return reinterpret_cast<uint32_t *>(p.dz);
        case 4: return reinterpret_cast<uint32_t *>(p.ux);
        case 5: return reinterpret_cast<uint32_t *>(p.uy);
        case 6: return reinterpret_cast<uint32_t *>(p.uz);
        default: return reinterpret_cast<uint32_t *>(p.w);
    }
}

constexpr int kOrderThreads = 512;
// Particles of a brick that the order pass orders through shared memory (a
// 16-bit rank and a source index each; 1.5x the 4096 particles the brick
// shapes aim at); a larger brick keeps its final slots in bk.bid and writes
// them directly.  The payload reads of the staged path are served by L1,
// which gets what shared memory leaves of each SM: at 37 KB per CTA and three
// CTAs per SM (40 registers at 512 threads) the whole reorder of the 3D
// Weibel headline takes 18.7 ms; with 8192 staged particles (49 KB per CTA)
// 20.4 ms, and with 8192 at four CTAs per SM (registers capped at 32) 50 ms.
constexpr uint32_t kOrderStage = 6144;
// Payload words a thread has in flight per array in the staged path.
constexpr int kOrderBatch = 8;

// 5. order brick b by cell and transpose (see the file comment).  Dynamic
//    shared memory: one counter per cell of the brick, then the source index
//    of every final slot (the inverse permutation) and a 16-bit rank per
//    particle.  A brick of at most kOrderStage particles builds the inverse
//    permutation in shared memory, after which every payload array is
//    written slot by slot (coalesced) from its source slot, a read that
//    stays inside the few KB of old slots the brick's particles came from;
//    the arrays need no barrier between them.  A larger brick keeps its
//    final slots in bk.bid and scatters each payload word to its final slot.
__global__ void __launch_bounds__(kOrderThreads) k_brick_order(GridP g, Bricks bk, PartF32 in, PartF32 out, int has_dz)
{
    extern __shared__ uint32_t s_dyn[];
    __shared__ uint32_t s_warp[kOrderThreads / 32];
    const int b = blockIdx.x;
    const uint32_t p0 = bk.tile_start[b], N = bk.tile_start[b + 1] - p0;
    if (N == 0) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int R = bk.t[0] * bk.t[1] * bk.t[2];
    uint32_t *s_cnt = s_dyn, *s_inv = s_dyn + R;
    uint16_t *s_m = reinterpret_cast<uint16_t *>(s_inv + kOrderStage);
    const int bx = b % bk.nb[0], byz = b / bk.nb[0], by = byz % bk.nb[1], bz = byz / bk.nb[1];
    const int lo0 = 3 + bx * bk.t[0], lo1 = 3 + by * bk.t[1], lo2 = 3 + bz * bk.t[2];
    for (int c = tid; c < R; c += kOrderThreads) s_cnt[c] = 0;
    __syncthreads();
    auto local_cell = [&](uint32_t key) {
        int i, j, k;
        decode_cell(g, (int)(key & kCellMask), i, j, k);
        const int kk = g.dims == 3 ? k - lo2 : 0;
        return (i - lo0) + bk.t[0] * ((j - lo1) + bk.t[1] * kk);
    };
    const bool staged = N <= kOrderStage;
    const uint32_t *__restrict__ gkey = out.key + p0;   // keys of the brick-grouped slots
    const uint32_t *__restrict__ src = bk.src + p0;
    uint32_t *__restrict__ tmp = bk.bid + p0;
    // rank within the cell
    if (staged) {
#pragma unroll 4
        for (uint32_t q = tid; q < N; q += kOrderThreads) s_m[q] = (uint16_t)atomicAdd(&s_cnt[local_cell(gkey[q])], 1u);
    } else {
        for (uint32_t q = tid; q < N; q += kOrderThreads) tmp[q] = atomicAdd(&s_cnt[local_cell(gkey[q])], 1u);
    }
    __syncthreads();
    // exclusive scan of the cell counts: contiguous chunks per thread, then
    // the chunk totals across the block
    {
        const int per = (R + kOrderThreads - 1) / kOrderThreads;
        const int c0 = min(tid * per, R), c1 = min(c0 + per, R);
        uint32_t tot = 0;
        for (int c = c0; c < c1; c++) tot += s_cnt[c];
        uint32_t incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        uint32_t base = incl - tot;
        for (int w2 = 0; w2 < warp; w2++) base += s_warp[w2];
        for (int c = c0; c < c1; c++) {
            const uint32_t v = s_cnt[c];
            s_cnt[c] = base;
            base += v;
        }
    }
    __syncthreads();
    if (staged) {
#pragma unroll 4
        for (uint32_t q = tid; q < N; q += kOrderThreads)
            s_inv[transposed_slot(s_cnt[local_cell(gkey[q])] + s_m[q], N, (uint32_t)R)] = src[q];
        __syncthreads();   // the inverse permutation complete, every key of the brick read
#pragma unroll
        for (int a = 0; a < 8; a++) {
            if (a == 3 && !has_dz) continue;
            const uint32_t *__restrict__ sa = payload_words(in, a);
            uint32_t *__restrict__ da = payload_words(out, a) + p0;
            for (uint32_t t0 = tid; t0 < N; t0 += kOrderBatch * kOrderThreads) {
                uint32_t v[kOrderBatch];
#pragma unroll
                for (int r = 0; r < kOrderBatch; r++) {
                    const uint32_t t = t0 + r * kOrderThreads;
                    if (t < N) v[r] = ldro(sa + s_inv[t]);
                }
#pragma unroll
                for (int r = 0; r < kOrderBatch; r++) {
                    const uint32_t t = t0 + r * kOrderThreads;
                    if (t < N) da[t] = v[r];
                }
            }
        }
    } else {
        for (uint32_t q = tid; q < N; q += kOrderThreads)
            tmp[q] = transposed_slot(s_cnt[local_cell(gkey[q])] + tmp[q], N, (uint32_t)R);
        __syncthreads();   // every key of the brick read before any slot is overwritten
#pragma unroll
        for (int a = 0; a < 8; a++) {
            if (a == 3 && !has_dz) continue;
            const uint32_t *__restrict__ sa = payload_words(in, a);
            uint32_t *__restrict__ da = payload_words(out, a) + p0;
            for (uint32_t q = tid; q < N; q += kOrderThreads) da[tmp[q]] = sa[src[q]];
        }
    }
}

// 4. cursors at the brick starts, boxes = the bricks (relative to the centre).
__global__ void k_brick_prepare(GridP g, Bricks bk)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= bk.ntiles) return;
    bk.cursor[b] = bk.tile_start[b];
    const int bi[3] = {b % bk.nb[0], (b / bk.nb[0]) % bk.nb[1], b / (bk.nb[0] * bk.nb[1])};
    const int n3[3] = {g.nx, g.ny, g.nz};
    int *box = bk.box + 8 * (size_t)b;
    for (int d = 0; d < 3; d++) {
        if (d >= g.dims) {
            box[d] = box[d + 3] = 0;
            continue;
        }
        const int lo = 3 + bi[d] * bk.t[d];
        const int hi = min(lo + bk.t[d] - 1, n3[d] + 2);
        const int hc = lo + (bk.t[d] >> 1);
        box[d] = lo - hc;
        box[d + 3] = hi - hc;
    }
    box[6] = box[7] = 0;
}

__global__ void k_brick_finish(Bricks bk, Counters *cnt)
{
    const long long live = bk.tile_start[bk.ntiles];
    cnt->used = live;
    cnt->np = live;
}

static unsigned grid_for(long long n)
{
    long long b = (n + kThreads - 1) / kThreads;
    if (b > (long long)kSMs * 32) b = (long long)kSMs * 32;
    return (unsigned)(b < 1 ? 1 : b);
}

void launch_reorder_f32(const GridP &g, const PartF32 &p, const PartF32 &out, Counters *cnt, long long capacity,
                        const Bricks &bk, int *err, cudaStream_t s)
{
    cudaMemsetAsync(bk.count, 0, (size_t)(bk.ntiles + 1) * sizeof(uint32_t), s);
    cudaMemsetAsync(bk.wmax_bits, 0, sizeof(uint32_t), s);
    k_brick_count<<<grid_for(capacity), kThreads, 0, s>>>(g, bk, p, cnt, bk.bid, err);
    scan_exclusive_u32(bk.count, bk.tile_start, (size_t)bk.ntiles + 1, bk.scan_tmp, nullptr, s);
    k_brick_prepare<<<(bk.ntiles + 255) / 256, 256, 0, s>>>(g, bk);
    k_brick_slots<<<grid_for(capacity), kThreads, 0, s>>>(bk, p, out, bk.bid, cnt);
    const int R = bk.t[0] * bk.t[1] * bk.t[2];
    const size_t smem = ((size_t)R + kOrderStage) * sizeof(uint32_t) + kOrderStage * sizeof(uint16_t);
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_brick_order, cudaFuncAttributeMaxDynamicSharedMemorySize, 100 * 1024);
        attr_set = true;
    }
    k_brick_order<<<bk.ntiles, kOrderThreads, smem, s>>>(g, bk, p, out, g.dims == 3);
    k_brick_finish<<<1, 1, 0, s>>>(bk, cnt);
    count_launches(6);
}

// Brick shape for a fill of ppc particles per cell: about 4096 particles per
// brick, x first, up to 8x8x8 (3D) / 32x32 (2D) so that the boxes of the
// brick plus one cell of margin always fit the mover's shared memory; or the
// requested shape, checked against the same limit.
bool choose_bricks(const GridP &g, double ppc, const int req[3], Bricks &bk)
{
    static const int s3[][3] = {{4, 4, 4}, {8, 4, 4}, {8, 8, 4}, {8, 8, 8}};
    static const int s2[][3] = {{8, 8, 1}, {16, 8, 1}, {16, 16, 1}, {32, 16, 1}, {32, 32, 1}};
    int t[3];
    if (req && req[0] > 0) {
        for (int d = 0; d < 3; d++) t[d] = d < g.dims ? req[d] : 1;
        for (int d = 0; d < g.dims; d++)
            if (t[d] < 1) return false;
    } else {
        const double target = 4096.0 / (ppc > 0.5 ? ppc : 0.5);
        const int ns = g.dims == 3 ? 4 : 5;
        int pick = ns - 1;
        for (int q = 0; q < ns; q++) {
            const int *c = g.dims == 3 ? s3[q] : s2[q];
            if ((double)c[0] * c[1] * c[2] >= target) {
                pick = q;
                break;
            }
        }
        const int *c = g.dims == 3 ? s3[pick] : s2[pick];
        for (int d = 0; d < 3; d++) t[d] = c[d];
    }
    const int n3[3] = {g.nx, g.ny, g.nz};
    for (int d = 0; d < 3; d++) {
        bk.t[d] = d < g.dims ? (t[d] < n3[d] ? t[d] : n3[d]) : 1;
        bk.nb[d] = d < g.dims ? (n3[d] + bk.t[d] - 1) / bk.t[d] : 1;
        bk.tmagic[d] = 0;
        bk.tshift[d] = 0;
        if (bk.t[d] >= 2) div_magic((unsigned)bk.t[d], bk.tmagic[d], bk.tshift[d]);
    }
    bk.ntiles = bk.nb[0] * bk.nb[1] * bk.nb[2];
    bk.smem_floats = kBrickSmemBytes / 4;
    // the fallback box (brick + 1 cell per side) must fit, and the per-cell
    // counters of the in-brick order must fit beside its staging words
    for (int d = 0; d < g.dims; d++)
        if (bk.t[d] + 2 > kBoxAxisMax) return false;
    if ((long long)bk.t[0] * bk.t[1] * bk.t[2] * 4 > 32 * 1024) return false;
    return box_floats(g.dims, bk.t[0] + 2, bk.t[1] + 2, g.dims == 3 ? bk.t[2] + 2 : 1, box_current_words(g)) <=
           bk.smem_floats;
}

}  // namespace pic
