// particles.cu -- particle bookkeeping on the device: the periodic wrap of
// the reference layout, the stable cell-key reorder, layout conversions and
// the Weibel loader.
//
// Reference: src/comm/loadprtlout.F90:13-106 + src/comm/comm_prtl.F90:11-66
// (outliers become holes and are re-appended, shifted by the box length, in
// neighbour-list order), src/mem/mem_prtl.F90:166-301 (ReorderPrtlArr: stable
// counting sort by the cell key (k-1)*mx*my+(j-1)*mx+i, holes dropped),
// src/init/init_prtl.F90:177-221 and src/init/prob_dist.F90:13-105,223-254
// (particle loading).
//
// All three are order-preserving scans over the particle array, so they share
// one tiling: tiles of 4096 particles, 8 warps x 512 contiguous particles per
// tile, and a device-wide exclusive scan of per-tile counts.  Within a warp the
// stable rank of a particle among its peers comes from __match_any_sync /
// __ballot_sync over 32 consecutive particles, walked in index order.
#include "common.cuh"
#include "kernels.cuh"

namespace pic {

constexpr int kTile = 4096;
constexpr int kTileWarps = 8;
constexpr int kWarpItems = kTile / kTileWarps;  // 512
constexpr int kScanBlock = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanBlock * kScanItems;

size_t sort_tiles(long long capacity) { return (size_t)((capacity + kTile - 1) / kTile) + 1; }

size_t scan_tmp_len(size_t n)
{
    size_t total = 0;
    while (n > 1) {
        n = (n + kScanTile - 1) / kScanTile;
        total += n + 1;
    }
    return total + 1;
}

// ---------------------------------------------------------------------------
// Device-wide exclusive scan of uint32 (block scan + recursive block sums).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive scan of in[0..n) into out; block b writes its total to sums[b]
// (when sums != nullptr) and, for a single-block call, the grand total to
// *total.
__global__ void __launch_bounds__(kScanBlock) k_scan_block(const uint32_t *__restrict__ in, uint32_t *out, size_t n,
                                                           uint32_t *sums, uint32_t *total)
{
    __shared__ uint32_t warp_tot[kScanBlock / 32];
    const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t acc = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        v[i] = (base + i < n) ? in[base + i] : 0u;
        acc += v[i];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t incl = warp_incl_scan(acc);
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t t = warp_tot[lane];
        t = warp_incl_scan(t);
        warp_tot[lane] = t;
    }
    __syncthreads();
    uint32_t run = (incl - acc) + (warp > 0 ? warp_tot[warp - 1] : 0u);
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
    if (threadIdx.x == kScanBlock - 1) {
        if (sums) sums[blockIdx.x] = run;
        if (total && gridDim.x == 1) *total = run;
    }
}

__global__ void k_scan_add(uint32_t *out, size_t n, const uint32_t *__restrict__ offs)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += offs[i / kScanTile];
}

void scan_exclusive_u32(const uint32_t *in, uint32_t *out, size_t n, uint32_t *tmp, uint32_t *total, cudaStream_t s)
{
    const size_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb <= 1) {
        k_scan_block<<<1, kScanBlock, 0, s>>>(in, out, n, nullptr, total);
        count_launches(1);
        return;
    }
    uint32_t *sums = tmp;
    uint32_t *rest = tmp + nb + 1;
    k_scan_block<<<(unsigned)nb, kScanBlock, 0, s>>>(in, out, n, sums, nullptr);
    count_launches(1);
    scan_exclusive_u32(sums, sums, nb, rest, total, s);
    k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, n, sums);
    count_launches(1);
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort of (key, index) pairs, up to 8 bits per pass.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t lanemask_lt()
{
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__global__ void __launch_bounds__(256) k_radix_hist(const uint32_t *__restrict__ keys, const long long *__restrict__ used,
                                                    int shift, uint32_t mask, uint32_t *hist, size_t ntiles)
{
    __shared__ uint32_t cnt[256];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const long long n = *used;
    const long long base = (long long)blockIdx.x * kTile;
    for (int r = 0; r < kTile / 256; r++) {
        const long long i = base + r * 256 + threadIdx.x;
        if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & mask], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

// first_pass: the index payload is the particle slot itself.
__global__ void __launch_bounds__(256) k_radix_scatter(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ iin,
                                                       uint32_t *kout, uint32_t *iout, const long long *__restrict__ used,
                                                       int shift, uint32_t mask, const uint32_t *__restrict__ offs,
                                                       size_t ntiles, int first_pass)
{
    __shared__ uint32_t wh[kTileWarps][256];
    for (int t = threadIdx.x; t < kTileWarps * 256; t += 256) (&wh[0][0])[t] = 0;
    __syncthreads();
    const long long n = *used;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long wbase = (long long)blockIdx.x * kTile + (long long)warp * kWarpItems;
    const uint32_t lt = lanemask_lt();
    // phase A: per-warp digit counts
    for (int r = 0; r < kWarpItems / 32; r++) {
        const long long i = wbase + r * 32 + lane;
        const bool ok = i < n;
        const uint32_t d = ok ? (kin[i] >> shift) & mask : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (ok && (peers & lt) == 0) wh[warp][d] += __popc(peers);
    }
    __syncthreads();
    // phase B: per-digit exclusive prefix over warps, based at the tile offset
    {
        const int d = threadIdx.x;
        uint32_t run = offs[(size_t)d * ntiles + blockIdx.x];
        for (int w = 0; w < kTileWarps; w++) {
            const uint32_t t = wh[w][d];
            wh[w][d] = run;
            run += t;
        }
    }
    __syncthreads();
    // phase C: stable scatter
    for (int r = 0; r < kWarpItems / 32; r++) {
        const long long i = wbase + r * 32 + lane;
        const bool ok = i < n;
        const uint32_t k = ok ? kin[i] : 0u;
        const uint32_t d = ok ? (k >> shift) & mask : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        uint32_t pos = 0;
        if (ok) pos = wh[warp][d] + __popc(peers & lt);
        __syncwarp();
        if (ok && (peers & lt) == 0) wh[warp][d] += __popc(peers);
        __syncwarp();
        if (ok) {
            kout[pos] = k;
            iout[pos] = first_pass ? (uint32_t)i : iin[i];
        }
    }
}

// Sorts sc.key[0]/sc.idx[0] (keys valid in [0,*used)); the result ends in
// sc.key[r]/sc.idx[r] with r returned.  Keys must be < 2^nbits.
static int radix_sort(SortScratch &sc, const long long *used, int nbits, size_t ntiles, cudaStream_t s)
{
    const int passes = (nbits + 7) / 8;
    const int bits = (nbits + passes - 1) / passes;
    const uint32_t mask = (1u << bits) - 1u;
    int cur = 0;
    for (int ps = 0; ps < passes; ps++) {
        const int shift = ps * bits;
        k_radix_hist<<<(unsigned)ntiles, 256, 0, s>>>(sc.key[cur], used, shift, mask, sc.hist, ntiles);
        count_launches(1);
        scan_exclusive_u32(sc.hist, sc.hist, 256 * ntiles, sc.scan_tmp, nullptr, s);
        k_radix_scatter<<<(unsigned)ntiles, 256, 0, s>>>(sc.key[cur], sc.idx[cur], sc.key[cur ^ 1], sc.idx[cur ^ 1], used,
                                                         shift, mask, sc.hist, ntiles, ps == 0);
        count_launches(1);
        cur ^= 1;
    }
    return cur;
}

int radix_sort_keys(SortScratch &sc, const long long *used, int nbits, cudaStream_t s)
{
    return radix_sort(sc, used, nbits, sc.ntiles, s);
}

static int key_bits(long long ncell)
{
    int b = 1;
    while ((1ll << b) <= ncell) b++;
    return b;
}

int sort_key_bits(long long ncell) { return key_bits(ncell); }

// ---------------------------------------------------------------------------
// ReorderPrtlArr (mem_prtl.F90:166-301)
// ---------------------------------------------------------------------------
__global__ void k_keys_f64(GridP g, PartF64 p, const long long *__restrict__ used, uint32_t *keys, long long *np,
                           int *err, unsigned long long *qmax)
{
    const long long n = *used;
    long long live = 0;
    unsigned long long qm = 0;   // bits of max |q| of this thread's live particles (when qmax is given)
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        uint32_t key = (uint32_t)g.ncell;  // holes sort last (mem_prtl.F90:179 skips them)
        if (p.flv[i] != 0) {
            const int ci = (int)floor(p.x[i]), cj = (int)floor(p.y[i]);
            const int ck = g.dims == 3 ? (int)floor(p.z[i]) : 1;
            if (ci >= 1 && ci <= g.mx && cj >= 1 && cj <= g.my && ck >= 1 && ck <= g.mz) {
                key = (uint32_t)cidx(g, ci, cj, ck);
                live++;
                if (qmax) qm = max(qm, (unsigned long long)__double_as_longlong(fabs(p.q[i])));
            } else {
                raise_error(err, PIC_DEVERR_RANGE);
            }
        }
        keys[i] = key;
    }
    // block-reduce the live count
    __shared__ long long red[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) live += __shfl_down_sync(0xffffffffu, live, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = live;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int w = 0; w < kThreads / 32; w++) t += red[w];
        atomicAdd((unsigned long long *)np, (unsigned long long)t);
    }
    if (qmax) {
        for (int o = 16; o > 0; o >>= 1) qm = max(qm, __shfl_down_sync(0xffffffffu, qm, o));
        if ((threadIdx.x & 31) == 0 && qm) atomicMax(qmax, qm);
    }
}

__global__ void k_gather_f64(PartF64 in, PartF64 out, const uint32_t *__restrict__ idx, const long long *__restrict__ used)
{
    const long long n = *used;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint32_t s = idx[i];
        out.q[i] = in.q[s];
        out.x[i] = in.x[s];
        out.y[i] = in.y[s];
        out.z[i] = in.z[s];
        out.u[i] = in.u[s];
        out.v[i] = in.v[s];
        out.w[i] = in.w[s];
        out.flv[i] = in.flv[s];
    }
}

__global__ void k_set_used_np(Counters *cnt) { cnt->used = cnt->np; }

static unsigned stream_grid(long long capacity)
{
    long long b = (capacity + kThreads - 1) / kThreads;
    if (b > (long long)kSMs * 32) b = (long long)kSMs * 32;
    return (unsigned)(b < 1 ? 1 : b);
}

void launch_reorder_f64(const GridP &g, const PartF64 &p, const PartF64 &out, Counters *cnt, SortScratch &sc,
                        long long capacity, int *err, cudaStream_t s, Tiles64 *tiles)
{
    cudaMemsetAsync(&cnt->np, 0, sizeof(long long), s);
    if (tiles) cudaMemsetAsync(tiles->qmax, 0, sizeof(unsigned long long), s);
    k_keys_f64<<<stream_grid(capacity), kThreads, 0, s>>>(g, p, &cnt->used, sc.key[0], &cnt->np, err,
                                                          tiles ? tiles->qmax : nullptr);
    count_launches(1);
    const size_t ntiles = sort_tiles(capacity);
    const int r = radix_sort(sc, &cnt->used, key_bits(g.ncell), ntiles, s);
    k_gather_f64<<<stream_grid(capacity), kThreads, 0, s>>>(p, out, sc.idx[r], &cnt->used);
    count_launches(1);
    k_set_used_np<<<1, 1, 0, s>>>(cnt);
    count_launches(1);
    // the tiles of the FP64 tiled mover: slot ranges from the sorted keys
    if (tiles) launch_tiles64_after_reorder(g, sc.key[r], cnt, *tiles, s);
}

// ---------------------------------------------------------------------------
// Periodic wrap of the reference layout: LoadPrtlOutliers + AppendParticles
// ---------------------------------------------------------------------------

// Face (1..6) through which LoadPrtlOutliers (loadprtlout.F90:29-96) sends a
// particle, 0 if it stays.  The first matching test in x, y, z order wins:
// a sent particle is holed at x=y=3.8 before the later tests look at it.
template <int DIMS>
__device__ __forceinline__ int outlier_face(const GridP &g, double x, double y, double z)
{
    const double xmin = g.xmin, xmax = g.xmax, ymin = g.ymin, ymax = g.ymax, zmin = g.zmin, zmax = g.zmax;
    if (x < xmin) {
        if ((y <= (ymax + xmin) - x) && (y >= (ymin - xmin) + x))
            if (DIMS == 2 || ((z <= (zmax + xmin) - x) && (z >= (zmin - xmin) + x))) return 1;
    } else if (x > xmax) {
        if ((y <= (ymax - xmax) + x) && (y >= (ymin + xmax) - x))
            if (DIMS == 2 || ((z <= (zmax - xmax) + x) && (z >= (zmin + xmax) - x))) return 2;
    }
    if (y < ymin) {
        if ((y < (ymin - xmin) + x) && (y < (ymin + xmax) - x))
            if (DIMS == 2 || ((z >= (zmin - ymin) + y) && (z <= (zmax + ymin) - y))) return 3;
    } else if (y > ymax) {
        if ((y > (ymax + xmin) - x) && (y > (ymax - xmax) + x))
            if (DIMS == 2 || ((z >= (zmin + ymax) - y) && (z <= (zmax - ymax) + y))) return 4;
    }
    if (DIMS == 3) {
        if (z < zmin) {
            if ((z < (zmin - xmin) + x) && (z < (zmin + xmax) - x))
                if ((z < (zmin - ymin) + y) && (z < (zmin + ymax) - y)) return 5;
        } else if (z > zmax) {
            if ((z > (zmax + xmin) - x) && (z > (zmax - xmax) + x))
                if ((z > (zmax + ymin) - y) && (z > (zmax - ymax) + y)) return 6;
        }
    }
    return 0;
}

// AppendParticles walks recv(1..6), which hold what left through faces
// 2,1,4,3,6,5: slot of a face in that order, -1 for none.  Faces whose
// neighbour is MPI_PROC_NULL (the r faces of a cylinder) append nothing.
__device__ __forceinline__ int append_slot(const GridP &g, int face)
{
    if (face == 0 || (face <= 2 && ((g.closed_x >> (face - 1)) & 1))) return -1;
    return (face - 1) ^ 1;
}

// The exchange in two passes over the particles of blocks of kTile slots.
// The count pass reads each particle's flavour and position once, with
// 16-byte loads of four consecutive slots per thread, and writes the face it
// leaves through (0: stays or a hole, 1..6: outlier_face) as one byte per
// slot, four to a word; it counts the leavers of each append slot per block.
// After the scan of those counts, the scatter pass reads only the face words
// and, for the few particles that leave, their state.  The append order is
// slot order within each face (LoadPrtlOutliers walks the array in order).
__device__ __forceinline__ void load_quad_f64(const double *a, long long i, long long n, double v[4])
{
    if (i + 4 <= n) {
        const double2 lo = *reinterpret_cast<const double2 *>(a + i);
        const double2 hi = *reinterpret_cast<const double2 *>(a + i + 2);
        v[0] = lo.x; v[1] = lo.y; v[2] = hi.x; v[3] = hi.y;
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) v[k] = i + k < n ? a[i + k] : 0.0;
    }
}

template <int DIMS>
__global__ void __launch_bounds__(256) k_exch_count(GridP g, PartF64 p, const long long *__restrict__ used,
                                                    uint32_t *counts, uint32_t *faces, size_t ntiles)
{
    __shared__ uint32_t c[6];
    if (threadIdx.x < 6) c[threadIdx.x] = 0;
    __syncthreads();
    const long long n = *used;
    const long long qbase = (long long)blockIdx.x * (kTile / 4);
    // a round's loads (flavours as one int4, each coordinate as two double2)
    // are in flight together; unrolling the rounds makes the compiler spill
#pragma unroll 1
    for (int r = 0; r < kTile / 1024; r++) {
        const long long q = qbase + r * 256 + threadIdx.x;   // four slots 4q .. 4q + 3
        const long long i = 4 * q;
        if (i >= n) continue;
        int f4[4];
        if (i + 4 <= n) {
            const int4 fl = *reinterpret_cast<const int4 *>(p.flv + i);
            f4[0] = fl.x; f4[1] = fl.y; f4[2] = fl.z; f4[3] = fl.w;
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) f4[k] = i + k < n ? p.flv[i + k] : 0;
        }
        double x4[4], y4[4], z4[4] = {0.0, 0.0, 0.0, 0.0};
        load_quad_f64(p.x, i, n, x4);
        load_quad_f64(p.y, i, n, y4);
        if (DIMS == 3) load_quad_f64(p.z, i, n, z4);
        uint32_t word = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int face = f4[k] != 0 ? outlier_face<DIMS>(g, x4[k], y4[k], z4[k]) : 0;
            word |= (uint32_t)face << (8 * k);
            const int sl = append_slot(g, face);
            if (sl >= 0) atomicAdd(&c[sl], 1u);
        }
        faces[q] = word;
    }
    __syncthreads();
    if (threadIdx.x < 6) counts[(size_t)threadIdx.x * ntiles + blockIdx.x] = c[threadIdx.x];
}

// RemovePrtl, loadprtlout.F90:164-181
template <int DIMS>
__device__ __forceinline__ void remove_prtl(const PartF64 &p, long long i)
{
    p.q[i] = 0.0;
    p.flv[i] = 0;
    p.u[i] = 0.0;
    p.v[i] = 0.0;
    p.w[i] = 0.0;
    p.x[i] = 3.8;
    p.y[i] = 3.8;
    p.z[i] = DIMS == 3 ? 3.8 : 1.5;
}

// Slab form (g.x_external): what leaves through the x faces goes to the
// neighbouring slabs instead: slots 0 and 1 (faces 2 and 1) fill the front of
// the scan order, so their particles go to `out` at their scan position
// (right-bound first, then left-bound; 8 doubles each: q, x, y, z, u, v, w,
// flv, x already in the receiver's coordinates), and the y / z leavers are
// appended after the local particles from scan position offs[2 ntiles] on.
template <int DIMS>
__global__ void __launch_bounds__(256) k_exch_scatter(GridP g, PartF64 p, Counters *cnt, const uint32_t *__restrict__ offs,
                                                      const uint32_t *__restrict__ total,
                                                      const uint32_t *__restrict__ faces, size_t ntiles,
                                                      long long capacity, int *err, double *out, long long out_cap)
{
    __shared__ uint32_t wh[kTileWarps][6];
    const long long n = cnt->used;
    const uint32_t sent = g.x_external ? offs[2 * ntiles] : 0u;   // particles leaving through the x faces
    if ((long long)(*total - sent) + n > capacity || (long long)sent > out_cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_error(err, PIC_DEVERR_OVERFLOW);
        return;
    }
    if (threadIdx.x < kTileWarps * 6) (&wh[0][0])[threadIdx.x] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // warp w takes slots [w kWarpItems, (w + 1) kWarpItems) of the block, 128
    // per round, four consecutive slots per lane
    const long long wq = (long long)blockIdx.x * (kTile / 4) + (long long)warp * (kWarpItems / 4);
    constexpr int kRounds = kWarpItems / 128;
    uint32_t words[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
        const long long q = wq + r * 32 + lane;
        words[r] = 4 * q < n ? faces[q] : 0u;
    }
    // the warp's leavers per append slot
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
        if (__ballot_sync(0xffffffffu, words[r] != 0u) == 0u) continue;   // uniform over the warp
        uint32_t c6[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int sl = append_slot(g, (int)((words[r] >> (8 * k)) & 0xffu));
#pragma unroll
            for (int f = 0; f < 6; f++) c6[f] += sl == f;
        }
#pragma unroll
        for (int f = 0; f < 6; f++) {
            const uint32_t t = __reduce_add_sync(0xffffffffu, c6[f]);
            if (lane == 0) wh[warp][f] += t;
        }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int f = threadIdx.x;
        uint32_t run = offs[(size_t)f * ntiles + blockIdx.x];
        for (int w = 0; w < kTileWarps; w++) {
            const uint32_t t = wh[w][f];
            wh[w][f] = run;
            run += t;
        }
    }
    __syncthreads();
    const double len[3] = {g.xlen, g.ylen, g.zlen};
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int r = 0; r < kRounds; r++) {
        const uint32_t word = words[r];
        if (__ballot_sync(0xffffffffu, word != 0u) == 0u) continue;   // uniform over the warp
        int sl[4];
#pragma unroll
        for (int k = 0; k < 4; k++) sl[k] = append_slot(g, (int)((word >> (8 * k)) & 0xffu));
        // position of each of the lane's leavers: the warp's base for its
        // slot, the same slot's leavers of the lower lanes, then those of the
        // lane's lower slots
        uint32_t pos[4] = {0, 0, 0, 0};
#pragma unroll
        for (int f = 0; f < 6; f++) {
            uint32_t below = 0, all = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint32_t m = __ballot_sync(0xffffffffu, sl[k] == f);
                below += __popc(m & lt);
                all += __popc(m);
            }
            uint32_t run = wh[warp][f] + below;
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (sl[k] == f) pos[k] = run++;
            __syncwarp();
            if (lane == 0) wh[warp][f] += all;
            __syncwarp();
        }
        const long long i0 = 4 * (wq + r * 32 + lane);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int face = (int)((word >> (8 * k)) & 0xffu);
            if (face == 0) continue;
            const long long i = i0 + k;
            if (sl[k] >= 0) {
                double pos3[3] = {p.x[i], p.y[i], p.z[i]};
                const int axis = (face - 1) >> 1;
                // CopyTransferPrtl subtracts the send list's shift, InsertPrtls adds
                // the receiving list's (subdomains.F90:720-740): low faces +len, high -len.
                if (face & 1) pos3[axis] = (pos3[axis] - 0.0) + len[axis];
                else pos3[axis] = (pos3[axis] - len[axis]) + 0.0;
                if (g.x_external && sl[k] <= 1) {
                    double *o = out + 8 * (size_t)pos[k];
                    o[0] = p.q[i];
                    o[1] = pos3[0];
                    o[2] = pos3[1];
                    o[3] = pos3[2];
                    o[4] = p.u[i];
                    o[5] = p.v[i];
                    o[6] = p.w[i];
                    o[7] = (double)p.flv[i];
                } else {
                    const long long d = n + (pos[k] - sent);
                    p.q[d] = p.q[i];
                    p.x[d] = pos3[0];
                    p.y[d] = pos3[1];
                    p.z[d] = pos3[2];
                    p.u[d] = p.u[i];
                    p.v[d] = p.v[i];
                    p.w[d] = p.w[i];
                    p.flv[d] = p.flv[i];
                }
            }
            // a leaver, or sent to MPI_PROC_NULL: RemovePrtl (without a
            // matching append in the second case)
            remove_prtl<DIMS>(p, i);
        }
    }
}

// The scatter stops before moving anything when the appended particles would
// pass the capacity or the x leavers the outbox; the count then stays as it
// was (and the overflow bit is set), so no stale slot becomes live.
__global__ void k_exch_finish(Counters *cnt, const uint32_t *__restrict__ total, const uint32_t *__restrict__ sent,
                              long long capacity, long long out_cap)
{
    const long long s = sent ? (long long)*sent : 0;
    const long long t = (long long)*total - s;
    cnt->append = t;
    if (cnt->used + t <= capacity && s <= out_cap) cnt->used += t;
}

void launch_exchange_f64(const GridP &g, PartF64 &p, Counters *cnt, SortScratch &sc, long long capacity, int *err,
                         cudaStream_t s, double *out, long long out_cap, uint32_t *sent_counts)
{
    const size_t ntiles = sort_tiles(capacity);
    uint32_t *counts = sc.hist;  // 6 * ntiles <= 256 * ntiles
    uint32_t *total = sc.scan_tmp + sc.scan_tmp_len - 1;
    // the face words: one per four slots below `used` (<= capacity / 4 + 1
    // words) in the radix-sort key buffer, which holds capacity words and is
    // free between reorders
    uint32_t *faces = sc.key[1];
    if (g.dims == 3) k_exch_count<3><<<(unsigned)ntiles, 256, 0, s>>>(g, p, &cnt->used, counts, faces, ntiles);
    else k_exch_count<2><<<(unsigned)ntiles, 256, 0, s>>>(g, p, &cnt->used, counts, faces, ntiles);
    scan_exclusive_u32(counts, counts, 6 * ntiles, sc.scan_tmp, total, s);
    if (g.dims == 3)
        k_exch_scatter<3><<<(unsigned)ntiles, 256, 0, s>>>(g, p, cnt, counts, total, faces, ntiles, capacity, err, out,
                                                          out_cap);
    else
        k_exch_scatter<2><<<(unsigned)ntiles, 256, 0, s>>>(g, p, cnt, counts, total, faces, ntiles, capacity, err, out,
                                                          out_cap);
    k_exch_finish<<<1, 1, 0, s>>>(cnt, total, g.x_external ? counts + 2 * ntiles : nullptr, capacity, out_cap);
    if (g.x_external && sent_counts) {
        // right-bound (face 2, slot 0) and right + left-bound particle counts
        cudaMemcpyAsync(sent_counts, counts + ntiles, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(sent_counts + 1, counts + 2 * ntiles, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    }
    count_launches(1);
    count_launches(2);
}

// ---------------------------------------------------------------------------
// Layout conversions
// ---------------------------------------------------------------------------
__global__ void k_f64_to_f32(GridP g, PartF64 in, PartF32 out, long long n, int *err)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int flv = in.flv[i];
        const double x = in.x[i], y = in.y[i], z = in.z[i];
        const double fx = floor(x), fy = floor(y), fz = g.dims == 3 ? floor(z) : 1.0;
        int ci = (int)fx, cj = (int)fy, ck = (int)fz;
        uint32_t key = 0;
        if (flv != 0) {
            if (!(x >= 2.0 && x < (double)(g.mx - 1) && y >= 2.0 && y < (double)(g.my - 1) &&
                  (g.dims == 2 || (z >= 2.0 && z < (double)(g.mz - 1)))) || flv > 15 || flv < 0) {
                raise_error(err, PIC_DEVERR_RANGE);
            } else {
                ci = wrap_index(ci, g.mx);
                cj = wrap_index(cj, g.my);
                if (g.dims == 3) ck = wrap_index(ck, g.mz);
                key = ((uint32_t)flv << kFlvShift) | (uint32_t)cidx(g, ci, cj, ck);
            }
        }
        out.key[i] = key;
        out.dx[i] = (float)(x - fx);
        out.dy[i] = (float)(y - fy);
        if (g.dims == 3) out.dz[i] = (float)(z - fz);
        out.ux[i] = (float)in.u[i];
        out.uy[i] = (float)in.v[i];
        out.uz[i] = (float)in.w[i];
        out.w[i] = (float)in.q[i];
    }
}

__global__ void k_f32_to_f64(GridP g, PartF32 in, PartF64 out, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint32_t key = in.key[i];
        const int flv = (int)(key >> kFlvShift);
        const int cell = (int)(key & kCellMask);
        const int ci = cell % g.mx + 1, jk = cell / g.mx, cj = jk % g.my + 1, ck = jk / g.my + 1;
        out.flv[i] = flv;
        out.q[i] = flv ? (double)in.w[i] : 0.0;
        out.x[i] = flv ? (double)ci + (double)in.dx[i] : 3.8;
        out.y[i] = flv ? (double)cj + (double)in.dy[i] : 3.8;
        out.z[i] = g.dims == 3 ? (flv ? (double)ck + (double)in.dz[i] : 3.8) : 1.5;
        out.u[i] = flv ? (double)in.ux[i] : 0.0;
        out.v[i] = flv ? (double)in.uy[i] : 0.0;
        out.w[i] = flv ? (double)in.uz[i] : 0.0;
    }
}

void launch_f64_to_f32(const GridP &g, const PartF64 &in, const PartF32 &out, long long n, int *err, cudaStream_t s)
{
    if (n > 0) k_f64_to_f32<<<stream_grid(n), kThreads, 0, s>>>(g, in, out, n, err);
    count_launches(n > 0 ? 1 : 0);
}

void launch_f32_to_f64(const GridP &g, const PartF32 &in, const PartF64 &out, long long n, cudaStream_t s)
{
    if (n > 0) k_f32_to_f64<<<stream_grid(n), kThreads, 0, s>>>(g, in, out, n);
    count_launches(n > 0 ? 1 : 0);
}

// Field arrays between the FP64 host layout and the FP32 device form.
__global__ void k_array_f64_to_f32(const double *__restrict__ in, float *__restrict__ out, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

__global__ void k_array_f32_to_f64(const float *__restrict__ in, double *__restrict__ out, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

void launch_array_f64_to_f32(const double *in, float *out, long long n, cudaStream_t s)
{
    if (n > 0) k_array_f64_to_f32<<<stream_grid(n), kThreads, 0, s>>>(in, out, n);
    count_launches(n > 0 ? 1 : 0);
}

void launch_array_f32_to_f64(const float *in, double *out, long long n, cudaStream_t s)
{
    if (n > 0) k_array_f32_to_f64<<<stream_grid(n), kThreads, 0, s>>>(in, out, n);
    count_launches(n > 0 ? 1 : 0);
}

// ---------------------------------------------------------------------------
// Weibel loader (setup_weibel.F90:17-61 via InitPrtl, init_prtl.F90:177-221)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                                              uint32_t k1, uint32_t out[4])
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

__device__ __forceinline__ double u01(uint32_t hi, uint32_t lo)
{
    const unsigned long long b = (((unsigned long long)hi << 32) | lo) >> 11;
    return (double)b * (1.0 / 9007199254740992.0);
}

struct TrialDraw {
    double r1, r2, r3, racpt;
};

__device__ __forceinline__ TrialDraw draw_trial(uint32_t seed, uint32_t n, uint32_t call)
{
    uint32_t r[4];
    TrialDraw t;
    philox4x32_10(n, call, 0, 0, seed, 0x50494354u, r);
    t.r1 = u01(r[0], r[1]);
    t.r2 = u01(r[2], r[3]);
    philox4x32_10(n, call, 1, 0, seed, 0x50494354u, r);
    t.r3 = u01(r[0], r[1]);
    t.racpt = u01(r[2], r[3]);
    return t;
}

__global__ void __launch_bounds__(256) k_weibel_count(WeibelParams w, uint32_t *counts, long long ntrials_total)
{
    __shared__ uint32_t c;
    if (threadIdx.x == 0) c = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * kTile;
    uint32_t mine = 0;
    for (int r = 0; r < kTile / 256; r++) {
        const long long t = base + r * 256 + threadIdx.x;
        if (t < ntrials_total) {
            const uint32_t call = (uint32_t)(t / w.ntrial), n = (uint32_t)(t % w.ntrial);
            const TrialDraw d = draw_trial(w.seed, n, call);
            if (d.racpt <= w.density) mine++;
        }
    }
    atomicAdd(&c, mine);
    __syncthreads();
    if (threadIdx.x == 0) counts[blockIdx.x] = c;
}

// prob_dist.F90:85-105 (1-based result)
__device__ int bsearch_table(int n, const double *A, double val)
{
    int imin = 1, imax = n, imid = (imin + imax) / 2;
    bool search = true;
    while (search) {
        const int prev = imid;
        if (A[imid - 1] >= val) imax = imid;
        if (A[imid - 1] <= val) imin = imid;
        imid = (imin + imax) / 2;
        if (imin + 1 >= imax) search = false;
        if (imid == prev) search = false;
    }
    return imin;
}

__device__ void maxwell_momentum(const double *X, const double *P, int nt, double temp, double rmb, double riso2,
                                 double riso3, double drift_x, double drift_y, double drift_z, double &u, double &v,
                                 double &w)
{
    // GetVelGamma_MaxBolt (prob_dist.F90:13-30) + InvPDF (:72-83)
    const int idx = bsearch_table(nt, P, rmb);
    double beta = (P[idx] == P[idx - 1]) ? X[idx - 1]
                                        : X[idx - 1] + (X[idx] - X[idx - 1]) * ((rmb - P[idx - 1]) / (P[idx] - P[idx - 1]));
    beta = sqrt(beta * temp);
    if (beta >= 1.0) beta = 0.0;
    const double gamma = 1.0 / sqrt((1.0 + beta) * (1.0 - beta));
    // iso3vel (:56-70)
    const double ct = 2.0 * riso2 - 1.0;
    const double st = sqrt(1.0 - ct * ct);
    const double phi = (2.0 * 3.14159265358979323846264) * riso3;
    u = (gamma * beta) * ct;
    v = ((gamma * beta) * st) * cos(phi);
    w = ((gamma * beta) * st) * sin(phi);
    // AddDriftVel (:223-254)
    const double vx = drift_x, vy = drift_y, vz = drift_z;
    const double dr = sqrt((vx * vx + vy * vy) + vz * vz);
    double db, dg;
    if (fabs(dr) < 1.0) {
        db = dr;
        dg = 1.0 / sqrt((1.0 - dr) * (1.0 + dr));
    } else {
        dg = fabs(dr);
        db = sqrt((dr - 1.0) * (dr + 1.0)) / dr;
    }
    double d0 = vx, d1 = vy, d2 = vz;
    const double mag = sqrt((d0 * d0 + d1 * d1) + d2 * d2);
    if (mag == 0) {
        d0 = d1 = d2 = 0;
    } else {
        d0 = d0 / mag;
        d1 = d1 / mag;
        d2 = d2 / mag;
    }
    const double gm = sqrt(((1.0 + u * u) + v * v) + w * w);
    const double projn = (u * d0 + v * d1) + w * d2;
    u = (u + ((dg - 1.0) * projn) * d0) + ((dg * db) * gm) * d0;
    v = (v + ((dg - 1.0) * projn) * d1) + ((dg * db) * gm) * d1;
    w = (w + ((dg - 1.0) * projn) * d2) + ((dg * db) * gm) * d2;
}

__global__ void __launch_bounds__(256) k_weibel_fill(GridP g, WeibelParams w, const double *__restrict__ X,
                                                     const double *__restrict__ P, int nt, PartF64 p64, PartF32 p32,
                                                     int use32, const uint32_t *__restrict__ offs,
                                                     const uint32_t *__restrict__ total, long long ntrials_total,
                                                     long long capacity, int *err)
{
    __shared__ uint32_t wh[kTileWarps];
    if (2ll * (long long)*total > capacity) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_error(err, PIC_DEVERR_OVERFLOW);
        return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long wbase = (long long)blockIdx.x * kTile + (long long)warp * kWarpItems;
    const uint32_t lt = lanemask_lt();
    uint32_t mine = 0;
    for (int r = 0; r < kWarpItems / 32; r++) {
        const long long t = wbase + r * 32 + lane;
        bool acc = false;
        if (t < ntrials_total) {
            const TrialDraw d = draw_trial(w.seed, (uint32_t)(t % w.ntrial), (uint32_t)(t / w.ntrial));
            acc = d.racpt <= w.density;
        }
        mine += __popc(__ballot_sync(0xffffffffu, acc));
    }
    if (lane == 0) wh[warp] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = offs[blockIdx.x];
        for (int k = 0; k < kTileWarps; k++) {
            const uint32_t t = wh[k];
            wh[k] = run;
            run += t;
        }
    }
    __syncthreads();
    uint32_t run = wh[warp];
    const double zmin = g.dims == 3 ? 3.0 : 1.0;
    const double x2 = g.nx, y2 = g.ny, z2 = g.dims == 3 ? g.nz : 1;
    for (int r = 0; r < kWarpItems / 32; r++) {
        const long long t = wbase + r * 32 + lane;
        bool acc = false;
        TrialDraw d;
        uint32_t call = 0, n = 0;
        if (t < ntrials_total) {
            call = (uint32_t)(t / w.ntrial);
            n = (uint32_t)(t % w.ntrial);
            d = draw_trial(w.seed, n, call);
            acc = d.racpt <= w.density;
        }
        const uint32_t b = __ballot_sync(0xffffffffu, acc);
        if (acc) {
            const long long slot = 2ll * (long long)(run + __popc(b & lt));
            const double xg = 0.0 + d.r1 * (x2 - 0.0), yg = 0.0 + d.r2 * (y2 - 0.0), zg = 0.0 + d.r3 * (z2 - 0.0);
            const double xl = (xg - 0.0) + 3.0, yl = (yg - 0.0) + 3.0, zl = (zg - 0.0) + zmin;
            for (int sp = 0; sp < 2; sp++) {
                uint32_t rr[4];
                philox4x32_10(n, call, 2 + sp, 0, w.seed, 0x50494354u, rr);
                const double rmb = u01(rr[0], rr[1]), riso2 = u01(rr[2], rr[3]);
                philox4x32_10(n, call, 4 + sp, 0, w.seed, 0x50494354u, rr);
                const double riso3 = u01(rr[0], rr[1]);
                const double sgn = ((call == 0) == (sp == 0)) ? -1.0 : 1.0;
                double u, v, ww;
                maxwell_momentum(X, P, nt, w.temp[sp], rmb, riso2, riso3, sgn * w.drift, 0.0, 0.0, u, v, ww);
                const long long o = slot + sp;
                const double q = (1.0 * (sp == 0 ? 1.0 : -1.0)) * 1.0;
                if (!use32) {
                    if (w.sgn_out) w.sgn_out[o] = sgn;
                    p64.x[o] = xl;
                    p64.y[o] = yl;
                    p64.z[o] = zl;
                    p64.u[o] = u;
                    p64.v[o] = v;
                    p64.w[o] = ww;
                    p64.q[o] = q;
                    p64.flv[o] = sp + 1;
                } else {
                    const double fx = floor(xl), fy = floor(yl), fz = g.dims == 3 ? floor(zl) : 1.0;
                    const uint32_t cell = (uint32_t)cidx(g, (int)fx, (int)fy, (int)fz);
                    p32.key[o] = ((uint32_t)(sp + 1) << kFlvShift) | cell;
                    p32.dx[o] = (float)(xl - fx);
                    p32.dy[o] = (float)(yl - fy);
                    if (g.dims == 3) p32.dz[o] = (float)(zl - fz);
                    p32.ux[o] = (float)u;
                    p32.uy[o] = (float)v;
                    p32.uz[o] = (float)ww;
                    p32.w[o] = (float)q;
                }
            }
        }
        run += __popc(b);
    }
}

__global__ void k_weibel_finish(Counters *cnt, const uint32_t *__restrict__ total, long long capacity)
{
    const long long n = 2ll * (long long)*total;
    if (n <= capacity) {
        cnt->used = n;
        cnt->np = n;
    }
}

int launch_weibel(const GridP &g, const WeibelParams &w, const double *X, const double *P, int nt, const PartF64 *p64,
                  const PartF32 *p32, Counters *cnt, SortScratch &sc, long long capacity, int *err, cudaStream_t s)
{
    const long long ntot = 2 * w.ntrial;
    const size_t ntiles = (size_t)((ntot + kTile - 1) / kTile);
    // counts/offsets live in the sort histogram buffer (256 * sort tiles)
    if (ntiles > 256 * sc.ntiles) return PIC_ERR_OVERFLOW;
    uint32_t *total = sc.scan_tmp + sc.scan_tmp_len - 1;
    k_weibel_count<<<(unsigned)ntiles, 256, 0, s>>>(w, sc.hist, ntot);
    count_launches(1);
    scan_exclusive_u32(sc.hist, sc.hist, ntiles, sc.scan_tmp, total, s);
    PartF64 a = p64 ? *p64 : PartF64{};
    PartF32 b = p32 ? *p32 : PartF32{};
    k_weibel_fill<<<(unsigned)ntiles, 256, 0, s>>>(g, w, X, P, nt, a, b, p32 != nullptr, sc.hist, total, ntot, capacity, err);
    count_launches(1);
    k_weibel_finish<<<1, 1, 0, s>>>(cnt, total, capacity);
    count_launches(1);
    return PIC_OK;
}

// ---------------------------------------------------------------------------
// Particle injection at an 'iflw' face: InjectNewPrtl (bc_inflow.F90:134-189)
// with GetNewPrtlPos (:237-256) and InsertPrtl_PSP (init_prtl.F90:138-169)
// for a uniform density and drift.  Trial n of call k draws from Philox
// (counter n, k, stream; key seed, "INJC"): streams 0, 1 the position and the
// acceptance, 2 + 2 sp and 3 + 2 sp the Maxwellian momentum of species sp.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void inflow_draw(const InflowParams &f, uint32_t n, uint32_t stream, double &a, double &b)
{
    uint32_t r[4];
    philox4x32_10(n, f.call, stream, 0, f.seed, 0x494E4A43u, r);
    a = u01(r[0], r[1]);
    b = u01(r[2], r[3]);
}

// The position of trial n (local coordinates) and whether it is accepted:
// the density, and only the layer the flow emptied in one step
// (bc_inflow.F90:165-178).
__device__ __forceinline__ bool inflow_trial(const InflowParams &f, uint32_t n, double &xl, double &yl, double &zl)
{
    double r1, r2, r3, racpt;
    inflow_draw(f, n, 0, r1, r2);
    inflow_draw(f, n, 1, r3, racpt);
    xl = f.x1 + r1 * (f.x2 - f.x1);
    yl = f.y1 + r2 * (f.y2 - f.y1);
    zl = f.z1 + r3 * (f.z2 - f.z1);
    const double xg = xl + (0.0 - 3.0), yg = yl + (0.0 - 3.0), zg = f.dims == 3 ? zl + (0.0 - 3.0) : zl;
    bool acpt = racpt <= f.density;
    switch (f.side) {
        case 1: if (xg > f.pos + f.drift[0] * f.c) acpt = false; break;
        case 2: if (xg < f.pos + f.drift[0] * f.c) acpt = false; break;
        case 3: if (yg > f.pos + f.drift[1] * f.c) acpt = false; break;
        case 4: if (yg < f.pos + f.drift[1] * f.c) acpt = false; break;
        case 5: if (zg > f.pos + f.drift[2] * f.c) acpt = false; break;
        default: if (zg < f.pos + f.drift[2] * f.c) acpt = false; break;
    }
    return acpt;
}

__global__ void __launch_bounds__(256) k_inflow_count(InflowParams f, uint32_t *counts)
{
    __shared__ uint32_t c;
    if (threadIdx.x == 0) c = 0;
    __syncthreads();
    const long long base = (long long)blockIdx.x * kTile;
    uint32_t mine = 0;
    for (int r = 0; r < kTile / 256; r++) {
        const long long t = base + r * 256 + threadIdx.x;
        double xl, yl, zl;
        if (t < f.ntrial && inflow_trial(f, (uint32_t)t, xl, yl, zl)) mine++;
    }
    atomicAdd(&c, mine);
    __syncthreads();
    if (threadIdx.x == 0) counts[blockIdx.x] = c;
}

// The accepted trials' particles, nsp per trial in species order, appended
// at used + nsp * (rank of the trial among the accepted ones): the
// reference's order of InsertParticleAt calls.  Nothing when they do not fit.
__global__ void __launch_bounds__(256) k_inflow_fill(GridP g, InflowParams f, const double *__restrict__ X,
                                                     const double *__restrict__ P, int nt, PartF64 p,
                                                     const Counters *__restrict__ cnt, const uint32_t *__restrict__ offs,
                                                     const uint32_t *__restrict__ total, long long capacity, int *err)
{
    __shared__ uint32_t wh[kTileWarps];
    const long long used = cnt->used;
    if (used + (long long)f.nsp * (long long)*total > capacity) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_error(err, PIC_DEVERR_OVERFLOW);
        return;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long wbase = (long long)blockIdx.x * kTile + (long long)warp * kWarpItems;
    const uint32_t lt = lanemask_lt();
    uint32_t mine = 0;
    for (int r = 0; r < kWarpItems / 32; r++) {
        const long long t = wbase + r * 32 + lane;
        double xl, yl, zl;
        const bool acc = t < f.ntrial && inflow_trial(f, (uint32_t)t, xl, yl, zl);
        mine += __popc(__ballot_sync(0xffffffffu, acc));
    }
    if (lane == 0) wh[warp] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = offs[blockIdx.x];
        for (int k = 0; k < kTileWarps; k++) {
            const uint32_t t = wh[k];
            wh[k] = run;
            run += t;
        }
    }
    __syncthreads();
    uint32_t run = wh[warp];
    for (int r = 0; r < kWarpItems / 32; r++) {
        const long long t = wbase + r * 32 + lane;
        double xl = 0, yl = 0, zl = 0;
        const bool acc = t < f.ntrial && inflow_trial(f, (uint32_t)t, xl, yl, zl);
        const uint32_t b = __ballot_sync(0xffffffffu, acc);
        if (acc) {
            const long long slot = used + (long long)f.nsp * (long long)(run + __popc(b & lt));
            for (int sp = 0; sp < f.nsp; sp++) {
                double rmb, riso2, riso3, unused;
                inflow_draw(f, (uint32_t)t, 2 + 2 * sp, rmb, riso2);
                inflow_draw(f, (uint32_t)t, 3 + 2 * sp, riso3, unused);
                double u, v, w;
                maxwell_momentum(X, P, nt, f.temp[sp], rmb, riso2, riso3, f.drift[0], f.drift[1], f.drift[2], u, v, w);
                const long long o = slot + sp;
                p.x[o] = xl;
                p.y[o] = yl;
                p.z[o] = zl;
                p.u[o] = u;
                p.v[o] = v;
                p.w[o] = w;
                p.q[o] = f.charge[sp];
                p.flv[o] = f.flv[sp];
            }
        }
        run += __popc(b);
    }
}

__global__ void k_inflow_finish(Counters *cnt, const uint32_t *__restrict__ total, int nsp, long long capacity)
{
    const long long n = (long long)nsp * (long long)*total;
    if (cnt->used + n <= capacity) cnt->used += n;
}

int launch_inflow(const GridP &g, const InflowParams &f, const double *X, const double *P, int nt, PartF64 &p,
                  Counters *cnt, SortScratch &sc, long long capacity, int *err, cudaStream_t s)
{
    if (f.ntrial <= 0) return PIC_OK;
    const size_t ntiles = (size_t)((f.ntrial + kTile - 1) / kTile);
    if (ntiles > 256 * sc.ntiles) return PIC_ERR_OVERFLOW;
    uint32_t *total = sc.scan_tmp + sc.scan_tmp_len - 1;
    k_inflow_count<<<(unsigned)ntiles, 256, 0, s>>>(f, sc.hist);
    count_launches(1);
    scan_exclusive_u32(sc.hist, sc.hist, ntiles, sc.scan_tmp, total, s);
    k_inflow_fill<<<(unsigned)ntiles, 256, 0, s>>>(g, f, X, P, nt, p, cnt, sc.hist, total, capacity, err);
    k_inflow_finish<<<1, 1, 0, s>>>(cnt, total, f.nsp, capacity);
    count_launches(2);
    return PIC_OK;
}

}  // namespace pic
