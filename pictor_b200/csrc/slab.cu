// slab.cu -- the x faces of one slab of a domain split along x.
//
// Reference: src/comm/comm_fld.F90:75-130 (SendRecvFlds: interior layers into
// the neighbours' ghosts), :15-72 and :288-307 (UpdateCurrentAllFaces /
// AddBuffToFld: ghost current added onto the neighbours' interior), the layer
// map of src/comm/subdomains.F90:592-612, src/comm/loadprtlout.F90:13-106 and
// src/comm/comm_prtl.F90:11-66 (particles through the x faces).  With one
// rank the neighbour is the rank itself and this is the periodic image that
// the single-domain kernels fold into their stores; in the slab form
// (GridP::x_external) those kernels leave the x ghosts alone and the host
// moves these face buffers between slabs (NCCL, or device copies when the
// slabs share a GPU).
//
// Face buffers are [component][layer][z][y] doubles (ghosted my x mz per
// layer, y fastest).  E and B send interior layers {3,4,5} to the left
// neighbour (its ghosts mx-2..mx) and {mx-4,mx-3} to the right one (its
// ghosts 1,2); J sends its ghost layers {1,2} left (added to the neighbour's
// mx-4,mx-3) and {mx-2..mx} right (added to its 3..5), and zeroes them.
#include "common.cuh"
#include "kernels.cuh"

namespace pic {

namespace {

// Layers of the face buffers (1-based x indices), by field kind (0 E, 1 B:
// copy; 2 J: add) and side (0 left, 1 right).
struct FaceLayers {
    int n;        // layers
    int x0;       // first layer (consecutive)
};
__host__ __device__ inline FaceLayers send_layers(int mx, int which, int side)
{
    if (which == 2) return side == 0 ? FaceLayers{2, 1} : FaceLayers{3, mx - 2};
    return side == 0 ? FaceLayers{3, 3} : FaceLayers{2, mx - 4};
}
__host__ __device__ inline FaceLayers recv_layers(int mx, int which, int side)
{
    // what the left neighbour sent right lands on our side 0, and so on
    if (which == 2) return side == 0 ? FaceLayers{3, 3} : FaceLayers{2, mx - 4};
    return side == 0 ? FaceLayers{2, 1} : FaceLayers{3, mx - 2};
}

// One face: buffer element q = ((comp * nl + l) * mz + k) * my + j; the
// buffers hold doubles for either precision of the fields (an FP32 value
// goes through them exactly).
template <typename T>
__global__ void k_slab_pack(GridP g, int which, T *F0, T *F1, T *F2, double *__restrict__ out, FaceLayers fl)
{
    const long long per = (long long)g.my * g.mz;
    const long long total = 3ll * fl.n * per;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int comp = (int)(q / (fl.n * per));
        const long long r = q - (long long)comp * fl.n * per;
        const int l = (int)(r / per);
        const long long jk = r - (long long)l * per;
        const long long c = (long long)(fl.x0 + l - 1) + g.mx * jk;   // (x, j, k) with jk = (j-1) + my (k-1)
        T *F = comp == 0 ? F0 : comp == 1 ? F1 : F2;
        out[q] = (double)F[c];
        if (which == 2) F[c] = (T)0;   // the ghost current leaves this slab
    }
}

template <typename T>
__global__ void k_slab_unpack(GridP g, int which, T *F0, T *F1, T *F2, const double *__restrict__ in, FaceLayers fl)
{
    const long long per = (long long)g.my * g.mz;
    const long long total = 3ll * fl.n * per;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        const int comp = (int)(q / (fl.n * per));
        const long long r = q - (long long)comp * fl.n * per;
        const int l = (int)(r / per);
        const long long jk = r - (long long)l * per;
        const long long c = (long long)(fl.x0 + l - 1) + g.mx * jk;
        T *F = comp == 0 ? F0 : comp == 1 ? F1 : F2;
        // AddBuffToFld adds the neighbour's ghost current after this slab's own
        // (the order of the fold's J + J(partner)); fields are copied
        F[c] = which == 2 ? F[c] + (T)in[q] : (T)in[q];
    }
}

// One received particle (8 doubles: q, x, y, z, u, v, w, flv, already in
// this slab's coordinates) into slot d of the reference layout.
__device__ __forceinline__ void append_record_f64(const PartF64 &p, long long d, const double *o)
{
    p.q[d] = o[0];
    p.x[d] = o[1];
    p.y[d] = o[2];
    p.z[d] = o[3];
    p.u[d] = o[4];
    p.v[d] = o[5];
    p.w[d] = o[6];
    p.flv[d] = (int)o[7];
}

// AppendParticles (comm_prtl.F90:11-30) of n received particles (8 doubles
// each, already in this slab's coordinates) after the used slots.
__global__ void k_slab_append(PartF64 p, Counters *cnt, const double *__restrict__ in, long long n, long long capacity,
                              int *err)
{
    const long long used = cnt->used;
    if (used + n > capacity) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_error(err, PIC_DEVERR_OVERFLOW);
        return;
    }
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        append_record_f64(p, used + t, in + 8 * t);
}

__global__ void k_slab_append_finish(Counters *cnt, long long n, long long capacity)
{
    if (cnt->used + n <= capacity) cnt->used += n;
}

// --- the FP32 form's x leavers ---------------------------------------------
// The FP32 mover of a slab leaves a particle that crossed an x face in the
// ghost cell beside it (cell 2: left, mx - 2: right; a move is below one
// cell).  These kernels send those particles to the outbox in the 8-double
// layout of the FP64 form, right-bound first, then left-bound, each group in
// slot order, x in the receiver's coordinates (+- the slab width, as the
// FP64 wrap shifts it), and leave holes.
constexpr int kSlabTile = 4096;

__device__ __forceinline__ int f32_side(const GridP &g, uint32_t key)
{
    if ((key >> kFlvShift) == 0) return -1;
    const int cell = (int)(key & kCellMask);
    const int ci = cell - fast_div((unsigned)cell, g.mx_magic, g.mx_shift) * g.mx + 1;
    return ci >= g.mx - 2 ? 0 : (ci <= 2 ? 1 : -1);   // 0 right-bound, 1 left-bound
}

// Each thread takes kSlabPer consecutive slots of a tile (16-byte loads of
// the keys, four at a time).
constexpr int kSlabPer = kSlabTile / 256;

__device__ __forceinline__ void load_tile_keys(const uint32_t *__restrict__ key, long long n0, long long used,
                                               uint32_t k[kSlabPer])
{
    if (n0 + kSlabPer <= used) {
#pragma unroll
        for (int v = 0; v < kSlabPer / 4; v++) {
            const uint4 q = *reinterpret_cast<const uint4 *>(key + n0 + 4 * v);
            k[4 * v] = q.x; k[4 * v + 1] = q.y; k[4 * v + 2] = q.z; k[4 * v + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int e = 0; e < kSlabPer; e++) k[e] = n0 + e < used ? key[n0 + e] : 0u;
    }
}

__global__ void __launch_bounds__(256) k_slab_count_f32(GridP g, PartF32 p, const Counters *__restrict__ cnt,
                                                        uint32_t *counts, int ntiles)
{
    __shared__ uint32_t c[2][8];
    const long long used = cnt->used, n0 = (long long)blockIdx.x * kSlabTile + (long long)threadIdx.x * kSlabPer;
    uint32_t k[kSlabPer];
    load_tile_keys(p.key, n0, used, k);
    uint32_t r = 0, l = 0;
#pragma unroll
    for (int e = 0; e < kSlabPer; e++) {
        const int sd = f32_side(g, k[e]);
        r += sd == 0;
        l += sd == 1;
    }
    r = __reduce_add_sync(0xffffffffu, r);
    l = __reduce_add_sync(0xffffffffu, l);
    if ((threadIdx.x & 31) == 0) {
        c[0][threadIdx.x >> 5] = r;
        c[1][threadIdx.x >> 5] = l;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        uint32_t t = 0;
        for (int w = 0; w < 8; w++) t += c[threadIdx.x][w];
        counts[(size_t)threadIdx.x * ntiles + blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(256) k_slab_scatter_f32(GridP g, PartF32 p, const Counters *__restrict__ cnt,
                                                          const uint32_t *__restrict__ offs,
                                                          const uint32_t *__restrict__ total, int ntiles, double *out,
                                                          long long out_cap, int *err)
{
    __shared__ uint32_t wsum[2][8];
    if ((long long)*total > out_cap) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_error(err, PIC_DEVERR_OVERFLOW);
        return;
    }
    const long long used = cnt->used, n0 = (long long)blockIdx.x * kSlabTile + (long long)threadIdx.x * kSlabPer;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t k[kSlabPer];
    load_tile_keys(p.key, n0, used, k);
    int sd[kSlabPer];
    uint32_t cr = 0, cl = 0;
#pragma unroll
    for (int e = 0; e < kSlabPer; e++) {
        sd[e] = f32_side(g, k[e]);
        cr += sd[e] == 0;
        cl += sd[e] == 1;
    }
    // the thread's first position per side: the tile's offset, the lower
    // warps' and the lower lanes' leavers (slot order within each side)
    uint32_t ir = cr, il = cl;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t vr = __shfl_up_sync(0xffffffffu, ir, o), vl = __shfl_up_sync(0xffffffffu, il, o);
        if (lane >= o) {
            ir += vr;
            il += vl;
        }
    }
    if (lane == 31) {
        wsum[0][warp] = ir;
        wsum[1][warp] = il;
    }
    __syncthreads();
    if ((__ballot_sync(0xffffffffu, cr + cl != 0)) == 0) return;   // no leaver in the warp's slots
    uint32_t pr = offs[blockIdx.x] + ir - cr, pl = offs[ntiles + blockIdx.x] + il - cl;
    for (int w = 0; w < warp; w++) {
        pr += wsum[0][w];
        pl += wsum[1][w];
    }
    const double len = g.xlen;
#pragma unroll
    for (int e = 0; e < kSlabPer; e++) {
        if (sd[e] < 0) continue;
        const long long n = n0 + e;
        const uint32_t key = k[e];
        const int flv = (int)(key >> kFlvShift);
        int ci, cj, ck;
        decode_cell(g, (int)(key & kCellMask), ci, cj, ck);
        // CopyTransferPrtl / InsertPrtls (subdomains.F90:720-740): a right
        // leaver -len, a left one +len
        const double x = (double)ci + (double)p.dx[n];
        double *o = out + 8 * (size_t)(sd[e] == 0 ? pr++ : pl++);
        o[0] = (double)p.w[n];
        o[1] = sd[e] == 0 ? (x - len) + 0.0 : (x - 0.0) + len;
        o[2] = (double)cj + (double)p.dy[n];
        o[3] = g.dims == 3 ? (double)ck + (double)p.dz[n] : 1.5;
        o[4] = (double)p.ux[n];
        o[5] = (double)p.uy[n];
        o[6] = (double)p.uz[n];
        o[7] = (double)flv;
        p.key[n] = 0u;   // a hole
    }
}

// One received particle (8 doubles, the FP64 layout) into slot d of the FP32
// form: its cell and offsets, FP32 momenta and weight; a particle outside
// the slab's interior in x (or its ghost frame in y, z) leaves a hole.
__device__ __forceinline__ void append_record_f32(const GridP &g, const PartF32 &p, long long d, const double *o,
                                                  int *err)
{
    const int flv = (int)o[7];
    const double x = o[1], y = o[2], z = o[3];
    const double fx = floor(x), fy = floor(y), fz = g.dims == 3 ? floor(z) : 1.0;
    uint32_t key = 0;
    if (flv < 1 || flv > 15 || !(x >= 3.0 && x < (double)(g.mx - 2) && y >= 2.0 && y < (double)(g.my - 1) &&
                                  (g.dims == 2 || (z >= 2.0 && z < (double)(g.mz - 1))))) {
        raise_error(err, PIC_DEVERR_RANGE);   // left a hole
    } else {
        const int ci = (int)fx, cj = wrap_index((int)fy, g.my), ck = g.dims == 3 ? wrap_index((int)fz, g.mz) : 1;
        key = ((uint32_t)flv << kFlvShift) | (uint32_t)cidx(g, ci, cj, ck);
    }
    p.key[d] = key;
    p.dx[d] = (float)(x - fx);
    p.dy[d] = (float)(y - fy);
    if (g.dims == 3) p.dz[d] = (float)(z - fz);
    p.ux[d] = (float)o[4];
    p.uy[d] = (float)o[5];
    p.uz[d] = (float)o[6];
    p.w[d] = (float)o[0];
}

// The received particles (8 doubles each, in this slab's coordinates)
// appended after the used slots, converted to the cell-relative layout.
__global__ void k_slab_append_f32(GridP g, PartF32 p, Counters *cnt, const double *__restrict__ in, long long n,
                                  long long capacity, int *err)
{
    const long long used = cnt->used;
    if (used + n > capacity) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_error(err, PIC_DEVERR_OVERFLOW);
        return;
    }
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        append_record_f32(g, p, used + t, in + 8 * t, err);
}

// --- fixed-size boxes ------------------------------------------------------
// A box of cap particles is cap + 1 records of 8 doubles: record 0 holds the
// count (word 0), the particles follow.  Nothing about the exchange then
// needs the host: the counts travel with the particles.
struct Inbox2 {
    const double *l, *r;   // from the left and from the right neighbour
    long long cap;
    int closed;            // GridP::closed_x: a face without neighbour receives nothing
};
__device__ __forceinline__ void inbox_counts(const Inbox2 &ib, long long &nl, long long &nr)
{
    nl = (ib.closed & 1) ? 0 : (long long)ib.l[0];
    nr = (ib.closed & 2) ? 0 : (long long)ib.r[0];
    nl = nl < 0 ? 0 : (nl > ib.cap ? ib.cap : nl);
    nr = nr < 0 ? 0 : (nr > ib.cap ? ib.cap : nr);
}

// After the pack into to_right's payload (right-bound records, then the
// left-bound ones): both headers, and the left-bound records moved to
// to_left's payload.  A pack that overflowed moved nothing: both counts 0.
__global__ void k_slab_split(const uint32_t *__restrict__ sent, double *to_left, double *to_right, long long cap)
{
    const long long all = (long long)sent[1];
    const bool ok = all <= cap;
    const long long nr = ok ? (long long)sent[0] : 0, nl = ok ? all - (long long)sent[0] : 0;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x, stride = (long long)gridDim.x * blockDim.x;
    if (tid < 8) {
        to_right[tid] = tid == 0 ? (double)nr : 0.0;
        to_left[tid] = tid == 0 ? (double)nl : 0.0;
    }
    for (long long w = tid; w < 8 * nl; w += stride) to_left[8 + w] = to_right[8 + 8 * nr + w];
}

// AppendParticles of both inboxes: from the left, then from the right.
template <bool F32>
__global__ void k_slab_append_fixed(GridP g, PartF64 p64, PartF32 p32, Counters *cnt, Inbox2 ib, long long capacity,
                                    int *err)
{
    long long nl, nr;
    inbox_counts(ib, nl, nr);
    const long long n = nl + nr, used = cnt->used;
    if (used + n > capacity) {
        if (blockIdx.x == 0 && threadIdx.x == 0) raise_error(err, PIC_DEVERR_OVERFLOW);
        return;
    }
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const double *o = t < nl ? ib.l + 8 * (t + 1) : ib.r + 8 * (t - nl + 1);
        if (F32) append_record_f32(g, p32, used + t, o, err);
        else append_record_f64(p64, used + t, o);
    }
}

__global__ void k_slab_append_fixed_finish(Counters *cnt, Inbox2 ib, long long capacity)
{
    long long nl, nr;
    inbox_counts(ib, nl, nr);
    if (cnt->used + nl + nr <= capacity) cnt->used += nl + nr;
}


int face_grid(const GridP &g, int nl)
{
    const long long total = 3ll * nl * g.my * g.mz;
    const long long b = (total + kThreads - 1) / kThreads;
    return (int)(b < kSMs * 8 ? (b > 0 ? b : 1) : kSMs * 8);
}

}  // namespace

template <typename T>
void launch_slab_pack_fields(const GridP &g, int which, T *const F[3], double *to_left, double *to_right, cudaStream_t s)
{
    for (int side = 0; side < 2; side++) {
        if ((g.closed_x >> side) & 1) continue;   // no neighbour on that face: nothing leaves
        const FaceLayers fl = send_layers(g.mx, which, side);
        k_slab_pack<T><<<face_grid(g, fl.n), kThreads, 0, s>>>(g, which, F[0], F[1], F[2],
                                                                side == 0 ? to_left : to_right, fl);
        count_launches(1);
    }
}

template <typename T>
void launch_slab_unpack_fields(const GridP &g, int which, T *const F[3], const double *from_left,
                               const double *from_right, cudaStream_t s)
{
    for (int side = 0; side < 2; side++) {
        if ((g.closed_x >> side) & 1) continue;   // no neighbour: the face's ghosts stay this grid's
        const FaceLayers fl = recv_layers(g.mx, which, side);
        k_slab_unpack<T><<<face_grid(g, fl.n), kThreads, 0, s>>>(g, which, F[0], F[1], F[2],
                                                                  side == 0 ? from_left : from_right, fl);
        count_launches(1);
    }
}
template void launch_slab_pack_fields<double>(const GridP &, int, double *const[3], double *, double *, cudaStream_t);
template void launch_slab_pack_fields<float>(const GridP &, int, float *const[3], double *, double *, cudaStream_t);
template void launch_slab_unpack_fields<double>(const GridP &, int, double *const[3], const double *, const double *,
                                                cudaStream_t);
template void launch_slab_unpack_fields<float>(const GridP &, int, float *const[3], const double *, const double *,
                                               cudaStream_t);

void launch_slab_append(const GridP &g, PartF64 &p, Counters *cnt, const double *in, long long n, long long capacity,
                        int *err, cudaStream_t s)
{
    if (n <= 0) return;
    const long long b = (n + kThreads - 1) / kThreads;
    k_slab_append<<<(int)(b < kSMs * 8 ? b : kSMs * 8), kThreads, 0, s>>>(p, cnt, in, n, capacity, err);
    k_slab_append_finish<<<1, 1, 0, s>>>(cnt, n, capacity);
    count_launches(2);
}

// The x leavers of an FP32 slab into `out` (out_cap particles of 8 doubles);
// sent = {right-bound, right + left-bound} on the device.  counts needs
// 2 (capacity / 4096 + 1) words, scan_tmp and total scan scratch.
void launch_slab_pack_f32(const GridP &g, PartF32 &p, const Counters *cnt, double *out, long long out_cap,
                          uint32_t *counts, uint32_t *scan_tmp, uint32_t *total, uint32_t *sent, long long capacity,
                          int *err, cudaStream_t s)
{
    const int ntiles = (int)((capacity + kSlabTile - 1) / kSlabTile);
    k_slab_count_f32<<<ntiles, 256, 0, s>>>(g, p, cnt, counts, ntiles);
    count_launches(1);
    scan_exclusive_u32(counts, counts, 2 * (size_t)ntiles, scan_tmp, total, s);
    k_slab_scatter_f32<<<ntiles, 256, 0, s>>>(g, p, cnt, counts, total, ntiles, out, out_cap, err);
    count_launches(1);
    cudaMemcpyAsync(sent, counts + ntiles, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(sent + 1, total, sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
}

// The x leavers into fixed-size boxes (record 0: the count; FP64 or FP32
// form): the pack writes right- then left-bound records into to_right's
// payload, the split moves the left-bound ones to to_left's.
void launch_slab_pack_fixed(const GridP &g, bool fp32, PartF64 &p64, PartF32 &p32, Counters *cnt, SortScratch &sc,
                            double *to_left, double *to_right, long long cap, uint32_t *sent, long long capacity,
                            int *err, cudaStream_t s)
{
    if (fp32)
        launch_slab_pack_f32(g, p32, cnt, to_right + 8, cap, sc.hist, sc.scan_tmp, sc.scan_tmp + sc.scan_tmp_len - 1,
                             sent, capacity, err, s);
    else
        launch_exchange_f64(g, p64, cnt, sc, capacity, err, s, to_right + 8, cap, sent);
    k_slab_split<<<kSMs, kThreads, 0, s>>>(sent, to_left, to_right, cap);
    count_launches(1);
}

void launch_slab_append_fixed(const GridP &g, bool fp32, PartF64 &p64, PartF32 &p32, Counters *cnt,
                              const double *from_left, const double *from_right, long long cap, long long capacity,
                              int *err, cudaStream_t s)
{
    const Inbox2 ib{from_left, from_right, cap, g.closed_x};
    if (fp32) k_slab_append_fixed<true><<<kSMs * 4, kThreads, 0, s>>>(g, p64, p32, cnt, ib, capacity, err);
    else k_slab_append_fixed<false><<<kSMs * 4, kThreads, 0, s>>>(g, p64, p32, cnt, ib, capacity, err);
    k_slab_append_fixed_finish<<<1, 1, 0, s>>>(cnt, ib, capacity);
    count_launches(2);
}

void launch_slab_append_f32(const GridP &g, PartF32 &p, Counters *cnt, const double *in, long long n,
                            long long capacity, int *err, cudaStream_t s)
{
    if (n <= 0) return;
    const long long b = (n + kThreads - 1) / kThreads;
    k_slab_append_f32<<<(int)(b < kSMs * 8 ? b : kSMs * 8), kThreads, 0, s>>>(g, p, cnt, in, n, capacity, err);
    k_slab_append_finish<<<1, 1, 0, s>>>(cnt, n, capacity);
    count_launches(2);
}

}  // namespace pic
