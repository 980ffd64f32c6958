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
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const double *o = in + 8 * t;
        const long long d = used + t;
        p.q[d] = o[0];
        p.x[d] = o[1];
        p.y[d] = o[2];
        p.z[d] = o[3];
        p.u[d] = o[4];
        p.v[d] = o[5];
        p.w[d] = o[6];
        p.flv[d] = (int)o[7];
    }
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
    const int ci = cell % g.mx + 1;
    return ci >= g.mx - 2 ? 0 : (ci <= 2 ? 1 : -1);   // 0 right-bound, 1 left-bound
}

__global__ void __launch_bounds__(256) k_slab_count_f32(GridP g, PartF32 p, const Counters *__restrict__ cnt,
                                                        uint32_t *counts, int ntiles)
{
    __shared__ uint32_t c[2];
    if (threadIdx.x < 2) c[threadIdx.x] = 0;
    __syncthreads();
    const long long used = cnt->used, base = (long long)blockIdx.x * kSlabTile;
    uint32_t r = 0, l = 0;
    for (int q = threadIdx.x; q < kSlabTile; q += 256) {
        const long long n = base + q;
        if (n >= used) break;
        const int sd = f32_side(g, p.key[n]);
        r += sd == 0;
        l += sd == 1;
    }
    r = __reduce_add_sync(0xffffffffu, r);
    l = __reduce_add_sync(0xffffffffu, l);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&c[0], r);
        atomicAdd(&c[1], l);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        counts[blockIdx.x] = c[0];
        counts[ntiles + blockIdx.x] = c[1];
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
    const long long used = cnt->used, base = (long long)blockIdx.x * kSlabTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    uint32_t run[2] = {offs[blockIdx.x], offs[ntiles + blockIdx.x]};
    const double len = g.xlen;
    for (int r0 = 0; r0 < kSlabTile; r0 += 256) {
        const long long n = base + r0 + threadIdx.x;
        const int sd = n < used ? f32_side(g, p.key[n]) : -1;
        const uint32_t b0 = __ballot_sync(0xffffffffu, sd == 0), b1 = __ballot_sync(0xffffffffu, sd == 1);
        if (lane == 0) {
            wsum[0][warp] = __popc(b0);
            wsum[1][warp] = __popc(b1);
        }
        __syncthreads();
        uint32_t before[2] = {0, 0}, chunk[2] = {0, 0};
        for (int w = 0; w < 8; w++)
            for (int k = 0; k < 2; k++) {
                if (w < warp) before[k] += wsum[k][w];
                chunk[k] += wsum[k][w];
            }
        if (sd >= 0) {
            const uint32_t pos = run[sd] + before[sd] + __popc((sd == 0 ? b0 : b1) & lt);
            const uint32_t key = p.key[n];
            const int flv = (int)(key >> kFlvShift), cell = (int)(key & kCellMask);
            const int ci = cell % g.mx + 1, jk = cell / g.mx, cj = jk % g.my + 1, ck = jk / g.my + 1;
            // CopyTransferPrtl / InsertPrtls (subdomains.F90:720-740): a right
            // leaver -len, a left one +len
            const double x = (double)ci + (double)p.dx[n];
            double *o = out + 8 * (size_t)pos;
            o[0] = (double)p.w[n];
            o[1] = sd == 0 ? (x - len) + 0.0 : (x - 0.0) + len;
            o[2] = (double)cj + (double)p.dy[n];
            o[3] = g.dims == 3 ? (double)ck + (double)p.dz[n] : 1.5;
            o[4] = (double)p.ux[n];
            o[5] = (double)p.uy[n];
            o[6] = (double)p.uz[n];
            o[7] = (double)flv;
            p.key[n] = 0u;   // a hole
        }
        run[0] += chunk[0];
        run[1] += chunk[1];
        __syncthreads();
    }
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
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const double *o = in + 8 * t;
        const long long d = used + t;
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
