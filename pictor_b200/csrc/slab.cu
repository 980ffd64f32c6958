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

// One face: buffer element q = ((comp * nl + l) * mz + k) * my + j.
__global__ void k_slab_pack(GridP g, int which, double *F0, double *F1, double *F2, double *__restrict__ out,
                            FaceLayers fl)
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
        double *F = comp == 0 ? F0 : comp == 1 ? F1 : F2;
        out[q] = F[c];
        if (which == 2) F[c] = 0.0;   // the ghost current leaves this slab
    }
}

__global__ void k_slab_unpack(GridP g, int which, double *F0, double *F1, double *F2, const double *__restrict__ in,
                              FaceLayers fl)
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
        double *F = comp == 0 ? F0 : comp == 1 ? F1 : F2;
        // AddBuffToFld adds the neighbour's ghost current after this slab's own
        // (the order of the fold's J + J(partner)); fields are copied
        F[c] = which == 2 ? F[c] + in[q] : in[q];
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

int face_grid(const GridP &g, int nl)
{
    const long long total = 3ll * nl * g.my * g.mz;
    const long long b = (total + kThreads - 1) / kThreads;
    return (int)(b < kSMs * 8 ? (b > 0 ? b : 1) : kSMs * 8);
}

}  // namespace

void launch_slab_pack_fields(const GridP &g, int which, double *const F[3], double *to_left, double *to_right,
                             cudaStream_t s)
{
    for (int side = 0; side < 2; side++) {
        const FaceLayers fl = send_layers(g.mx, which, side);
        k_slab_pack<<<face_grid(g, fl.n), kThreads, 0, s>>>(g, which, F[0], F[1], F[2], side == 0 ? to_left : to_right,
                                                             fl);
    }
    count_launches(2);
}

void launch_slab_unpack_fields(const GridP &g, int which, double *const F[3], const double *from_left,
                               const double *from_right, cudaStream_t s)
{
    for (int side = 0; side < 2; side++) {
        const FaceLayers fl = recv_layers(g.mx, which, side);
        k_slab_unpack<<<face_grid(g, fl.n), kThreads, 0, s>>>(g, which, F[0], F[1], F[2],
                                                               side == 0 ? from_left : from_right, fl);
    }
    count_launches(2);
}

void launch_slab_append(const GridP &g, PartF64 &p, Counters *cnt, const double *in, long long n, long long capacity,
                        int *err, cudaStream_t s)
{
    if (n <= 0) return;
    const long long b = (n + kThreads - 1) / kThreads;
    k_slab_append<<<(int)(b < kSMs * 8 ? b : kSMs * 8), kThreads, 0, s>>>(p, cnt, in, n, capacity, err);
    k_slab_append_finish<<<1, 1, 0, s>>>(cnt, n, capacity);
    count_launches(2);
}

}  // namespace pic
