// noalloc.cu -- field energy of caller-owned device arrays without any device
// allocation.
//
// Some callers cannot allocate device memory at the point where they want a
// diagnostic: a host whose memory pool has reserved the GPU's memory up front
// (every byte belongs to that pool, so a direct cudaMalloc can fail although
// the pool has room), or a host that steps the simulation in device arrays it
// manages itself and must not let a library cudaMalloc / cudaFree in between
// (cudaFree synchronizes the whole device).  pic_field_energy_noalloc serves
// them: the caller passes the field arrays and a 2-double output, both on the
// device, and the per-block partial sums of the reduction live in a
// fixed-size array in this file's device memory instead of a buffer the
// library would allocate.
//
// That array is global to the library: every GPU that loads the library holds
// it until the process exits, and every call shares it, so calls whose work
// overlaps on the GPU (on different streams, or from different host threads)
// race on it.  Each call overwrites every partial it later reads, so nothing
// in it has to start at zero, and it keeps the last call's contents.
#include "common.cuh"
#include "kernels.cuh"

namespace pic {

// At most this many per-block partial pairs: the reduction launches at most
// kSMs * 8 blocks (field_energy_blocks) and strides over any grid size.
constexpr int kNoAllocMaxBlocks = kSMs * 8;

static __device__ __align__(256) double g_energy_partials[2 * kNoAllocMaxBlocks];

// Device address of g_energy_partials in the current context: in host code
// the symbol is only a host-side stand-in.  Looked up on every call (no
// allocation, a table look-up in the runtime), so the address stays right
// after a cudaDeviceReset or on another device made current.
static int noalloc_scratch(double **out)
{
    double *p = nullptr;
    if (cudaGetSymbolAddress((void **)&p, g_energy_partials) != cudaSuccess || !p) return PIC_ERR_CUDA;
    *out = p;
    return PIC_OK;
}

}  // namespace pic

using namespace pic;

extern "C" int pic_field_energy_noalloc(const double *Ex, const double *Ey, const double *Ez, const double *Bx,
                                        const double *By, const double *Bz, int32_t nx, int32_t ny, int32_t nz,
                                        int32_t dims, double *out2, void *stream)
{
    if (!Ex || !Ey || !Ez || !Bx || !By || !Bz || !out2) return PIC_ERR_INVALID;
    if ((dims != 2 && dims != 3) || nx < 1 || ny < 1 || (dims == 3 && nz < 1)) return PIC_ERR_INVALID;
    GridP g = {};
    g.dims = dims;
    g.nx = nx;
    g.ny = ny;
    g.nz = dims == 3 ? nz : 1;
    g.mx = nx + 5;
    g.my = ny + 5;
    g.mz = dims == 3 ? nz + 5 : 1;
    g.sy = g.mx;
    g.sz = (long long)g.mx * g.my;
    g.ncell = g.sz * g.mz;
    g.geom = PIC_GEOM_CARTESIAN;
    const int nblocks = field_energy_blocks(g);
    if (nblocks < 1 || nblocks > kNoAllocMaxBlocks) return PIC_ERR_INVALID;  // beyond the scratch array
    double *partials = nullptr;
    const int r = noalloc_scratch(&partials);
    if (r) return r;
    const void *E[3] = {Ex, Ey, Ez}, *B[3] = {Bx, By, Bz};
    launch_field_energy(g, E, B, false, partials, nblocks, out2, (cudaStream_t)stream);
    return cudaGetLastError() == cudaSuccess ? PIC_OK : PIC_ERR_CUDA;
}
