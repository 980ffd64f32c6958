// common.cuh -- shared device-side definitions of the B200 PIC step.
//
// Grid layout (both precisions): column-major (mx,my,mz) with 2 low and 3 high
// ghost layers per axis (mx = nx+5; mz = 1 in 2D), as in the reference
// (src/comm/subdomains/subdomains.F90:42-50).  Indices in comments are 1-based
// like the reference; memory offsets are 0-based.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pictor_b200.h"

namespace pic {

constexpr int kThreads = 256;         // threads per CTA for streaming kernels
constexpr int kSMs = 148;             // B200 SM count (2 dies x 74)

// Scalar parameters every kernel needs, passed by value (fits in the 4 KB
// kernel parameter space).
struct GridP {
    int dims, nx, ny, nz, mx, my, mz;
    int fdtd;
    long long ncell;                  // mx*my*mz
    long long sy, sz;                 // strides of j and k: mx, mx*my
    double c, h, fc, sqc, cinv, qi;   // Courant, fld_halfc, fldc, c^2, 1/c, qi
    double bext[3];
    double lehe[12];                  // alpha_x..z, beta_xy,xz,yx,yz,zx,zy, delta_x..z
    double qm[PIC_MAX_FLVR + 1];      // flvrqm (index 0 = hole -> 0)
    // particle bounds (subdomains.F90:52-67)
    double xmin, xmax, ymin, ymax, zmin, zmax, xlen, ylen, zlen;
    int geom;                         // PIC_GEOM_*
    int closed_x;                     // bit 0 / bit 1: the low / high x face has no neighbour (a cylinder's
                                      // axis or outer radius): leavers through it are dropped
    int inc_axis;                     // cylindrical: the axis is this grid's low x face
    double rmin;                      // cylindrical: r of the first interior cell's inner edge (xborders + rshift)
    int x_external;                   // slab form: x faces exchanged with neighbouring slabs (no x images)
    int exact_charge;                 // FP32 3D: exactly charge-conserving segment currents (pic_config)
    unsigned int mx_magic, my_magic;  // n / m = umulhi(n, magic) >> shift, exact for n < 2^28 (div_magic)
    int mx_shift, my_shift;
    // FP32 copies for the FP32 form: c, c^2, 1/c, qi, external B, q/m * 0.5
    float c_f, sqc_f, cinv_f, qi_f, bext_f[3];
    float qm_half_f[PIC_MAX_FLVR + 1];
};

// n / d by multiply-shift (the magic of GridP); exact for n < 2^28, d <= 4096.
__host__ __device__ inline void div_magic(unsigned int d, unsigned int &magic, int &shift)
{
    // k = max(32, 28 + ceil(log2 d)), magic = ceil(2^k / d) < 2^32 for d >= 2;
    // floor(n * magic / 2^k) = floor(n / d) when n * (magic d - 2^k) < 2^k,
    // which holds for n < 2^28 since magic d - 2^k < d <= 2^(k - 28)
    int l = 0;
    while ((1u << l) < d) l++;
    const int k = 28 + l > 32 ? 28 + l : 32;
    magic = (unsigned int)(((1ull << k) + d - 1) / d);
    shift = k - 32;
}
__device__ __forceinline__ int fast_div(unsigned int n, unsigned int magic, int shift)
{
    return (int)(__umulhi(n, magic) >> shift);
}
// (i,j,k), 1-based, of a linear ghosted cell index.
__device__ __forceinline__ void decode_cell(const GridP &g, int cell, int &i, int &j, int &k)
{
    const int jk = fast_div((unsigned)cell, g.mx_magic, g.mx_shift);
    i = cell - jk * g.mx + 1;
    k = fast_div((unsigned)jk, g.my_magic, g.my_shift);
    j = jk - k * g.my + 1;
    k += 1;
}

__host__ __device__ inline long long cidx(const GridP &g, int i, int j, int k)
{
    return (long long)(i - 1) + g.sy * (long long)(j - 1) + g.sz * (long long)(k - 1);
}

// Periodic image of a (possibly ghost) 1-based index along an axis with m
// entries and n = m-5 interior cells: ghosts 1,2 -> m-4,m-3 and m-2..m -> 3..5
// (the layer map of subdomains.F90:592-612 with a single periodic rank).
__host__ __device__ inline int wrap_index(int i, int m)
{
    const int n = m - 5;
    if (i < 3) return i + n;
    if (i > m - 3) return i - n;
    return i;
}

// Kernel-launch accounting (for the launch count a benchmark reports): every
// host launcher adds the number of kernels it enqueued.
void count_launches(int n);

// Loads of data a kernel does not write while it runs (ldro) and of data it
// may write through other threads (ldco).  The persistent ensemble step
// (ensemble.cu, compiled with PIC_COHERENT_LOADS) runs every phase of many
// steps in one launch: a work item reads what earlier items wrote on other
// SMs.  The non-coherent read-only path (ld.global.nc) is only defined for
// data that no thread writes during the kernel, so there both are weak
// loads (ld.global.ca): the PTX memory model orders them after the writers'
// stores through the items' release / acquire counters (one thread
// acquires, then a CTA barrier), whatever level of cache serves them.
#ifdef PIC_COHERENT_LOADS
template <typename T>
__device__ __forceinline__ T ldro(const T *p) { return __ldca(p); }
template <typename T>
__device__ __forceinline__ T ldco(const T *p) { return __ldca(p); }
#else
template <typename T>
__device__ __forceinline__ T ldro(const T *p) { return __ldg(p); }
template <typename T>
__device__ __forceinline__ T ldco(const T *p) { return *p; }
#endif

// Error bits written by kernels (never __trap): see PIC_DEVERR_*.
__device__ inline void raise_error(int *err, int bit) { atomicOr(err, bit); }

// A momentum triple is finite (false for NaN or +-Inf in any component).
// The movers test the pushed momentum before any index is formed from the
// new position: a non-finite displacement would truncate to an arbitrary
// cell, so the particle is left as it was and PIC_DEVERR_NAN is raised.
__device__ __forceinline__ bool finite3(float a, float b, float c)
{
    return fabsf(a) + fabsf(b) + fabsf(c) <= 3.402823466e38f;
}
__device__ __forceinline__ bool finite3(double a, double b, double c)
{
    return fabs(a) + fabs(b) + fabs(c) <= 1.7976931348623157e308;
}

// Device-side particle counters shared by the step kernels.
struct Counters {
    long long used;        // used_prtl_arr_size
    long long np;          // live particles (after a reorder)
    long long append;      // particles appended by the last exchange
    long long scratch[5];
};

}  // namespace pic
