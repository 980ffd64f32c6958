// adjoint.cu -- the differentiable form of the 2D Cartesian periodic step:
// forward step, hand-written adjoint kernels for the FDTD, the push and the
// deposit, checkpointed particle and field state with recomputation between
// checkpoints, and the gradient of J = sum_t 1/2 sum_cells |B_t|^2 with
// respect to every initial momentum and to the drift and temperatures of the
// Weibel loader.  No counterpart in the reference.
//
// The forward step restates the FP64 step of this library (MAIN.F90:42-284
// in 2D: UpdateBfieldHalf, MoveDepositPrtl with node-averaged gather
// movdep_routines.F90:6-223, relativistic Boris movdep.F90:143-167, zigzag
// deposit movdep.F90:177-237 and the z wrap :241-249, UpdateBfieldHalf,
// UpdateEfield + AddCurrent em_update.F90) on interior arrays with periodic
// indices instead of ghost layers, positions counted from the first interior
// cell (x_ref - 3), particles in fixed slots (the periodic wrap shifts the
// position by the box length; no holes, no reorder).  One change makes J a
// continuous function of the state: the out-of-plane current is split
// between the two zigzag segments at the z midpoint, as in the FP32 form;
// the reference's 2D z relay jumps when z crosses 1 or 2 in a step that also
// crosses an x or y cell face.  Without out-of-plane motion the step equals
// the FP64 step up to the order of the FP sums.
//
// Reverse step t, given the cotangents Ebar_t, Bbar_t of the fields after the
// step and pbar of the particles after it (x, y, z, u, v, w):
//   Bbar += B_t                                   (the objective term)
//   Bbar += c curlB^T(Ebar_t); Ebar_prev = Ebar_t (E_t = E + c curlB - J)
//   Ebar_prev += -c/2 curlE^T(Bbar)               (second B half step)
//   mover adjoint: J-bar = -Ebar_t; pbar <- d(move)^T pbar; the gather's
//   adjoint adds into Ebar_prev and Bbar
//   Ebar_prev += -c/2 curlE^T(Bbar)               (first B half step)
// The mover adjoint recomputes the particle's forward step from the tape and
// differentiates it by hand; floor() and the relay point's min/max are
// piecewise linear, so the derivative is the one of the active branch (the
// relay point moves with the midpoint only when the particle stays in its
// cell).
//
// Precision: T = double is the reference adjoint; T = float the FP32 form.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace pic {
namespace adj {

struct AG {
    int nx, ny;
    double c, h, fc, sqc, cinv, qi, bext[3], qm_half[PIC_MAX_FLVR + 1];
};

template <typename T>
struct PS {
    T *x, *y, *z, *u, *v, *w;
};

template <typename T>
struct F3 {
    T *x, *y, *z;
};

__device__ __forceinline__ int wrapi(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }
__device__ __forceinline__ int at(const AG &g, int i, int j) { return wrapi(i, g.nx) + g.nx * wrapi(j, g.ny); }

// ---------------------------------------------------------------------------
// Field operators (em_update.F90, 2D Yee, periodic)
// ---------------------------------------------------------------------------
// Bout = Bin - h curlE(E) in the reference's expression order
template <typename T>
__global__ void k_bhalf(AG g, F3<T> E, F3<T> Bin, F3<T> Bout)
{
    const T h = (T)g.h;
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c % g.nx, j = c / g.nx;
        const int cy = at(g, i, j + 1), cx = at(g, i + 1, j);
        const T bx = Bin.x[c] - h * (E.z[cy] - E.z[c]);
        const T by = Bin.y[c] + h * (E.z[cx] - E.z[c]);
        const T bz = (Bin.z[c] - h * (E.y[cx] - E.y[c])) + h * (E.x[cy] - E.x[c]);
        Bout.x[c] = bx;
        Bout.y[c] = by;
        Bout.z[c] = bz;
    }
}

// E <- E + c curlB(B) - J; J <- 0
template <typename T>
__global__ void k_efield(AG g, F3<T> E, F3<T> B, F3<T> J)
{
    const T fc = (T)g.fc;
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c % g.nx, j = c / g.nx;
        const int cy = at(g, i, j - 1), cx = at(g, i - 1, j);
        const T ex = (E.x[c] + fc * (B.z[c] - B.z[cy])) - J.x[c];
        const T ey = (E.y[c] - fc * (B.z[c] - B.z[cx])) - J.y[c];
        const T ez = ((E.z[c] + fc * (B.y[c] - B.y[cx])) - fc * (B.x[c] - B.x[cy])) - J.z[c];
        E.x[c] = ex;
        E.y[c] = ey;
        E.z[c] = ez;
        J.x[c] = J.y[c] = J.z[c] = (T)0;
    }
}

// acc += 1/2 sum |B|^2 (double accumulation)
template <typename T>
__global__ void k_benergy(AG g, F3<T> B, double *acc)
{
    __shared__ double red[8];
    double s = 0;
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const double bx = B.x[c], by = B.y[c], bz = B.z[c];
        s += 0.5 * (bx * bx + by * by + bz * bz);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        atomicAdd(acc, t);
    }
}

// Ebar += s * curlE^T(Bbar) (the adjoint of B -= h curlE with s = -h)
template <typename T>
__global__ void k_curlE_T(AG g, F3<T> Bbar, F3<T> Ebar, T s)
{
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c % g.nx, j = c / g.nx;
        const int jm = at(g, i, j - 1), im = at(g, i - 1, j);
        // curlE: x = Ez[j+1]-Ez, y = -(Ez[i+1]-Ez), z = (Ey[i+1]-Ey) - (Ex[j+1]-Ex)
        Ebar.z[c] += s * ((Bbar.x[jm] - Bbar.x[c]) + (Bbar.y[c] - Bbar.y[im]));
        Ebar.y[c] += s * (Bbar.z[im] - Bbar.z[c]);
        Ebar.x[c] += s * (Bbar.z[c] - Bbar.z[jm]);
    }
}

// Bbar += s * curlB^T(Ebar) (the adjoint of E += c curlB with s = c)
template <typename T>
__global__ void k_curlB_T(AG g, F3<T> Ebar, F3<T> Bbar, T s)
{
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c % g.nx, j = c / g.nx;
        const int jp = at(g, i, j + 1), ip = at(g, i + 1, j);
        // curlB: x = Bz - Bz[j-1], y = -(Bz - Bz[i-1]), z = (By - By[i-1]) - (Bx - Bx[j-1])
        Bbar.z[c] += s * ((Ebar.x[c] - Ebar.x[jp]) + (Ebar.y[ip] - Ebar.y[c]));
        Bbar.y[c] += s * (Ebar.z[c] - Ebar.z[ip]);
        Bbar.x[c] += s * (Ebar.z[jp] - Ebar.z[c]);
    }
}

template <typename T>
__global__ void k_axpy3(int n, F3<T> y, F3<T> x, T a)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        y.x[c] += a * x.x[c];
        y.y[c] += a * x.y[c];
        y.z[c] += a * x.z[c];
    }
}

// ---------------------------------------------------------------------------
// One particle's forward step with the intermediates its adjoint needs
// ---------------------------------------------------------------------------
template <typename T>
struct Mv {
    int ip0, jp0, kp0, ip, jp, kp;
    T dx, dy, wx[2], wy[2], V[4][6];
    T qm, q, pE[3], pB[3], a[3], gg, b[3], ff, t[3], s[3], U[3], G2;
    T x1, y1, z1, xr, yr, zr;
    bool xa, ya, za;   // relay point = midpoint (the particle stays in its cell along that axis)
    T F1[3], F2[3], W1[2], W2[2];
};

template <typename T>
__device__ __forceinline__ void node_values(const AG &g, const F3<T> &E, const F3<T> &B, int a, int b, T V[6])
{
    const int c = at(g, a, b), cxm = at(g, a - 1, b), cym = at(g, a, b - 1), cxym = at(g, a - 1, b - 1);
    V[0] = (E.x[cxm] + E.x[c]) * (T)0.5;
    V[1] = (E.y[cym] + E.y[c]) * (T)0.5;
    V[2] = E.z[c];
    V[3] = (B.x[cym] + B.x[c]) * (T)0.5 + (T)g.bext[0];
    V[4] = (B.y[cxm] + B.y[c]) * (T)0.5 + (T)g.bext[1];
    V[5] = (((B.z[cxym] + B.z[cxm]) + B.z[cym]) + B.z[c]) * (T)0.25 + (T)g.bext[2];
}

template <typename T>
__device__ __forceinline__ T relay(int i0, int i1, T mid, bool &active)
{
    const T lo = (T)max(i0, i1), hi = (T)(min(i0, i1) + 1);
    active = mid > lo && mid < hi;
    return fmin(hi, fmax(lo, mid));
}

// Frozen branches.  The step is piecewise smooth in the state: floor() of
// the start and end positions, the side the relay point's clamp takes and
// the periodic wrap are discrete decisions.  A forward run can record them
// per particle and step (one word each) and a later run replay them, which
// makes the replayed run a smooth function of its inputs whose derivative
// at the recorded state is the adjoint's (the derivative of the active
// branch): central differences of replayed runs check the adjoint without
// the jumps of the zigzag current.  Word: start cell x, y (20 bits each),
// end-cell offsets + 1, relay sides (0 lower bound, 1 midpoint, 2 upper
// bound), wrap shifts + 1 (2 bits each).
enum { kBranchFree = 0, kBranchRecord = 1, kBranchReplay = 2 };

struct Branch {
    int ip0, jp0, dip, djp, rx, ry, wx, wy;
};

__device__ __forceinline__ unsigned long long pack_branch(const Branch &b)
{
    return (unsigned long long)(unsigned)b.ip0 | ((unsigned long long)(unsigned)b.jp0 << 20) |
           ((unsigned long long)(b.dip + 1) << 40) | ((unsigned long long)(b.djp + 1) << 42) |
           ((unsigned long long)b.rx << 44) | ((unsigned long long)b.ry << 46) |
           ((unsigned long long)(b.wx + 1) << 48) | ((unsigned long long)(b.wy + 1) << 50);
}

__device__ __forceinline__ Branch unpack_branch(unsigned long long w)
{
    Branch b;
    b.ip0 = (int)(w & 0xfffffu);
    b.jp0 = (int)((w >> 20) & 0xfffffu);
    b.dip = (int)((w >> 40) & 3u) - 1;
    b.djp = (int)((w >> 42) & 3u) - 1;
    b.rx = (int)((w >> 44) & 3u);
    b.ry = (int)((w >> 46) & 3u);
    b.wx = (int)((w >> 48) & 3u) - 1;
    b.wy = (int)((w >> 50) & 3u) - 1;
    return b;
}

// The relay point on a given side of the clamp.
template <typename T>
__device__ __forceinline__ T relay_side(int i0, int i1, T mid, int side)
{
    return side == 0 ? (T)max(i0, i1) : (side == 2 ? (T)(min(i0, i1) + 1) : mid);
}
template <typename T>
__device__ __forceinline__ int relay_side_of(int i0, int i1, T mid)
{
    const T lo = (T)max(i0, i1), hi = (T)(min(i0, i1) + 1);
    return mid > lo ? (mid < hi ? 1 : 2) : 0;
}

template <typename T, int BR = kBranchFree>
__device__ void move_fwd(const AG &g, T x0, T y0, T z0, T u, T v, T w, T qthis, T qm, const F3<T> &E, const F3<T> &B,
                         Mv<T> &M, Branch *br = nullptr)
{
    M.ip0 = BR == kBranchReplay ? br->ip0 : (int)floor(x0);
    M.jp0 = BR == kBranchReplay ? br->jp0 : (int)floor(y0);
    M.kp0 = (int)floor(z0);
    M.dx = x0 - (T)M.ip0;
    M.dy = y0 - (T)M.jp0;
    M.wx[0] = (T)1 - M.dx;
    M.wx[1] = M.dx;
    M.wy[0] = (T)1 - M.dy;
    M.wy[1] = M.dy;
    T Ep[3] = {0, 0, 0}, Bp[3] = {0, 0, 0};
    for (int n = 0; n < 4; n++) {
        node_values<T>(g, E, B, M.ip0 + (n & 1), M.jp0 + (n >> 1), M.V[n]);
        const T wt = M.wx[n & 1] * M.wy[n >> 1];
        for (int k = 0; k < 3; k++) {
            Ep[k] = Ep[k] + wt * M.V[n][k];
            Bp[k] = Bp[k] + wt * M.V[n][3 + k];
        }
    }
    M.qm = qm;
    M.q = qthis;
    for (int k = 0; k < 3; k++) {
        M.pE[k] = Ep[k] * qm;
        M.pB[k] = Bp[k] * qm;
    }
    const T c = (T)g.c, sqc = (T)g.sqc, cinv = (T)g.cinv;
    M.a[0] = c * u + M.pE[0];
    M.a[1] = c * v + M.pE[1];
    M.a[2] = c * w + M.pE[2];
    M.gg = (T)1 / sqrt(((sqc + M.a[0] * M.a[0]) + M.a[1] * M.a[1]) + M.a[2] * M.a[2]);
    for (int k = 0; k < 3; k++) M.b[k] = M.gg * M.pB[k];
    M.ff = (T)2 / ((((T)1 + M.b[0] * M.b[0]) + M.b[1] * M.b[1]) + M.b[2] * M.b[2]);
    M.t[0] = (M.a[0] + M.a[1] * M.b[2]) - M.a[2] * M.b[1];
    M.t[1] = (M.a[1] + M.a[2] * M.b[0]) - M.a[0] * M.b[2];
    M.t[2] = (M.a[2] + M.a[0] * M.b[1]) - M.a[1] * M.b[0];
    for (int k = 0; k < 3; k++) M.s[k] = M.t[k] * M.ff;
    M.U[0] = ((M.a[0] + M.s[1] * M.b[2]) - M.s[2] * M.b[1]) + M.pE[0];
    M.U[1] = ((M.a[1] + M.s[2] * M.b[0]) - M.s[0] * M.b[2]) + M.pE[1];
    M.U[2] = ((M.a[2] + M.s[0] * M.b[1]) - M.s[1] * M.b[0]) + M.pE[2];
    M.G2 = ((sqc + M.U[0] * M.U[0]) + M.U[1] * M.U[1]) + M.U[2] * M.U[2];
    const T g2 = sqc / sqrt(M.G2);
    M.x1 = x0 + (M.U[0] * cinv) * g2;
    M.y1 = y0 + (M.U[1] * cinv) * g2;
    M.z1 = z0 + (M.U[2] * cinv) * g2;
    M.ip = BR == kBranchReplay ? M.ip0 + br->dip : (int)floor(M.x1);
    M.jp = BR == kBranchReplay ? M.jp0 + br->djp : (int)floor(M.y1);
    M.kp = (int)floor(M.z1);
    if (BR == kBranchReplay) {
        M.xr = relay_side<T>(M.ip0, M.ip, (T)0.5 * (x0 + M.x1), br->rx);
        M.yr = relay_side<T>(M.jp0, M.jp, (T)0.5 * (y0 + M.y1), br->ry);
        M.xa = br->rx == 1;
        M.ya = br->ry == 1;
    } else {
        M.xr = relay<T>(M.ip0, M.ip, (T)0.5 * (x0 + M.x1), M.xa);
        M.yr = relay<T>(M.jp0, M.jp, (T)0.5 * (y0 + M.y1), M.ya);
        if (BR == kBranchRecord) {
            br->ip0 = M.ip0;
            br->jp0 = M.jp0;
            br->dip = M.ip - M.ip0;
            br->djp = M.jp - M.jp0;
            br->rx = relay_side_of<T>(M.ip0, M.ip, (T)0.5 * (x0 + M.x1));
            br->ry = relay_side_of<T>(M.jp0, M.jp, (T)0.5 * (y0 + M.y1));
        }
    }
    // out-of-plane current: both segments carry half of the z displacement
    // (the midpoint relay of the FP32 form; continuous in z, unlike the z
    // relay of movdep.F90:185, which jumps when z crosses 1 or 2)
    M.zr = (T)0.5 * (z0 + M.z1);
    M.za = true;
    M.F1[0] = qthis * (M.xr - x0);
    M.F1[1] = qthis * (M.yr - y0);
    M.F1[2] = qthis * (M.zr - z0);
    M.F2[0] = qthis * (M.x1 - M.xr);
    M.F2[1] = qthis * (M.y1 - M.yr);
    M.F2[2] = qthis * (M.z1 - M.zr);
    M.W1[0] = (T)0.5 * (x0 + M.xr) - (T)M.ip0;
    M.W1[1] = (T)0.5 * (y0 + M.yr) - (T)M.jp0;
    M.W2[0] = (T)0.5 * (M.x1 + M.xr) - (T)M.ip;
    M.W2[1] = (T)0.5 * (M.y1 + M.yr) - (T)M.jp;
}

// 2D scatter of one segment into J (movdep_routines.F90:276-303)
template <typename T>
__device__ __forceinline__ void scatter_seg(const AG &g, F3<T> &J, int cx, int cy, const T F[3], const T W[2])
{
    const int c = at(g, cx, cy), cpx = at(g, cx + 1, cy), cpy = at(g, cx, cy + 1), cpxy = at(g, cx + 1, cy + 1);
    atomicAdd(J.x + c, F[0] * ((T)1 - W[1]));
    atomicAdd(J.x + cpy, F[0] * W[1]);
    atomicAdd(J.y + c, F[1] * ((T)1 - W[0]));
    atomicAdd(J.y + cpx, F[1] * W[0]);
    atomicAdd(J.z + c, (F[2] * ((T)1 - W[0])) * ((T)1 - W[1]));
    atomicAdd(J.z + cpx, (F[2] * W[0]) * ((T)1 - W[1]));
    atomicAdd(J.z + cpy, (F[2] * ((T)1 - W[0])) * W[1]);
    atomicAdd(J.z + cpxy, (F[2] * W[0]) * W[1]);
}

// Reverse of scatter_seg with Jbar: the cotangents of F and W.
template <typename T>
__device__ __forceinline__ void scatter_seg_T(const AG &g, const F3<T> &Jbar, T sgn, int cx, int cy, const T F[3],
                                              const T W[2], T Fb[3], T Wb[2])
{
    const int c = at(g, cx, cy), cpx = at(g, cx + 1, cy), cpy = at(g, cx, cy + 1), cpxy = at(g, cx + 1, cy + 1);
    const T jx0 = sgn * Jbar.x[c], jx1 = sgn * Jbar.x[cpy];
    const T jy0 = sgn * Jbar.y[c], jy1 = sgn * Jbar.y[cpx];
    const T z00 = sgn * Jbar.z[c], z10 = sgn * Jbar.z[cpx], z01 = sgn * Jbar.z[cpy], z11 = sgn * Jbar.z[cpxy];
    const T ox = (T)1 - W[0], oy = (T)1 - W[1];
    Fb[0] = jx0 * oy + jx1 * W[1];
    Fb[1] = jy0 * ox + jy1 * W[0];
    Fb[2] = z00 * ox * oy + z10 * W[0] * oy + z01 * ox * W[1] + z11 * W[0] * W[1];
    Wb[0] = F[1] * (jy1 - jy0) + F[2] * ((z10 - z00) * oy + (z11 - z01) * W[1]);
    Wb[1] = F[0] * (jx1 - jx0) + F[2] * ((z01 - z00) * ox + (z11 - z10) * W[0]);
}

template <typename T>
__device__ __forceinline__ T wrap_pos(T x, int n)
{
    if (x >= (T)n) x -= (T)n;
    else if (x < (T)0) x += (T)n;
    return x;
}

// Particle of work item L in the mover adjoint: the lanes of a warp take
// particles np/32 apart.  The loader writes particles cell by cell, so
// consecutive slots share cells and their 24 cotangent atomics would hit the
// same words; spread this way the lanes of a warp land in different cells.
// The particle state of this form is small enough to stay in L2, where the
// scattered loads hit.  (The forward mover, with fewer atomics per particle,
// is faster with coalesced loads.)
__device__ __forceinline__ long long spread_slot(long long L, long long q) { return (L & 31) * q + (L >> 5); }

// Shift of the periodic wrap of x in [-1, n + 1): -1 (x -= n), +1 or 0.
template <typename T>
__device__ __forceinline__ int wrap_shift(T x, int n)
{
    return x >= (T)n ? -1 : (x < (T)0 ? 1 : 0);
}

// Forward mover; BR: free, record the branches into tape[n] or replay them.
template <typename T, int BR>
__global__ void k_move(AG g, PS<T> p, const T *__restrict__ qw, const int *__restrict__ flv, long long np, F3<T> E,
                       F3<T> B, F3<T> J, unsigned long long *tape)
{
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < np; n += (long long)gridDim.x * blockDim.x) {
        Mv<T> M;
        Branch br;
        if (BR == kBranchReplay) br = unpack_branch(tape[n]);
        const T z0 = p.z[n];
        move_fwd<T, BR>(g, p.x[n], p.y[n], z0, p.u[n], p.v[n], p.w[n], qw[n] * (T)g.qi, (T)g.qm_half[flv[n]], E, B, M,
                        &br);
        scatter_seg<T>(g, J, M.ip0, M.jp0, M.F1, M.W1);
        scatter_seg<T>(g, J, M.ip, M.jp, M.F2, M.W2);
        const T cinv = (T)g.cinv;
        p.u[n] = M.U[0] * cinv;
        p.v[n] = M.U[1] * cinv;
        p.w[n] = M.U[2] * cinv;
        if (BR == kBranchFree) {
            p.x[n] = wrap_pos<T>(M.x1, g.nx);
            p.y[n] = wrap_pos<T>(M.y1, g.ny);
        } else {
            if (BR == kBranchRecord) {
                br.wx = wrap_shift<T>(M.x1, g.nx);
                br.wy = wrap_shift<T>(M.y1, g.ny);
                tape[n] = pack_branch(br);
            }
            p.x[n] = M.x1 + (T)(br.wx * g.nx);
            p.y[n] = M.y1 + (T)(br.wy * g.ny);
        }
        T zn = M.z1;   // movdep.F90:241-249 (zmin = 1, zmax = 2)
        if (zn > (T)2) zn = zn - (T)1;
        else if (zn < (T)1) zn = (T)1 + zn;
        p.z[n] = zn;
    }
}

// The mover's adjoint.  P is the tape's state at the start of the step, pb
// the cotangents of the particle after the step (replaced by those before),
// Ebt the cotangent of E after the step (J-bar = -Ebt); Nb (6 arrays: E x,
// y, z, B x, y, z) receives the gather's cotangents of the node-averaged
// fields, which k_node_T then takes back to the staggered E and B.
template <typename T>
__global__ void k_move_T(AG g, PS<T> P, const T *__restrict__ qw, const int *__restrict__ flv, long long np, F3<T> E,
                         F3<T> B, F3<T> Ebt, PS<T> pb, T *Nb)
{
    const size_t nc = (size_t)g.nx * g.ny;
    const T c = (T)g.c, cinv = (T)g.cinv;
    const long long q = (np + 31) >> 5;
    for (long long L = (long long)blockIdx.x * blockDim.x + threadIdx.x; L < 32 * q; L += (long long)gridDim.x * blockDim.x) {
        const long long n = spread_slot(L, q);
        if (n >= np) continue;
        Mv<T> M;
        const T x0 = P.x[n], y0 = P.y[n], z0 = P.z[n];
        move_fwd<T>(g, x0, y0, z0, P.u[n], P.v[n], P.w[n], qw[n] * (T)g.qi, (T)g.qm_half[flv[n]], E, B, M);
        // deposit
        T Fb1[3], Wb1[2], Fb2[3], Wb2[2];
        scatter_seg_T<T>(g, Ebt, (T)-1, M.ip0, M.jp0, M.F1, M.W1, Fb1, Wb1);
        scatter_seg_T<T>(g, Ebt, (T)-1, M.ip, M.jp, M.F2, M.W2, Fb2, Wb2);
        const T q = M.q;
        // position cotangents: output + deposit (x0, x1, relay points)
        T x0b = 0, y0b = 0, z0b = 0;
        T x1b = pb.x[n], y1b = pb.y[n], z1b = pb.z[n];
        T xrb = q * Fb1[0] - q * Fb2[0] + (T)0.5 * Wb1[0] + (T)0.5 * Wb2[0];
        T yrb = q * Fb1[1] - q * Fb2[1] + (T)0.5 * Wb1[1] + (T)0.5 * Wb2[1];
        T zrb = q * Fb1[2] - q * Fb2[2];
        x0b += -q * Fb1[0] + (T)0.5 * Wb1[0];
        y0b += -q * Fb1[1] + (T)0.5 * Wb1[1];
        z0b += -q * Fb1[2];
        x1b += q * Fb2[0] + (T)0.5 * Wb2[0];
        y1b += q * Fb2[1] + (T)0.5 * Wb2[1];
        z1b += q * Fb2[2];
        if (M.xa) { x0b += (T)0.5 * xrb; x1b += (T)0.5 * xrb; }
        if (M.ya) { y0b += (T)0.5 * yrb; y1b += (T)0.5 * yrb; }
        if (M.za) { z0b += (T)0.5 * zrb; z1b += (T)0.5 * zrb; }
        // x1 = x0 + d
        x0b += x1b;
        y0b += y1b;
        z0b += z1b;
        const T db[3] = {x1b, y1b, z1b};
        // d = c U / sqrt(G2), u_out = U / c
        const T rs = (T)1 / sqrt(M.G2), rs3 = rs * rs * rs;
        const T Ud = M.U[0] * db[0] + M.U[1] * db[1] + M.U[2] * db[2];
        T Ub[3];
        const T uob[3] = {pb.u[n], pb.v[n], pb.w[n]};
        for (int k = 0; k < 3; k++) Ub[k] = c * (rs * db[k] - rs3 * M.U[k] * Ud) + uob[k] * cinv;
        // U = a + s x b + pE
        T ab[3], pEb[3], pBb[3] = {0, 0, 0}, bb[3], sb[3];
        for (int k = 0; k < 3; k++) {
            ab[k] = Ub[k];
            pEb[k] = Ub[k];
        }
        sb[0] = M.b[1] * Ub[2] - M.b[2] * Ub[1];   // b x Ub
        sb[1] = M.b[2] * Ub[0] - M.b[0] * Ub[2];
        sb[2] = M.b[0] * Ub[1] - M.b[1] * Ub[0];
        bb[0] = Ub[1] * M.s[2] - Ub[2] * M.s[1];   // Ub x s
        bb[1] = Ub[2] * M.s[0] - Ub[0] * M.s[2];
        bb[2] = Ub[0] * M.s[1] - Ub[1] * M.s[0];
        // s = ff t
        T tb[3];
        for (int k = 0; k < 3; k++) tb[k] = M.ff * sb[k];
        const T ffb = sb[0] * M.t[0] + sb[1] * M.t[1] + sb[2] * M.t[2];
        // ff = 2 / D, D = 1 + |b|^2
        const T Db = -(M.ff * M.ff * (T)0.5) * ffb;
        for (int k = 0; k < 3; k++) bb[k] += (T)2 * M.b[k] * Db;
        // t = a + a x b
        for (int k = 0; k < 3; k++) ab[k] += tb[k];
        ab[0] += M.b[1] * tb[2] - M.b[2] * tb[1];   // b x tb
        ab[1] += M.b[2] * tb[0] - M.b[0] * tb[2];
        ab[2] += M.b[0] * tb[1] - M.b[1] * tb[0];
        bb[0] += tb[1] * M.a[2] - tb[2] * M.a[1];   // tb x a
        bb[1] += tb[2] * M.a[0] - tb[0] * M.a[2];
        bb[2] += tb[0] * M.a[1] - tb[1] * M.a[0];
        // b = gg pB, gg = G^-1/2, G = c^2 + |a|^2
        T ggb = 0;
        for (int k = 0; k < 3; k++) {
            pBb[k] += M.gg * bb[k];
            ggb += bb[k] * M.pB[k];
        }
        const T Gb = (T)-0.5 * M.gg * M.gg * M.gg * ggb;
        for (int k = 0; k < 3; k++) ab[k] += (T)2 * M.a[k] * Gb;
        // a = c u + pE
        pb.u[n] = c * ab[0];
        pb.v[n] = c * ab[1];
        pb.w[n] = c * ab[2];
        for (int k = 0; k < 3; k++) pEb[k] += ab[k];
        // gather: pE = qm Ep, Ep = sum wt V
        T Epb[3], Bpb[3];
        for (int k = 0; k < 3; k++) {
            Epb[k] = M.qm * pEb[k];
            Bpb[k] = M.qm * pBb[k];
        }
        T wxb[2] = {0, 0}, wyb[2] = {0, 0};
        for (int nn = 0; nn < 4; nn++) {
            const int ax = nn & 1, ay = nn >> 1;
            const T wt = M.wx[ax] * M.wy[ay];
            T wtb = 0;
            for (int k = 0; k < 3; k++) wtb += M.V[nn][k] * Epb[k] + M.V[nn][3 + k] * Bpb[k];
            wxb[ax] += wtb * M.wy[ay];
            wyb[ay] += wtb * M.wx[ax];
            // cotangents of the node values (node averaging undone by k_node_T)
            const size_t cc = (size_t)at(g, M.ip0 + ax, M.jp0 + ay);
#pragma unroll
            for (int k = 0; k < 3; k++) {
                atomicAdd(Nb + k * nc + cc, wt * Epb[k]);
                atomicAdd(Nb + (3 + k) * nc + cc, wt * Bpb[k]);
            }
        }
        x0b += wxb[1] - wxb[0];
        y0b += wyb[1] - wyb[0];
        pb.x[n] = x0b;
        pb.y[n] = y0b;
        pb.z[n] = z0b;
    }
}

// Adjoint of the node averaging (movdep_routines.F90:6-223 in 2D: E x and B y
// averaged over the cells at x-1 and x, E y and B x over y-1 and y, B z over
// the four cells around the node): Eb, Bb += the node cotangents Nb taken
// back to the staggered components.
template <typename T>
__global__ void k_node_T(AG g, const T *__restrict__ Nb, F3<T> Eb, F3<T> Bb)
{
    const int n = g.nx * g.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int i = c % g.nx, j = c / g.nx;
        const int cx = at(g, i + 1, j), cy = at(g, i, j + 1), cxy = at(g, i + 1, j + 1);
        const T *N0 = Nb, *N1 = Nb + n, *N2 = Nb + 2 * n, *N3 = Nb + 3 * n, *N4 = Nb + 4 * n, *N5 = Nb + 5 * n;
        Eb.x[c] += (T)0.5 * (N0[c] + N0[cx]);
        Eb.y[c] += (T)0.5 * (N1[c] + N1[cy]);
        Eb.z[c] += N2[c];
        Bb.x[c] += (T)0.5 * (N3[c] + N3[cy]);
        Bb.y[c] += (T)0.5 * (N4[c] + N4[cx]);
        Bb.z[c] += (T)0.25 * (((N5[c] + N5[cx]) + N5[cy]) + N5[cxy]);
    }
}

// Gradient w.r.t. the loader's drift D and per-flavour temperatures: the
// closed-form Jacobian of AddDriftVel (a boost along x by vx = sgn D,
// prob_dist.F90:223-254) and of the Maxwell momentum sqrt(X T)
// (prob_dist.F90:13-30) applied to the cotangents of the initial momenta.
template <typename T>
__global__ void k_param_grad(PS<T> p0, const double *__restrict__ sgn, const int *__restrict__ flv, long long np,
                             PS<T> pb, double drift, const double *__restrict__ temp, double *out)
{
    __shared__ double red[3][8];
    double gD = 0, gT[2] = {0, 0};
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < np; n += (long long)gridDim.x * blockDim.x) {
        const double s = sgn[n], vx = s * drift;
        const double uf = p0.u[n], vf = p0.v[n], wf = p0.w[n];
        const double gf = sqrt(1.0 + uf * uf + vf * vf + wf * wf);
        const double gd = 1.0 / sqrt((1.0 - vx) * (1.0 + vx));
        const double ur = gd * (uf - vx * gf), vr = vf, wr = wf;
        const double gr = sqrt(1.0 + ur * ur + vr * vr + wr * wr);
        const double ub = pb.u[n], vb = pb.v[n], wb = pb.w[n];
        gD += ub * s * (gd * gd * vx * uf + gd * gr);
        const int sp = flv[n] - 1;
        const double Tsp = temp[sp];
        if (Tsp > 0 && (sp == 0 || sp == 1)) {
            const double k = gr * gr / (2.0 * Tsp);
            const double dur = ur * k, dvr = vr * k, dwr = wr * k;
            const double dgr = (ur * ur + vr * vr + wr * wr) * gr / (2.0 * Tsp);
            gT[sp] += ub * gd * (dur + vx * dgr) + vb * dvr + wb * dwr;
        }
    }
    double v3[3] = {gD, gT[0], gT[1]};
    for (int k = 0; k < 3; k++) {
        for (int o = 16; o > 0; o >>= 1) v3[k] += __shfl_down_sync(0xffffffffu, v3[k], o);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v3[k];
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[threadIdx.x][w];
        atomicAdd(out + threadIdx.x, t);
    }
}

// reference layout (ghosted, 1-based) <-> interior coordinates
template <typename T>
__global__ void k_from_ref(PartF64 in, long long np, PS<T> out, double *qout, int *fout, const double *sgn_in,
                           double *sgn_out)
{
    for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < np; n += (long long)gridDim.x * blockDim.x) {
        out.x[n] = (T)(in.x[n] - 3.0);
        out.y[n] = (T)(in.y[n] - 3.0);
        out.z[n] = (T)in.z[n];
        out.u[n] = (T)in.u[n];
        out.v[n] = (T)in.v[n];
        out.w[n] = (T)in.w[n];
        qout[n] = in.q[n];
        fout[n] = in.flv[n];
        sgn_out[n] = sgn_in ? sgn_in[n] : 0.0;
    }
}

template <typename T>
__global__ void k_to_double(const T *in, double *out, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

template <typename T>
__global__ void k_qcast(const double *in, T *out, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (T)in[i];
}

}  // namespace adj
}  // namespace pic

using namespace pic;
using namespace pic::adj;

// ---------------------------------------------------------------------------
// The engine
// ---------------------------------------------------------------------------
struct pic_adjoint {
    pic_config cfg;
    AG g = {};
    bool fp32 = false;
    cudaStream_t s = nullptr;
    long long cap = 0, np = 0;
    size_t tsz = 8;                 // sizeof(T)
    std::vector<void *> allocs;
    // particles: initial state, current state, cotangents (x, y, z, u, v, w)
    void *p0[6] = {}, *p[6] = {}, *pb[6] = {};
    void *qw = nullptr;             // weights (T)
    double *q64 = nullptr, *sgn = nullptr;
    int *flv = nullptr;
    // fields: E, B, J, scratch B_a, B_t, cotangents Ebar (2), Bbar; initial E, B
    void *E[3] = {}, *B[3] = {}, *J[3] = {}, *Ba[3] = {}, *Bt[3] = {}, *Ebar[2][3] = {}, *Bbar[3] = {};
    void *E0[3] = {}, *B0[3] = {};
    void *Nb = nullptr;               // node cotangents of the gather (6 planes)
    // the forward run and the reverse sweep captured as CUDA graphs, rebuilt
    // when the step count, the checkpoint interval or the particle count change
    cudaGraphExec_t gf = nullptr, gb = nullptr;
    long long gf_key[4] = {-1, -1, -1, -1}, gb_key[4] = {-1, -1, -1, -1};
    // frozen branches of the forward mover (record / replay), one word per
    // particle and step of the recorded run
    int br_mode = 0;
    unsigned long long *br_tape = nullptr;
    long long br_words = 0, br_np = 0, br_steps = 0;
    // checkpoints (every K steps) and the tape of one segment
    int K = 0, T = 0, tapeK = 0;
    std::vector<void *> ck_p, ck_f;   // per checkpoint: 6 particle arrays / 6 field arrays
    void *tape_p = nullptr, *tape_f = nullptr;
    double *acc = nullptr;            // objective, then 3 parameter gradients
    pic_handle *loader = nullptr;     // FP64 handle whose Weibel loader fills the initial state
};

namespace {

int cstat(cudaError_t e) { return e == cudaSuccess ? PIC_OK : (e == cudaErrorMemoryAllocation ? PIC_ERR_OOM : PIC_ERR_CUDA); }
#define ACK(x)                                  \
    do {                                        \
        cudaError_t e_ = (x);                   \
        if (e_ != cudaSuccess) return cstat(e_); \
    } while (0)

int aalloc(pic_adjoint *a, void **p, size_t bytes)
{
    ACK(cudaMalloc(p, bytes ? bytes : 1));
    a->allocs.push_back(*p);
    return PIC_OK;
}

unsigned grid_of(long long n)
{
    long long b = (n + 255) / 256;
    if (b > (long long)kSMs * 16) b = (long long)kSMs * 16;
    return (unsigned)(b < 1 ? 1 : b);
}

size_t cells(const pic_adjoint *a) { return (size_t)a->g.nx * a->g.ny; }

template <typename T>
F3<T> f3(void *const v[3])
{
    return F3<T>{(T *)v[0], (T *)v[1], (T *)v[2]};
}
template <typename T>
PS<T> ps(void *const v[6])
{
    return PS<T>{(T *)v[0], (T *)v[1], (T *)v[2], (T *)v[3], (T *)v[4], (T *)v[5]};
}
template <typename T>
F3<T> f3_at(void *base, size_t ncell, int k)   // k-th triple of a packed field block
{
    T *b = (T *)base + (size_t)k * 3 * ncell;
    return F3<T>{b, b + ncell, b + 2 * ncell};
}
template <typename T>
PS<T> ps_at(void *base, size_t np)
{
    T *b = (T *)base;
    return PS<T>{b, b + np, b + 2 * np, b + 3 * np, b + 4 * np, b + 5 * np};
}

// state <- (particles, E, B) of a packed block (or the reverse)
template <typename T>
int copy_state(pic_adjoint *a, void *pdst[6], void *Edst[3], void *Bdst[3], PS<T> psrc, F3<T> Esrc, F3<T> Bsrc)
{
    const size_t pn = (size_t)a->np * sizeof(T), fn = cells(a) * sizeof(T);
    T *src_p[6] = {psrc.x, psrc.y, psrc.z, psrc.u, psrc.v, psrc.w};
    for (int k = 0; k < 6; k++) ACK(cudaMemcpyAsync(pdst[k], src_p[k], pn, cudaMemcpyDeviceToDevice, a->s));
    T *se[3] = {Esrc.x, Esrc.y, Esrc.z}, *sb[3] = {Bsrc.x, Bsrc.y, Bsrc.z};
    for (int k = 0; k < 3; k++) {
        ACK(cudaMemcpyAsync(Edst[k], se[k], fn, cudaMemcpyDeviceToDevice, a->s));
        ACK(cudaMemcpyAsync(Bdst[k], sb[k], fn, cudaMemcpyDeviceToDevice, a->s));
    }
    return PIC_OK;
}

// Packed blocks hold 6 particle arrays of stride cap, then E and B.
template <typename T>
int save_state(pic_adjoint *a, void *pbase, void *fbase)
{
    PS<T> d = ps_at<T>(pbase, (size_t)a->cap);
    F3<T> e = f3_at<T>(fbase, cells(a), 0), b = f3_at<T>(fbase, cells(a), 1);
    const size_t pn = (size_t)a->np * sizeof(T), fn = cells(a) * sizeof(T);
    T *dp[6] = {d.x, d.y, d.z, d.u, d.v, d.w};
    for (int k = 0; k < 6; k++) ACK(cudaMemcpyAsync(dp[k], a->p[k], pn, cudaMemcpyDeviceToDevice, a->s));
    T *de[3] = {e.x, e.y, e.z}, *db[3] = {b.x, b.y, b.z};
    for (int k = 0; k < 3; k++) {
        ACK(cudaMemcpyAsync(de[k], a->E[k], fn, cudaMemcpyDeviceToDevice, a->s));
        ACK(cudaMemcpyAsync(db[k], a->B[k], fn, cudaMemcpyDeviceToDevice, a->s));
    }
    return PIC_OK;
}

template <typename T>
int restore_state(pic_adjoint *a, void *pbase, void *fbase)
{
    return copy_state<T>(a, a->p, a->E, a->B, ps_at<T>(pbase, (size_t)a->cap), f3_at<T>(fbase, cells(a), 0),
                         f3_at<T>(fbase, cells(a), 1));
}

// One forward step on the current state; obj accumulates 1/2 |B_t|^2.
template <typename T>
void step_fwd(pic_adjoint *a, bool obj, int t)
{
    const AG &g = a->g;
    const unsigned gc = grid_of((long long)cells(a)), gp = grid_of(a->np);
    F3<T> E = f3<T>(a->E), B = f3<T>(a->B), J = f3<T>(a->J);
    k_bhalf<T><<<gc, 256, 0, a->s>>>(g, E, B, B);
    unsigned long long *tape = t >= 0 && a->br_mode != kBranchFree ? a->br_tape + (size_t)t * (size_t)a->np : nullptr;
    if (tape && a->br_mode == kBranchRecord)
        k_move<T, kBranchRecord><<<gp, 256, 0, a->s>>>(g, ps<T>(a->p), (const T *)a->qw, a->flv, a->np, E, B, J, tape);
    else if (tape)
        k_move<T, kBranchReplay><<<gp, 256, 0, a->s>>>(g, ps<T>(a->p), (const T *)a->qw, a->flv, a->np, E, B, J, tape);
    else
        k_move<T, kBranchFree><<<gp, 256, 0, a->s>>>(g, ps<T>(a->p), (const T *)a->qw, a->flv, a->np, E, B, J, nullptr);
    k_bhalf<T><<<gc, 256, 0, a->s>>>(g, E, B, B);
    k_efield<T><<<gc, 256, 0, a->s>>>(g, E, B, J);
    if (obj) k_benergy<T><<<gc, 256, 0, a->s>>>(g, B, a->acc);
    count_launches(obj ? 5 : 4);
}

// Reverse of step t from the tape entry (state at the start of the step).
template <typename T>
void step_rev(pic_adjoint *a, PS<T> P, F3<T> E, F3<T> B, int &cur)
{
    const AG &g = a->g;
    const unsigned gc = grid_of((long long)cells(a)), gp = grid_of(a->np);
    const size_t fn = cells(a) * sizeof(T);
    F3<T> Ba = f3<T>(a->Ba), Bt = f3<T>(a->Bt), Bb = f3<T>(a->Bbar);
    F3<T> Ebt = f3<T>(a->Ebar[cur]), Ebp = f3<T>(a->Ebar[cur ^ 1]);
    k_bhalf<T><<<gc, 256, 0, a->s>>>(g, E, B, Ba);
    k_bhalf<T><<<gc, 256, 0, a->s>>>(g, E, Ba, Bt);
    k_axpy3<T><<<gc, 256, 0, a->s>>>((int)cells(a), Bb, Bt, (T)1);                  // objective
    k_curlB_T<T><<<gc, 256, 0, a->s>>>(g, Ebt, Bb, (T)g.fc);                        // E_t = E + c curlB(B_t) - J
    for (int k = 0; k < 3; k++) cudaMemcpyAsync(a->Ebar[cur ^ 1][k], a->Ebar[cur][k], fn, cudaMemcpyDeviceToDevice, a->s);
    k_curlE_T<T><<<gc, 256, 0, a->s>>>(g, Bb, Ebp, (T)-g.h);                        // second half step
    cudaMemsetAsync(a->Nb, 0, 6 * fn, a->s);
    k_move_T<T><<<gp, 256, 0, a->s>>>(g, P, (const T *)a->qw, a->flv, a->np, E, Ba, Ebt, ps<T>(a->pb), (T *)a->Nb);
    k_node_T<T><<<gc, 256, 0, a->s>>>(g, (const T *)a->Nb, Ebp, Bb);
    k_curlE_T<T><<<gc, 256, 0, a->s>>>(g, Bb, Ebp, (T)-g.h);                        // first half step
    count_launches(8);
    cur ^= 1;
}

// Launch the graph cached in *ge for key, or capture enqueue() on a->s into
// a new one first.
template <typename F>
int launch_cached(pic_adjoint *a, cudaGraphExec_t *ge, long long *cached, const long long key[4], F enqueue)
{
    if (!*ge || cached[0] != key[0] || cached[1] != key[1] || cached[2] != key[2] || cached[3] != key[3]) {
        if (*ge) {
            cudaGraphExecDestroy(*ge);
            *ge = nullptr;
        }
        ACK(cudaStreamBeginCapture(a->s, cudaStreamCaptureModeThreadLocal));
        const int r = enqueue();
        cudaGraph_t gr = nullptr;
        const cudaError_t e = cudaStreamEndCapture(a->s, &gr);
        if (r || e != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            cudaGetLastError();
            return r ? r : cstat(e);
        }
        const cudaError_t ei = cudaGraphInstantiate(ge, gr, 0);
        cudaGraphDestroy(gr);
        if (ei != cudaSuccess) {
            *ge = nullptr;
            return cstat(ei);
        }
        for (int k = 0; k < 4; k++) cached[k] = key[k];
    }
    ACK(cudaGraphLaunch(*ge, a->s));
    return PIC_OK;
}

template <typename T>
int enqueue_forward(pic_adjoint *a, int nsteps, int K)
{
    // fresh state from the initial particles and fields
    const size_t pn = (size_t)a->np * sizeof(T), fn = cells(a) * sizeof(T);
    for (int k = 0; k < 6; k++) ACK(cudaMemcpyAsync(a->p[k], a->p0[k], pn, cudaMemcpyDeviceToDevice, a->s));
    for (int k = 0; k < 3; k++) {
        ACK(cudaMemcpyAsync(a->E[k], a->E0[k], fn, cudaMemcpyDeviceToDevice, a->s));
        ACK(cudaMemcpyAsync(a->B[k], a->B0[k], fn, cudaMemcpyDeviceToDevice, a->s));
        ACK(cudaMemsetAsync(a->J[k], 0, fn, a->s));
    }
    ACK(cudaMemsetAsync(a->acc, 0, 4 * sizeof(double), a->s));
    for (int t = 0; t < nsteps; t++) {
        if (t % K == 0) {
            int r = save_state<T>(a, a->ck_p[t / K], a->ck_f[t / K]);
            if (r) return r;
        }
        step_fwd<T>(a, true, t);
    }
    ACK(cudaGetLastError());
    return PIC_OK;
}

template <typename T>
int run_forward(pic_adjoint *a, int nsteps, int K, double *objective)
{
    const int nck = (nsteps + K - 1) / K;
    // checkpoint storage (kept between calls)
    for (int c = (int)a->ck_p.size(); c < nck; c++) {
        void *pp = nullptr, *ff = nullptr;
        int r;
        if ((r = aalloc(a, &pp, 6 * (size_t)a->cap * sizeof(T))) || (r = aalloc(a, &ff, 6 * cells(a) * sizeof(T))))
            return r;
        a->ck_p.push_back(pp);
        a->ck_f.push_back(ff);
    }
    if (a->br_mode == kBranchReplay && (a->br_np != a->np || a->br_steps < nsteps)) return PIC_ERR_INVALID;
    if (a->br_mode == kBranchRecord && a->br_words < (long long)nsteps * a->np) {
        if (a->br_tape) {
            cudaFree(a->br_tape);
            a->allocs.erase(std::find(a->allocs.begin(), a->allocs.end(), (void *)a->br_tape));
            a->br_tape = nullptr;
        }
        a->br_words = 0;
        int q = aalloc(a, (void **)&a->br_tape, (size_t)nsteps * (size_t)a->np * sizeof(unsigned long long));
        if (q) return q;
        a->br_words = (long long)nsteps * a->np;
        if (a->gf) {   // captured with the old tape
            cudaGraphExecDestroy(a->gf);
            a->gf = nullptr;
        }
    }
    const long long key[4] = {nsteps, K, a->np, a->br_mode};
    int r = launch_cached(a, &a->gf, a->gf_key, key, [&] { return enqueue_forward<T>(a, nsteps, K); });
    if (r) return r;
    ACK(cudaMemcpyAsync(objective, a->acc, sizeof(double), cudaMemcpyDeviceToHost, a->s));
    ACK(cudaStreamSynchronize(a->s));
    a->K = K;
    a->T = nsteps;
    if (a->br_mode == kBranchRecord) {
        a->br_np = a->np;
        a->br_steps = nsteps;
    }
    return PIC_OK;
}

// The tape holds one segment of K steps (allocated outside any capture).
template <typename T>
int ensure_tape(pic_adjoint *a)
{
    const int K = a->K;
    if (K <= a->tapeK) return PIC_OK;
    for (void *t : {a->tape_p, a->tape_f}) {
        if (!t) continue;
        cudaFree(t);
        a->allocs.erase(std::find(a->allocs.begin(), a->allocs.end(), t));
    }
    a->tape_p = a->tape_f = nullptr;
    if (a->gb) {   // the cached sweep refers to the old tape
        cudaGraphExecDestroy(a->gb);
        a->gb = nullptr;
    }
    int r;
    if ((r = aalloc(a, &a->tape_p, (size_t)K * 6 * (size_t)a->cap * sizeof(T))) ||
        (r = aalloc(a, &a->tape_f, (size_t)K * 6 * cells(a) * sizeof(T))))
        return r;
    a->tapeK = K;
    return PIC_OK;
}

template <typename T>
int enqueue_backward(pic_adjoint *a)
{
    const size_t pn = (size_t)a->np * sizeof(T), fn = cells(a) * sizeof(T);
    const int K = a->K, nsteps = a->T;
    for (int k = 0; k < 6; k++) ACK(cudaMemsetAsync(a->pb[k], 0, pn, a->s));
    for (int k = 0; k < 3; k++) {
        ACK(cudaMemsetAsync(a->Ebar[0][k], 0, fn, a->s));
        ACK(cudaMemsetAsync(a->Ebar[1][k], 0, fn, a->s));
        ACK(cudaMemsetAsync(a->Bbar[k], 0, fn, a->s));
    }
    int cur = 0;
    for (int seg = (nsteps - 1) / K; seg >= 0; seg--) {
        const int t0 = seg * K, t1 = std::min(nsteps, t0 + K);
        int r = restore_state<T>(a, a->ck_p[seg], a->ck_f[seg]);
        if (r) return r;
        for (int k = 0; k < 3; k++) ACK(cudaMemsetAsync(a->J[k], 0, fn, a->s));
        for (int t = t0; t < t1; t++) {
            const int s = t - t0;
            if ((r = save_state<T>(a, (char *)a->tape_p + (size_t)s * 6 * a->cap * sizeof(T),
                                   (char *)a->tape_f + (size_t)s * 6 * cells(a) * sizeof(T))))
                return r;
            step_fwd<T>(a, false, -1);
        }
        for (int t = t1 - 1; t >= t0; t--) {
            const int s = t - t0;
            void *pbase = (char *)a->tape_p + (size_t)s * 6 * a->cap * sizeof(T);
            void *fbase = (char *)a->tape_f + (size_t)s * 6 * cells(a) * sizeof(T);
            step_rev<T>(a, ps_at<T>(pbase, (size_t)a->cap), f3_at<T>(fbase, cells(a), 0), f3_at<T>(fbase, cells(a), 1),
                        cur);
        }
    }
    ACK(cudaGetLastError());
    return PIC_OK;
}

// The reverse sweep of the last forward run; the particle cotangents are of
// the initial state afterwards.
template <typename T>
int run_backward(pic_adjoint *a)
{
    int r = ensure_tape<T>(a);
    if (r) return r;
    const long long key[4] = {a->T, a->K, a->np, 0};
    if ((r = launch_cached(a, &a->gb, a->gb_key, key, [&] { return enqueue_backward<T>(a); }))) return r;
    ACK(cudaStreamSynchronize(a->s));
    return PIC_OK;
}

}  // namespace

extern "C" {

int pic_adj_create(const pic_config *cfg, pic_adjoint **out)
{
    if (!cfg || !out) return PIC_ERR_INVALID;
    *out = nullptr;
    const pic_config &c = *cfg;
    if (c.dims != 2 || c.geom != PIC_GEOM_CARTESIAN || c.fdtd != PIC_FDTD_YEE || c.curr_filter != 0 ||
        (c.precision != PIC_PREC_FP64 && c.precision != PIC_PREC_FP32) || c.nx < 4 || c.ny < 4 || c.nflvr < 1 ||
        c.nflvr > PIC_MAX_FLVR || !(c.c > 0.0 && c.c < 1.0) || c.capacity < 1 || c.capacity >= (1ll << 31))
        return PIC_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return PIC_ERR_NOGPU;
    }
    pic_adjoint *a = new pic_adjoint();
    a->cfg = c;
    a->fp32 = c.precision == PIC_PREC_FP32;
    a->tsz = a->fp32 ? sizeof(float) : sizeof(double);
    AG &g = a->g;
    g.nx = c.nx;
    g.ny = c.ny;
    g.c = c.c;
    g.h = (c.c * 0.5) * 1.0;
    g.fc = c.c * 1.0;
    g.sqc = c.c * c.c;
    g.cinv = 1.0 / c.c;
    g.qi = c.qi;
    for (int d = 0; d < 3; d++) g.bext[d] = c.bext[d];
    g.qm_half[0] = 0.0;
    for (int f = 1; f <= PIC_MAX_FLVR; f++) g.qm_half[f] = (f <= c.nflvr ? c.qm[f] : 0.0) * 0.5;
    a->cap = c.capacity;
    int r = PIC_OK;
    if (cudaStreamCreateWithFlags(&a->s, cudaStreamNonBlocking) != cudaSuccess) r = PIC_ERR_CUDA;
    const size_t pn = (size_t)a->cap * a->tsz, fn = cells(a) * a->tsz;
    for (int k = 0; k < 6 && !r; k++)
        if ((r = aalloc(a, &a->p0[k], pn)) || (r = aalloc(a, &a->p[k], pn)) || (r = aalloc(a, &a->pb[k], pn))) break;
    if (!r) r = aalloc(a, &a->qw, pn);
    if (!r) r = aalloc(a, (void **)&a->q64, (size_t)a->cap * sizeof(double));
    if (!r) r = aalloc(a, (void **)&a->sgn, (size_t)a->cap * sizeof(double));
    if (!r) r = aalloc(a, (void **)&a->flv, (size_t)a->cap * sizeof(int));
    void **fl[] = {a->E, a->B, a->J, a->Ba, a->Bt, a->Ebar[0], a->Ebar[1], a->Bbar, a->E0, a->B0};
    for (void **f : fl)
        for (int k = 0; k < 3 && !r; k++) {
            if ((r = aalloc(a, &f[k], fn))) break;
            if (cudaMemset(f[k], 0, fn) != cudaSuccess) r = PIC_ERR_CUDA;
        }
    if (!r) r = aalloc(a, &a->Nb, 6 * fn);
    if (!r && cudaMemset(a->Nb, 0, 6 * fn) != cudaSuccess) r = PIC_ERR_CUDA;
    if (!r) r = aalloc(a, (void **)&a->acc, 4 * sizeof(double));
    if (r) {
        pic_adj_destroy(a);
        return r;
    }
    *out = a;
    return PIC_OK;
}

void pic_adj_destroy(pic_adjoint *a)
{
    if (!a) return;
    if (a->s) cudaStreamSynchronize(a->s);
    if (a->gf) cudaGraphExecDestroy(a->gf);
    if (a->gb) cudaGraphExecDestroy(a->gb);
    for (void *p : a->allocs) cudaFree(p);
    if (a->loader) pic_destroy(a->loader);
    if (a->s) cudaStreamDestroy(a->s);
    delete a;
}

static int adopt_ref(pic_adjoint *a, const PartF64 &src, long long n, const double *sgn_dev)
{
    if (n > a->cap) return PIC_ERR_OVERFLOW;
    a->np = n;
    if (n == 0) return PIC_OK;
    if (a->fp32) {
        k_from_ref<float><<<grid_of(n), 256, 0, a->s>>>(src, n, ps<float>(a->p0), a->q64, a->flv, sgn_dev, a->sgn);
        k_qcast<float><<<grid_of(n), 256, 0, a->s>>>(a->q64, (float *)a->qw, n);
    } else {
        k_from_ref<double><<<grid_of(n), 256, 0, a->s>>>(src, n, ps<double>(a->p0), a->q64, a->flv, sgn_dev, a->sgn);
        k_qcast<double><<<grid_of(n), 256, 0, a->s>>>(a->q64, (double *)a->qw, n);
    }
    count_launches(2);
    ACK(cudaGetLastError());
    ACK(cudaStreamSynchronize(a->s));
    return PIC_OK;
}

int pic_adj_init_weibel(pic_adjoint *a, double epc, double density, double drift, double temp_ion, double temp_elc,
                        uint32_t seed, int64_t *n)
{
    if (!a || a->cfg.nflvr < 2) return PIC_ERR_INVALID;
    if (!a->loader) {
        pic_config c = a->cfg;
        c.precision = PIC_PREC_FP64;
        c.reorder_period = 0;
        c.brick[0] = c.brick[1] = c.brick[2] = 0;
        int r = pic_create(&c, &a->loader);
        if (r) return r;
    }
    PartF64 view;
    long long cnt = 0;
    // the signs land in a->sgn in loader slot order, the order adopt_ref keeps
    int r = weibel_with_signs(a->loader, epc, density, drift, temp_ion, temp_elc, seed, a->sgn, &view, &cnt);
    if (r) return r;
    r = adopt_ref(a, view, cnt, a->sgn);
    if (n) *n = cnt;
    return r;
}

int pic_adj_load_particles(pic_adjoint *a, int64_t n, const double *q, const double *x, const double *y,
                           const double *z, const double *u, const double *v, const double *w, const int32_t *flv,
                           const double *drift_sign)
{
    if (!a || n < 0 || n > a->cap || (n > 0 && (!q || !x || !y || !z || !u || !v || !w || !flv))) return PIC_ERR_INVALID;
    // stage through a temporary FP64 reference-layout block
    std::vector<void *> tmp;
    PartF64 d;
    double *blk = nullptr, *sg = nullptr;
    const size_t m = (size_t)(n > 0 ? n : 1);
    ACK(cudaMalloc((void **)&blk, m * (7 * sizeof(double) + sizeof(int32_t))));
    if (drift_sign && cudaMalloc((void **)&sg, m * sizeof(double)) != cudaSuccess) {
        cudaFree(blk);
        return PIC_ERR_OOM;
    }
    d.q = blk; d.x = blk + m; d.y = blk + 2 * m; d.z = blk + 3 * m; d.u = blk + 4 * m; d.v = blk + 5 * m; d.w = blk + 6 * m;
    d.flv = (int32_t *)(blk + 7 * m);
    const double *src[7] = {q, x, y, z, u, v, w};
    double *dst[7] = {d.q, d.x, d.y, d.z, d.u, d.v, d.w};
    int r = PIC_OK;
    for (int k = 0; k < 7 && n; k++)
        if (cudaMemcpyAsync(dst[k], src[k], (size_t)n * sizeof(double), cudaMemcpyHostToDevice, a->s) != cudaSuccess)
            r = PIC_ERR_CUDA;
    if (n && cudaMemcpyAsync(d.flv, flv, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, a->s) != cudaSuccess)
        r = PIC_ERR_CUDA;
    if (n && sg && cudaMemcpyAsync(sg, drift_sign, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, a->s) != cudaSuccess)
        r = PIC_ERR_CUDA;
    if (!r) r = adopt_ref(a, d, n, sg);
    cudaStreamSynchronize(a->s);
    cudaFree(blk);
    if (sg) cudaFree(sg);
    return r;
}

int pic_adj_fetch_particles(pic_adjoint *a, int64_t *nout, double *q, double *x, double *y, double *z, double *u,
                            double *v, double *w, int32_t *flv, double *drift_sign)
{
    if (!a) return PIC_ERR_INVALID;
    if (nout) *nout = a->np;
    const long long n = a->np;
    if (n == 0) return PIC_OK;
    double *tmp = nullptr;
    ACK(cudaMalloc((void **)&tmp, (size_t)n * sizeof(double)));
    double *dst[6] = {x, y, z, u, v, w};
    const double off[6] = {3.0, 3.0, 0.0, 0.0, 0.0, 0.0};
    int r = PIC_OK;
    std::vector<double> h((size_t)n);
    for (int k = 0; k < 6 && !r; k++) {
        if (!dst[k]) continue;
        if (a->fp32) k_to_double<float><<<grid_of(n), 256, 0, a->s>>>((const float *)a->p0[k], tmp, n);
        else k_to_double<double><<<grid_of(n), 256, 0, a->s>>>((const double *)a->p0[k], tmp, n);
        if (cudaMemcpyAsync(dst[k], tmp, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, a->s) != cudaSuccess ||
            cudaStreamSynchronize(a->s) != cudaSuccess)
            r = PIC_ERR_CUDA;
        for (long long i = 0; i < n && !r; i++) dst[k][i] += off[k];
    }
    cudaFree(tmp);
    if (!r && q && cudaMemcpy(q, a->q64, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) r = PIC_ERR_CUDA;
    if (!r && flv && cudaMemcpy(flv, a->flv, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess) r = PIC_ERR_CUDA;
    if (!r && drift_sign && cudaMemcpy(drift_sign, a->sgn, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        r = PIC_ERR_CUDA;
    return r;
}

int pic_adj_branches(pic_adjoint *a, int32_t mode)
{
    if (!a || mode < kBranchFree || mode > kBranchReplay) return PIC_ERR_INVALID;
    if (mode == kBranchReplay && a->br_steps == 0) return PIC_ERR_INVALID;
    a->br_mode = mode;
    return PIC_OK;
}

int pic_adj_forward(pic_adjoint *a, int32_t nsteps, int32_t checkpoint_every, double *objective)
{
    if (!a || nsteps < 1 || checkpoint_every < 1 || !objective) return PIC_ERR_INVALID;
    const int K = checkpoint_every < nsteps ? checkpoint_every : nsteps;
    return a->fp32 ? run_forward<float>(a, nsteps, K, objective) : run_forward<double>(a, nsteps, K, objective);
}

int pic_adj_gradient(pic_adjoint *a, double drift, const double *temp, double *du, double *dv, double *dw, double *dx,
                     double *dy, double *dparam)
{
    if (!a || a->T < 1) return PIC_ERR_INVALID;
    int r = a->fp32 ? run_backward<float>(a) : run_backward<double>(a);
    if (r) return r;
    const long long n = a->np;
    double *tmp = nullptr;
    ACK(cudaMalloc((void **)&tmp, (size_t)(n > 0 ? n : 1) * sizeof(double)));
    double *dst[6] = {dx, dy, nullptr, du, dv, dw};
    for (int k = 0; k < 6 && !r && n; k++) {
        if (!dst[k]) continue;
        if (a->fp32) k_to_double<float><<<grid_of(n), 256, 0, a->s>>>((const float *)a->pb[k], tmp, n);
        else k_to_double<double><<<grid_of(n), 256, 0, a->s>>>((const double *)a->pb[k], tmp, n);
        if (cudaMemcpyAsync(dst[k], tmp, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, a->s) != cudaSuccess ||
            cudaStreamSynchronize(a->s) != cudaSuccess)
            r = PIC_ERR_CUDA;
    }
    cudaFree(tmp);
    if (r) return r;
    if (dparam) {
        double *t2 = nullptr;
        ACK(cudaMalloc((void **)&t2, 2 * sizeof(double)));
        const double tt[2] = {temp ? temp[0] : 0.0, temp && a->cfg.nflvr > 1 ? temp[1] : 0.0};
        cudaMemcpy(t2, tt, sizeof(tt), cudaMemcpyHostToDevice);
        cudaMemsetAsync(a->acc + 1, 0, 3 * sizeof(double), a->s);
        if (n) {
            if (a->fp32)
                k_param_grad<float><<<grid_of(n), 256, 0, a->s>>>(ps<float>(a->p0), a->sgn, a->flv, n, ps<float>(a->pb),
                                                                   drift, t2, a->acc + 1);
            else
                k_param_grad<double><<<grid_of(n), 256, 0, a->s>>>(ps<double>(a->p0), a->sgn, a->flv, n,
                                                                    ps<double>(a->pb), drift, t2, a->acc + 1);
        }
        cudaMemcpyAsync(dparam, a->acc + 1, 3 * sizeof(double), cudaMemcpyDeviceToHost, a->s);
        cudaStreamSynchronize(a->s);
        cudaFree(t2);
        ACK(cudaGetLastError());
    }
    return PIC_OK;
}

}  // extern "C"
