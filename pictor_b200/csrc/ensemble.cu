// ensemble.cu -- the persistent step of an ensemble of FP32 runs: every
// phase of every run for a span of steps in one launch (no counterpart in the
// reference, which runs one simulation per job).
//
// The work of a step is a list of items in the order (phase, run, item): the
// B half step of every run (blocks of 32 x 32 interior cells), the mover of
// every run (bricks), the second B half step, the E update with the current
// fold and AddCurrent; the span of S steps is S such lists, one after the
// other.  A grid of resident CTAs takes the items in that order from one
// atomic counter.  An item waits until its run has finished the phase it
// depends on: the run's counter of finished items of that phase reaches the
// run's item count times the step (B half step <- the previous E update,
// mover <- B half step, second B half step <- mover, E update <- second B
// half step).  So each run steps at its own pace while the others fill the
// SMs, as the runs' step graphs on separate streams do, without a launch per
// phase and run.
//
// Ordering: a CTA finishes an item with a barrier, then one thread makes a
// release increment of the run's counter; a waiting CTA's thread spins on an
// acquire load of it, then a barrier.  The items read fields, currents and
// particles that other SMs wrote in the same launch, so this file is compiled
// with PIC_COHERENT_LOADS: those reads are weak loads, which the release /
// acquire pattern orders after the writes (never the non-coherent read-only
// path, which is only defined for data no thread writes during the kernel).
//
// Progress: items are claimed in order and an item waits only on earlier
// items.  The earliest unfinished item is either being worked on or claimed
// by a CTA whose current item is finished (a CTA claims one item ahead), so
// it always proceeds: the waits end without any assumption on which CTAs are
// resident.
//
// Every wait is bounded: after `spin_limit` polls (with a short sleep each)
// the CTA records PIC_DEVERR_TIMEOUT in the launch's status word, raises the
// abort flag, and every CTA stops taking items.  A test forces this bound to
// run out (`force_timeout`: the first mover item waits for a count nothing
// reaches) and checks that the call returns PIC_ERR_TIMEOUT with the GPU
// still usable.
#define PIC_COHERENT_LOADS 1

#include "common.cuh"
#include "field_math.cuh"
#include "kernels.cuh"
#include "mover_f32.cuh"

namespace pic {

namespace {

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void red_release_add(unsigned *p, unsigned v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int run_of(const int *__restrict__ start, int n, int item)
{
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (start[mid] <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <typename S>
__device__ __forceinline__ void copy_words(S *dst, const S *src)
{
    const int *a = reinterpret_cast<const int *>(src);
    int *b = reinterpret_cast<int *>(dst);
    for (int w = threadIdx.x; w < (int)(sizeof(S) / 4); w += blockDim.x) b[w] = ldco(a + w);
}

// The work of one item, outside the scheduling loop (not inlined, so that
// the loop keeps few registers live and the item bodies get the kernel's
// registers without spilling).
template <int DIMS, bool XC>
__device__ __noinline__ void persist_move_item(const BatchRun &sr, int b, float *sm, TileShared &ts)
{
    move_brick<DIMS, XC>(sr.g, sr.p[sr.cur], sr.bk, b, sm, ts, sr.E[0], sr.E[1], sr.E[2], sr.B[0], sr.B[1], sr.B[2],
                         sr.J[0], sr.J[1], sr.J[2], sr.err);
}
template <int DIMS, int FDTD>
__device__ __noinline__ void persist_field_item(const BatchRun &sr, int phase, int local)
{
    const int tid = threadIdx.x;
    // kPersistFieldRows blocks of 32 x 8 interior cells (the tiling of the
    // field kernels) stacked along y
    const int nby = (sr.fb[1] + kPersistFieldRows - 1) / kPersistFieldRows;
    const int bx = local % sr.fb[0], byz = local / sr.fb[0], byq = byz % nby, bz = byz / nby;
    for (int sub = 0; sub < kPersistFieldRows; sub++) {
        const int by = byq * kPersistFieldRows + sub;
        if (by >= sr.fb[1]) break;
        const CellIter it = interior_cell_at<DIMS>(sr.g, bx, by, bz, tid & 31, tid >> 5);
        if (phase == 3)
            efield_at<float, DIMS, 1>(sr.g, it, sr.E[0], sr.E[1], sr.E[2], sr.B[0], sr.B[1], sr.B[2], sr.J[0], sr.J[1],
                                      sr.J[2]);
        else
            bhalf_at<float, DIMS, FDTD>(sr.g, it, sr.E[0], sr.E[1], sr.E[2], sr.B[0], sr.B[1], sr.B[2]);
    }
}

// ctl: [0] next item, [1] abort flag, [2] status bits, [3 + 4 r + phase]
// finished items of run r's phase (cumulative over the span's steps).
//
// Thread 0 schedules: it claims the item after the current one while the
// CTA works on the current one (the claim's latency overlaps the work),
// waits for the current item's dependency, and publishes it in shared
// memory; two CTA barriers per item.  A run's descriptor is copied into
// shared memory only when the run changes (the descriptors do not change
// during a launch).
template <int DIMS, int FDTD, bool XC>
__global__ void __launch_bounds__(kTileThreads, 3)
    k_ensemble_persistent(const BatchRun *__restrict__ runs, const int *__restrict__ fstart,
                          const int *__restrict__ mstart, int n, int nsteps, unsigned *ctl, unsigned spin_limit,
                          int force_timeout)
{
    extern __shared__ __align__(16) float sm[];
    __shared__ TileShared ts;
    __shared__ BatchRun sr;
    __shared__ int s_go, s_run, s_phase, s_local;
    const int tid = threadIdx.x;
    unsigned *next = ctl, *abort_flag = ctl + 1, *status = ctl + 2, *done = ctl + 3;
    unsigned claim = 0;
    if (tid == 0) claim = atomicAdd(next, 1u);
    int loaded = -1;   // the run whose descriptor sr holds
    for (;;) {
        if (tid == 0) {
            const int F = fstart[n], M = mstart[n];
            const unsigned W = 3u * (unsigned)F + (unsigned)M;
            const unsigned item = claim;
            int go = item < W * (unsigned)nsteps && *(volatile unsigned *)abort_flag == 0;
            if (go) {
                claim = atomicAdd(next, 1u);   // consumed at the next item
                const unsigned s = item / W, rem = item - s * W;
                int phase, local;
                if (rem < (unsigned)F) { phase = 0; local = (int)rem; }
                else if (rem < (unsigned)(F + M)) { phase = 1; local = (int)rem - F; }
                else if (rem < (unsigned)(2 * F + M)) { phase = 2; local = (int)rem - F - M; }
                else { phase = 3; local = (int)rem - 2 * F - M; }
                const int r = phase == 1 ? run_of(mstart, n, local) : run_of(fstart, n, local);
                const unsigned fb = (unsigned)(fstart[r + 1] - fstart[r]), nb = (unsigned)(mstart[r + 1] - mstart[r]);
                // the phase this item depends on and the count it waits for
                int dep = -1;
                unsigned need = 0;
                if (phase == 0 && s > 0) { dep = 3; need = s * fb; }
                else if (phase == 1) { dep = 0; need = (s + 1) * fb; }
                else if (phase == 2) { dep = 1; need = (s + 1) * nb; }
                else if (phase == 3) { dep = 2; need = (s + 1) * fb; }
                if (force_timeout && phase == 1) need = 0xffffffffu;
                if (dep >= 0) {
                    const unsigned *c = done + 4 * r + dep;
                    unsigned polls = 0;
                    while (ld_acquire(c) < need) {
                        if (*(volatile unsigned *)abort_flag != 0) { go = 0; break; }
                        if (++polls > spin_limit) {
                            atomicOr(status, (unsigned)PIC_DEVERR_TIMEOUT);
                            atomicExch(abort_flag, 1u);
                            go = 0;
                            break;
                        }
                        __nanosleep(200);
                    }
                }
                s_run = r;
                s_phase = phase;
                s_local = local - (phase == 1 ? mstart[r] : fstart[r]);
            }
            s_go = go;
        }
        __syncthreads();   // the item is published; the previous one is finished
        if (!s_go) break;
        const int r = s_run, phase = s_phase, local = s_local;
        if (r != loaded) {
            copy_words(&sr, &runs[r]);
            loaded = r;
            __syncthreads();
        }
        if (phase == 1) persist_move_item<DIMS, XC>(sr, local, sm, ts);
        else persist_field_item<DIMS, FDTD>(sr, phase, local);
        __syncthreads();   // every thread's writes of the item precede the release
        if (tid == 0) {
            __threadfence();
            red_release_add(done + 4 * r + phase, 1u);
        }
    }
}

}  // namespace

int persistent_blocks_per_sm() { return 3; }

void launch_ensemble_persistent(int dims, int fdtd, bool exact_charge, const BatchRun *runs, const int *fstart,
                                const int *mstart, int n, int nsteps, unsigned *ctl, unsigned spin_limit,
                                int force_timeout, cudaStream_t s)
{
    static bool attr_set = false;
    auto set = [](const void *k) {
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kBrickSmemBytes);
    };
    if (!attr_set) {
        set((const void *)k_ensemble_persistent<2, PIC_FDTD_YEE, false>);
        set((const void *)k_ensemble_persistent<2, PIC_FDTD_LEHE, false>);
        set((const void *)k_ensemble_persistent<3, PIC_FDTD_YEE, false>);
        set((const void *)k_ensemble_persistent<3, PIC_FDTD_LEHE, false>);
        set((const void *)k_ensemble_persistent<3, PIC_FDTD_YEE, true>);
        set((const void *)k_ensemble_persistent<3, PIC_FDTD_LEHE, true>);
        attr_set = true;
    }
    // the words of the launch's counters start at zero
    cudaMemsetAsync(ctl, 0, sizeof(unsigned) * (3 + 4 * (size_t)n), s);
    const int grid = kSMs * persistent_blocks_per_sm();
    const int b = kTileThreads, sh = kBrickSmemBytes;
#define PIC_PERSIST(D, FD, X)                                                                                       \
    k_ensemble_persistent<D, FD, X><<<grid, b, sh, s>>>(runs, fstart, mstart, n, nsteps, ctl, spin_limit, force_timeout)
    if (dims == 2) {
        if (fdtd == PIC_FDTD_YEE) PIC_PERSIST(2, PIC_FDTD_YEE, false);
        else PIC_PERSIST(2, PIC_FDTD_LEHE, false);
    } else if (!exact_charge) {
        if (fdtd == PIC_FDTD_YEE) PIC_PERSIST(3, PIC_FDTD_YEE, false);
        else PIC_PERSIST(3, PIC_FDTD_LEHE, false);
    } else {
        if (fdtd == PIC_FDTD_YEE) PIC_PERSIST(3, PIC_FDTD_YEE, true);
        else PIC_PERSIST(3, PIC_FDTD_LEHE, true);
    }
#undef PIC_PERSIST
    count_launches(1);
}

}  // namespace pic
