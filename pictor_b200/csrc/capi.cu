// capi.cu -- the C ABI of include/pictor_b200.h: handle lifetime, host <->
// device copies, the phase entry points that replace the reference's
// `#ifdef gpu` subroutines (walls of src/bc and the x faces of a slab
// included), the CUDA-graph step loop and the ensemble steps.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "common.cuh"
#include "kernels.cuh"

using namespace pic;

namespace {
// NVTX ranges (header-only NVTX v3): one per step of pic_step and, in the
// profiling mode, one per phase, named as the reference's timers are
// (MAIN.F90:440-452), for nsys / ncu range filters.
const char *const kPhaseNames[PIC_PHASE_COUNT] = {"UpdateBfieldHalf", "MoveDepositPrtl", "ExchangePrtl",
                                                  "UpdateBfieldHalf2", "UpdateEfield+AddCurrent", "ReorderPrtl"};
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};
}  // namespace

struct pic_handle {
    pic_config cfg;
    GridP g;
    cudaStream_t s = nullptr;
    bool fp32 = false;
    void *E[3] = {}, *B[3] = {}, *J[3] = {};
    void *Jtmp = nullptr;
    double *open_col = nullptr;   // den, vel per (j, k) column of an 'open' particle face (2 my mz)
    // convolutional PML: per-axis tables (6 doubles and a flag per index),
    // twelve psi grids in the handle's precision (E psi1 x,y,z, psi2 x,y,z,
    // then B), kept across pic_bc_pml calls as the reference keeps them
    double *pml_coef = nullptr;
    uint8_t *pml_flag = nullptr;
    void *pml_psi = nullptr;
    bool pml_on = false;
    // cylindrical modal form: the fields on modes m = 0, 1, (mx, 3, mz) each;
    // E and B above are kept equal to their theta-gridded synthesis
    bool modal = false;
    void *Em[3] = {}, *Bm[3] = {}, *Jm[3] = {};   // the handle's precision
    PartF64 p64[2] = {};
    PartF32 p32[2] = {};
    int cur = 0;
    long long capacity = 0;
    Counters *cnt = nullptr;
    int *err = nullptr;
    SortScratch sc = {};
    double *tab_x = nullptr, *tab_p = nullptr;
    int ntab = 10000;
    double *diag_partials = nullptr;
    int diag_blocks = 0;
    double *diag_out = nullptr;
    double *rho = nullptr, *rho_pos = nullptr;
    long long t = 0;
    cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    int graph_kernels[2][2] = {{0, 0}, {0, 0}};
    bool profiling = false;
    double phase_ms[PIC_PHASE_COUNT] = {};
    long long phase_launches[PIC_PHASE_COUNT] = {};
    long long prof_steps = 0;
    long long launches = 0;   // kernels launched by pic_step since the last pic_launch_count
    // FP32 bricks (tile ranges valid while `sorted`: set by a reorder, cleared by loads)
    Bricks bricks = {};
    // host <-> device staging of the FP32 form (allocated at the first load or
    // fetch): two device buffers so that the copies of one chunk, on the copy
    // stream, overlap the conversion kernel of the other, on h->s
    cudaStream_t cs = nullptr;
    char *stage[2] = {nullptr, nullptr};
    size_t stage_bytes = 0;
    cudaEvent_t ev_copied[2] = {nullptr, nullptr}, ev_done[2] = {nullptr, nullptr};
    bool sorted = false;
    // slab form: device counts of the particles sent through the x faces
    uint32_t *slab_sent = nullptr;
    // phase entry points wait for their work (pic_set_sync)
    bool sync = true;
    // FP64 current summed in the serial order (pic_config.exact_current)
    bool exact = false;
    SegRecords rec = {};
    // FP64 Cartesian mover by tiles of cells after a reorder (valid while `sorted`)
    bool tiled64 = false;
    Tiles64 t64 = {};
    std::vector<void *> allocs;
};

static thread_local long long g_launches = 0;
static void batch_forget(pic_handle *h);
static void persist_forget(pic_handle *h);

namespace pic {
void count_launches(int n) { g_launches += n; }
}  // namespace pic

namespace {

int cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return PIC_OK;
    if (e == cudaErrorMemoryAllocation) return PIC_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return PIC_ERR_NOGPU;
    return PIC_ERR_CUDA;
}

#define CK(x)                                   \
    do {                                        \
        cudaError_t e_ = (x);                   \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

template <typename T>
int dalloc(pic_handle *h, T **p, size_t n)
{
    void *q = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T));
    if (e != cudaSuccess) return cuda_status(e);
    h->allocs.push_back(q);
    *p = (T *)q;
    return PIC_OK;
}

// Lehe coefficients, em_update_lehe.F90:8-25 (grid_dx = dy = dz = 1).
void lehe_coefficients(int dims, double c, double *o)
{
    const double pi = 3.14159265358979323846264;
    const double cinv = 1.0 / c;
    const double bxy = 0.125 * (1.0 * 1.0), bxz = 0.125 * (1.0 * 1.0);
    const double byx = 0.125, byz = 0.0, bzx = 0.125, bzy = 0.0;
    const double s = std::sin((0.5 * pi) * c);
    const double dxl = 0.25 * (1.0 - (cinv * cinv) * (s * s));
    const double dyl = 0.0, dzl = 0.0;
    if (dims == 3) {
        o[0] = ((1.0 - 2.0 * bxy) - 2.0 * bxz) - 3.0 * dxl;
        o[1] = ((1.0 - 2.0 * byx) - 2.0 * byz) - 3.0 * dyl;
        o[2] = ((1.0 - 2.0 * bzx) - 2.0 * bzy) - 3.0 * dzl;
    } else {
        o[0] = (1.0 - 2.0 * bxy) - 3.0 * dxl;
        o[1] = (1.0 - 2.0 * byx) - 3.0 * dyl;
        o[2] = 1.0;
    }
    o[3] = bxy; o[4] = bxz; o[5] = byx; o[6] = byz; o[7] = bzx; o[8] = bzy;
    o[9] = dxl; o[10] = dyl; o[11] = dzl;
}

// Lehe coefficients of cyl_em_update_lehe.F90:6-17 (grid_dx = dz = 1,
// dtheta = 2 pi/ny): the extended stencil acts along z.
void cyl_lehe_coefficients(double c, int ny, double *o)
{
    const double pi = 3.14159265358979323846264;
    const double dtheta = 2.0 * pi / ny;
    const double cinv = 1.0 / c;
    o[3] = 0.0;
    o[4] = 0.125;
    o[5] = 0.0;
    o[6] = 0.125;
    o[7] = 0.125 * ((1.0 / 1.0) * (1.0 / 1.0));
    o[8] = 0.125 * ((1.0 / (1.0 * dtheta)) * (1.0 / (1.0 * dtheta)));
    o[9] = 0.0;
    o[10] = 0.0;
    const double s = std::sin((0.5 * pi) * c);
    o[11] = 0.25 * (1.0 - (cinv * cinv) * (s * s));
    o[0] = ((1.0 - 2.0 * o[3]) - 2.0 * o[4]) - 3.0 * o[9];
    o[1] = ((1.0 - 2.0 * o[5]) - 2.0 * o[6]) - 3.0 * o[10];
    o[2] = ((1.0 - 2.0 * o[7]) - 2.0 * o[8]) - 3.0 * o[11];
}

// Init_MaxBolt_Table, prob_dist.F90:34-54.
void maxbolt_table(int n, std::vector<double> &X, std::vector<double> &P)
{
    X.assign(n, 0.0);
    P.assign(n, 0.0);
    const double dX = (15.0 - 0.0) / (double)(n - 1);
    for (int i = 1; i <= n; i++) X[i - 1] = dX * (double)(i - 1);
    double s = 0;
    for (int i = 2; i <= n; i++) {
        s = s + std::sqrt(X[i - 1]) * std::exp(-X[i - 1]);
        P[i - 1] = s;
    }
    for (int i = 0; i < n; i++) P[i] = P[i] / s;
}

int check_device_errors(pic_handle *h)
{
    int bits = 0;
    CK(cudaMemcpyAsync(&bits, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    if (bits & PIC_DEVERR_OVERFLOW) return PIC_ERR_OVERFLOW;
    if (bits & PIC_DEVERR_RANGE) return PIC_ERR_RANGE;
    if (bits & PIC_DEVERR_NAN) return PIC_ERR_NAN;
    if (bits & (PIC_DEVERR_SUBSTEP | PIC_DEVERR_TIMEOUT)) return PIC_ERR_TIMEOUT;
    return PIC_OK;
}

// Finish a synchronous entry point: launch errors, stream errors, device error word.
int finish(pic_handle *h)
{
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->s));
    return check_device_errors(h);
}

// Finish a phase entry point: as finish, or, with pic_set_sync(h, 0), launch
// errors only (the work stays queued on the handle's stream).
int finish_phase(pic_handle *h)
{
    if (h->sync) return finish(h);
    CK(cudaGetLastError());
    return PIC_OK;
}

template <typename T>
void field_ptrs(pic_handle *h, T *E[3], T *B[3], T *J[3])
{
    for (int c = 0; c < 3; c++) {
        E[c] = (T *)h->E[c];
        B[c] = (T *)h->B[c];
        J[c] = (T *)h->J[c];
    }
}

// The modal field phases (cyl_modes = 2) in the handle's precision T: each
// leaves the theta-gridded E / B equal to the synthesis of the modes.
template <typename T>
void modal_ptrs(pic_handle *h, T *Em[3], T *Bm[3], T *Jm[3])
{
    for (int k = 0; k < 3; k++) {
        Em[k] = (T *)h->Em[k];
        Bm[k] = (T *)h->Bm[k];
        Jm[k] = (T *)h->Jm[k];
    }
}
template <typename T>
void modal_bhalf(pic_handle *h)
{
    T *E[3], *B[3], *J[3], *Em[3], *Bm[3], *Jm[3];
    field_ptrs(h, E, B, J);
    modal_ptrs(h, Em, Bm, Jm);
    launch_modal_bhalf<T>(h->g, Em, Bm, h->s);
    launch_modal_synth<T>(h->g, Bm, B, h->s);
}
template <typename T>
void modal_update_e(pic_handle *h)
{
    T *E[3], *B[3], *J[3], *Em[3], *Bm[3], *Jm[3];
    field_ptrs(h, E, B, J);
    modal_ptrs(h, Em, Bm, Jm);
    launch_modal_efield<T>(h->g, 0, Em, Bm, Jm, h->s);
    launch_modal_synth<T>(h->g, Em, E, h->s);
}
// AddCurrent of the (folded) theta-gridded J, projected onto the modes.
template <typename T>
void modal_add_current(pic_handle *h)
{
    T *E[3], *B[3], *J[3], *Em[3], *Bm[3], *Jm[3];
    field_ptrs(h, E, B, J);
    modal_ptrs(h, Em, Bm, Jm);
    launch_modal_project<T>(h->g, J, Jm, h->s);
    launch_modal_efield<T>(h->g, 2, Em, Bm, Jm, h->s);
    launch_modal_synth<T>(h->g, Em, E, h->s);
}
// The E phase of a step: E update, fold, projection, AddCurrent, synthesis.
template <typename T>
void modal_efield_phase(pic_handle *h)
{
    T *E[3], *B[3], *J[3], *Em[3], *Bm[3], *Jm[3];
    field_ptrs(h, E, B, J);
    modal_ptrs(h, Em, Bm, Jm);
    launch_modal_efield<T>(h->g, 0, Em, Bm, Jm, h->s);
    launch_cyl_fold<T>(h->g, J, h->s);
    launch_modal_project<T>(h->g, J, Jm, h->s);
    launch_modal_efield<T>(h->g, 2, Em, Bm, Jm, h->s);
    launch_modal_synth<T>(h->g, Em, E, h->s);
}
// Loaded theta-gridded fields -> their modes m = 0, 1; E, B become the synthesis.
template <typename T>
void modal_load(pic_handle *h)
{
    T *E[3], *B[3], *J[3], *Em[3], *Bm[3], *Jm[3];
    field_ptrs(h, E, B, J);
    modal_ptrs(h, Em, Bm, Jm);
    launch_modal_project<T>(h->g, E, Em, h->s);
    launch_modal_project<T>(h->g, B, Bm, h->s);
    launch_modal_synth<T>(h->g, Em, E, h->s);
    launch_modal_synth<T>(h->g, Bm, B, h->s);
}

// One phase of a full step (MAIN.F90:42-284), enqueued on h->s; reads
// buffer `cur` and, for the reorder phase, leaves the particles in cur^1.
// Returns the number of kernels it launched.
int enqueue_phase(pic_handle *h, int cur, bool reorder, int phase)
{
    const GridP &g = h->g;
    const bool filt = h->cfg.curr_filter > 0;
    g_launches = 0;
    if (g.geom == PIC_GEOM_CYLINDRICAL && h->fp32) {  // the FP32 cell-relative form
        float *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        switch (phase) {
            case PIC_PHASE_BHALF1:
            case PIC_PHASE_BHALF2:
                if (h->modal) modal_bhalf<float>(h);
                else launch_cyl_bhalf<float>(g, E, B, h->s);
                break;
            case PIC_PHASE_MOVE:  // push, deposit and the wrap / outer-radius drop
                if (h->sorted)
                    launch_cyl_move_deposit_f32_tiled(g, h->p32[cur], h->bricks, E, B, J, h->err, h->s);
                else
                    launch_cyl_move_deposit_f32(g, h->p32[cur], h->cnt, E, B, J, h->err, h->s);
                break;
            case PIC_PHASE_EXCHANGE:
                break;
            case PIC_PHASE_EFIELD:
                if (h->modal) {
                    modal_efield_phase<float>(h);
                } else {
                    launch_cyl_efield<float>(g, 0, E, B, J, h->s);
                    launch_cyl_fold<float>(g, J, h->s);
                    launch_cyl_efield<float>(g, 2, E, B, J, h->s);
                }
                for (int c = 0; c < 3; c++) cudaMemsetAsync(J[c], 0, (size_t)g.ncell * sizeof(float), h->s);
                break;
            case PIC_PHASE_REORDER:
                if (reorder)
                    launch_reorder_f32(g, h->p32[cur], h->p32[cur ^ 1], h->cnt, h->capacity, h->bricks, h->err, h->s);
                break;
        }
        return (int)g_launches;
    }
    if (g.geom == PIC_GEOM_CYLINDRICAL) {
        double *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        switch (phase) {
            case PIC_PHASE_BHALF1:  // cyl_em_update.F90:49-110 + halo
            case PIC_PHASE_BHALF2:
                if (h->modal) modal_bhalf<double>(h);
                else launch_cyl_bhalf(g, E, B, h->s);
                break;
            case PIC_PHASE_MOVE:  // cyl_movdep_strang.F90:14-378
                launch_cyl_move_deposit(g, h->p64[cur], h->cnt, E, B, J, h->err, h->s,
                                        h->tiled64 && h->sorted ? &h->t64 : nullptr);
                break;
            case PIC_PHASE_EXCHANGE:
                launch_exchange_f64(g, h->p64[cur], h->cnt, h->sc, h->capacity, h->err, h->s);
                break;
            case PIC_PHASE_EFIELD:  // UpdateEfield, halo, fold, AddCurrent, halo, ResetCurrent
                if (h->modal) {
                    modal_efield_phase<double>(h);
                } else {
                    launch_cyl_efield(g, 0, E, B, J, h->s);
                    launch_cyl_fold(g, J, h->s);
                    launch_cyl_efield(g, 2, E, B, J, h->s);
                }
                for (int c = 0; c < 3; c++) cudaMemsetAsync(J[c], 0, (size_t)g.ncell * sizeof(double), h->s);
                break;
            case PIC_PHASE_REORDER:
                if (reorder)
                    launch_reorder_f64(g, h->p64[cur], h->p64[cur ^ 1], h->cnt, h->sc, h->capacity, h->err, h->s,
                                       h->tiled64 ? &h->t64 : nullptr);
                break;
        }
        return (int)g_launches;
    }
    if (!h->fp32) {
        double *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        switch (phase) {
            case PIC_PHASE_BHALF1:  // MAIN.F90:49-58
            case PIC_PHASE_BHALF2:  // MAIN.F90:101-105
                launch_bhalf<double>(g, E, B, h->s);
                break;
            case PIC_PHASE_MOVE:  // MAIN.F90:63-71
                if (h->tiled64 && h->sorted)
                    launch_move_deposit_f64_tiled(g, h->p64[cur], h->cnt, h->t64, E, B, J, h->err, h->s);
                else
                    launch_move_deposit_f64(g, h->p64[cur], h->cnt, E, B, J, h->err, h->s, h->exact ? &h->rec : nullptr);
                break;
            case PIC_PHASE_EXCHANGE:  // MAIN.F90:86-94 + 145-150
                launch_exchange_f64(g, h->p64[cur], h->cnt, h->sc, h->capacity, h->err, h->s);
                break;
            case PIC_PHASE_EFIELD:  // MAIN.F90:108-110, 124, 158, 170-184
                if (!filt) {
                    launch_efield<double>(g, 1, E, B, J, h->s);
                } else {
                    launch_fold<double>(g, J, h->s);
                    for (int k = 0; k < h->cfg.curr_filter; k++) launch_filter<double>(g, J, (double *)h->Jtmp, h->s);
                    launch_efield<double>(g, 3, E, B, J, h->s);
                    for (int c = 0; c < 3; c++) cudaMemsetAsync(J[c], 0, (size_t)g.ncell * sizeof(double), h->s);
                }
                break;
            case PIC_PHASE_REORDER:  // MAIN.F90:259-265
                if (reorder)
                    launch_reorder_f64(g, h->p64[cur], h->p64[cur ^ 1], h->cnt, h->sc, h->capacity, h->err, h->s,
                                       h->tiled64 ? &h->t64 : nullptr);
                break;
        }
    } else {
        float *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        switch (phase) {
            case PIC_PHASE_BHALF1:
            case PIC_PHASE_BHALF2:
                launch_bhalf<float>(g, E, B, h->s);
                break;
            case PIC_PHASE_MOVE:
                if (h->sorted)
                    launch_move_deposit_f32_tiled(g, h->p32[cur], h->bricks, h->cnt, E, B, J, h->err, h->s);
                else
                    launch_move_deposit_f32(g, h->p32[cur], h->cnt, E, B, J, h->err, h->s);
                break;
            case PIC_PHASE_EXCHANGE:  // the FP32 form wraps inside the mover
                break;
            case PIC_PHASE_EFIELD:
                if (!filt) {
                    launch_efield<float>(g, 1, E, B, J, h->s);
                } else {
                    launch_fold<float>(g, J, h->s);
                    for (int k = 0; k < h->cfg.curr_filter; k++) launch_filter<float>(g, J, (float *)h->Jtmp, h->s);
                    launch_efield<float>(g, 3, E, B, J, h->s);
                    for (int c = 0; c < 3; c++) cudaMemsetAsync(J[c], 0, (size_t)g.ncell * sizeof(float), h->s);
                }
                break;
            case PIC_PHASE_REORDER:
                if (reorder)
                    launch_reorder_f32(g, h->p32[cur], h->p32[cur ^ 1], h->cnt, h->capacity, h->bricks, h->err, h->s);
                break;
        }
    }
    return (int)g_launches;
}

int enqueue_step(pic_handle *h, int cur, bool reorder)
{
    int n = 0;
    for (int ph = 0; ph < PIC_PHASE_COUNT; ph++) n += enqueue_phase(h, cur, reorder, ph);
    return n;
}

int get_graph(pic_handle *h, int cur, bool reorder, cudaGraphExec_t *out)
{
    cudaGraphExec_t &ge = h->graph[reorder ? 1 : 0][cur];
    if (!ge) {
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
        h->graph_kernels[reorder ? 1 : 0][cur] = enqueue_step(h, cur, reorder);
        cudaError_t e = cudaStreamEndCapture(h->s, &graph);
        if (e != cudaSuccess) return cuda_status(e);
        e = cudaGraphInstantiate(&ge, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            ge = nullptr;
            return cuda_status(e);
        }
    }
    *out = ge;
    return PIC_OK;
}

// pic_step with an event pair around every phase of every step (no graphs).
int step_profiled(pic_handle *h, int32_t nsteps)
{
    const int NE = PIC_PHASE_COUNT + 1;
    std::vector<cudaEvent_t> ev((size_t)nsteps * NE);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    int rc = PIC_OK;
    for (int32_t i = 0; i < nsteps && rc == PIC_OK; i++) {
        h->t += 1;
        const bool reorder = h->cfg.reorder_period > 0 && (h->t % h->cfg.reorder_period) == 0;
        cudaEvent_t *e = &ev[(size_t)i * NE];
        cudaEventRecord(e[0], h->s);
        for (int ph = 0; ph < PIC_PHASE_COUNT; ph++) {
            NvtxRange r(kPhaseNames[ph]);
            h->phase_launches[ph] += enqueue_phase(h, h->cur, reorder, ph);
            cudaEventRecord(e[ph + 1], h->s);
        }
        if (reorder) {
            h->cur ^= 1;
            if (h->fp32 || h->tiled64) h->sorted = true;  // eager launches: no graph to drop
        }
        h->prof_steps += 1;
        if (cudaGetLastError() != cudaSuccess) rc = PIC_ERR_CUDA;
    }
    if (cudaStreamSynchronize(h->s) != cudaSuccess) rc = PIC_ERR_CUDA;
    for (int32_t i = 0; i < nsteps && rc == PIC_OK; i++)
        for (int ph = 0; ph < PIC_PHASE_COUNT; ph++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[(size_t)i * NE + ph], ev[(size_t)i * NE + ph + 1]);
            h->phase_ms[ph] += ms;
        }
    for (auto &e : ev) cudaEventDestroy(e);
    return rc;
}

// The FP32 mover variant is baked into the step graphs: drop them when the
// tile ranges become valid or stale.
void set_sorted(pic_handle *h, bool sorted)
{
    if (h->sorted == sorted) return;
    h->sorted = sorted;
    for (auto &row : h->graph)
        for (auto &ge : row)
            if (ge) {
                cudaGraphExecDestroy(ge);
                ge = nullptr;
            }
}

// One step of pic_step as a graph launch on h->s (graphs captured on first use).
int enqueue_graph_step(pic_handle *h)
{
    NvtxRange range("pic_step");
    h->t += 1;
    const bool reorder = h->cfg.reorder_period > 0 && (h->t % h->cfg.reorder_period) == 0;
    cudaGraphExec_t ge = nullptr;
    int r = get_graph(h, h->cur, reorder, &ge);
    if (r) return r;
    CK(cudaGraphLaunch(ge, h->s));
    h->launches += h->graph_kernels[reorder ? 1 : 0][h->cur];
    if (reorder) {
        h->cur ^= 1;
        if ((h->fp32 || h->tiled64) && !h->sorted) {  // tile ranges are valid from now on
            CK(cudaStreamSynchronize(h->s));
            set_sorted(h, true);
        }
    }
    return PIC_OK;
}

size_t field_bytes(const pic_handle *h) { return (size_t)h->g.ncell * (h->fp32 ? sizeof(float) : sizeof(double)); }

int alloc_particles(pic_handle *h)
{
    const size_t n = (size_t)h->capacity;
    for (int b = 0; b < 2; b++) {
        if (!h->fp32) {
            PartF64 &p = h->p64[b];
            int r;
            if ((r = dalloc(h, &p.q, n)) || (r = dalloc(h, &p.x, n)) || (r = dalloc(h, &p.y, n)) ||
                (r = dalloc(h, &p.z, n)) || (r = dalloc(h, &p.u, n)) || (r = dalloc(h, &p.v, n)) ||
                (r = dalloc(h, &p.w, n)) || (r = dalloc(h, &p.flv, n)))
                return r;
        } else {
            PartF32 &p = h->p32[b];
            int r;
            if ((r = dalloc(h, &p.key, n)) || (r = dalloc(h, &p.dx, n)) || (r = dalloc(h, &p.dy, n)) ||
                (h->g.dims == 3 && (r = dalloc(h, &p.dz, n))) || (r = dalloc(h, &p.ux, n)) ||
                (r = dalloc(h, &p.uy, n)) || (r = dalloc(h, &p.uz, n)) || (r = dalloc(h, &p.w, n)))
                return r;
        }
    }
    return PIC_OK;
}

// Staging of the FP32 form: chunks of at most kConvChunk particles (60 B each
// in the reference layout) or kFieldChunk field values.
constexpr long long kConvChunk = 1ll << 23;
constexpr long long kFieldChunk = 1ll << 24;
constexpr size_t kPartBytes = 7 * sizeof(double) + sizeof(int32_t);

int ensure_stage(pic_handle *h)
{
    if (h->stage[0]) return PIC_OK;
    const long long np = h->capacity < kConvChunk ? (h->capacity > 0 ? h->capacity : 1) : kConvChunk;
    const long long nf = h->g.ncell < kFieldChunk ? h->g.ncell : kFieldChunk;
    size_t bytes = (size_t)np * kPartBytes;
    if ((size_t)nf * sizeof(double) > bytes) bytes = (size_t)nf * sizeof(double);
    for (int b = 0; b < 2; b++) {
        int r = dalloc(h, &h->stage[b], bytes);
        if (r) return r;
        CK(cudaEventCreateWithFlags(&h->ev_copied[b], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&h->ev_done[b], cudaEventDisableTiming));
    }
    CK(cudaStreamCreateWithFlags(&h->cs, cudaStreamNonBlocking));
    h->stage_bytes = bytes;
    return PIC_OK;
}

// Particles of chunk size m in staging buffer b, reference layout.
PartF64 stage_particles(pic_handle *h, int b, long long m)
{
    PartF64 p;
    double *d = (double *)h->stage[b];
    p.q = d; p.x = d + m; p.y = d + 2 * m; p.z = d + 3 * m; p.u = d + 4 * m; p.v = d + 5 * m; p.w = d + 6 * m;
    p.flv = (int32_t *)(d + 7 * m);
    return p;
}

long long stage_particle_chunk(const pic_handle *h) { return (long long)(h->stage_bytes / kPartBytes); }
long long stage_field_chunk(const pic_handle *h) { return (long long)(h->stage_bytes / sizeof(double)); }

// Host FP64 array -> device FP32 array through the staging buffers.
int load_array_f32(pic_handle *h, const double *src, float *dst, long long n, int &k)
{
    const long long chunk = stage_field_chunk(h);
    for (long long o = 0; o < n; o += chunk, k++) {
        const int b = k & 1;
        const long long m = (n - o) < chunk ? (n - o) : chunk;
        double *t = (double *)h->stage[b];
        CK(cudaStreamWaitEvent(h->cs, h->ev_done[b], 0));
        CK(cudaMemcpyAsync(t, src + o, (size_t)m * sizeof(double), cudaMemcpyHostToDevice, h->cs));
        CK(cudaEventRecord(h->ev_copied[b], h->cs));
        CK(cudaStreamWaitEvent(h->s, h->ev_copied[b], 0));
        launch_array_f64_to_f32(t, dst + o, m, h->s);
        CK(cudaEventRecord(h->ev_done[b], h->s));
    }
    return PIC_OK;
}

// Device FP32 array -> host FP64 array through the staging buffers.
int fetch_array_f32(pic_handle *h, const float *src, double *dst, long long n, int &k)
{
    const long long chunk = stage_field_chunk(h);
    for (long long o = 0; o < n; o += chunk, k++) {
        const int b = k & 1;
        const long long m = (n - o) < chunk ? (n - o) : chunk;
        double *t = (double *)h->stage[b];
        CK(cudaStreamWaitEvent(h->s, h->ev_copied[b], 0));
        launch_array_f32_to_f64(src + o, t, m, h->s);
        CK(cudaEventRecord(h->ev_done[b], h->s));
        CK(cudaStreamWaitEvent(h->cs, h->ev_done[b], 0));
        CK(cudaMemcpyAsync(dst + o, t, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, h->cs));
        CK(cudaEventRecord(h->ev_copied[b], h->cs));
    }
    return PIC_OK;
}

int sync_both(pic_handle *h)
{
    CK(cudaStreamSynchronize(h->s));
    if (h->cs) CK(cudaStreamSynchronize(h->cs));
    return PIC_OK;
}

}  // namespace

// The batched form of pic_step_many: FP32 runs of one dimensionality, all
// reordered once (bricks valid), no current filter.  Every phase of a group
// of runs is one launch (k_field_batch, k_move_f32_batch; the four launches
// of a step captured in one CUDA graph on the group's stream); a run whose
// reorder period comes up is reordered right after the step, on the same
// stream, and its current buffer is flipped on the device.
static bool batchable(pic_handle *const *hs, int32_t n)
{
    if (n < 1) return false;
    for (int32_t a = 0; a < n; a++) {
        const pic_handle *h = hs[a];
        if (!h->fp32 || !h->sorted || h->g.geom != PIC_GEOM_CARTESIAN || h->cfg.curr_filter != 0 || h->profiling ||
            h->g.dims != hs[0]->g.dims || h->g.fdtd != hs[0]->g.fdtd || h->g.exact_charge != hs[0]->g.exact_charge)
            return false;
    }
    return true;
}

// The device descriptors, work lists and the captured step graph of one
// group of runs, kept for the next call with the same runs (the descriptors
// are uploaded again at every call: a run's current buffer may have changed).
struct BatchGroup {
    std::vector<pic_handle *> runs;
    cudaStream_t s = nullptr;
    int nf = 0, nm = 0;
    BatchRun *druns = nullptr;
    int *dstart = nullptr;
    cudaGraphExec_t ge = nullptr;
    long long step_kernels = 0;
    void release()
    {
        if (ge) cudaGraphExecDestroy(ge);
        if (druns) cudaFree(druns);
        if (dstart) cudaFree(dstart);
        ge = nullptr;
        druns = nullptr;
        dstart = nullptr;
        runs.clear();
    }
};
struct BatchCache {
    std::vector<pic_handle *> key;
    std::vector<BatchGroup> groups;
    void release()
    {
        for (BatchGroup &g : groups) g.release();
        groups.clear();
        key.clear();
    }
};
static BatchCache g_batch;
static std::mutex g_batch_mu;

// The persistent form of pic_step_batched (ensemble.cu): all runs in one
// group; the device descriptors and work lists uploaded once per set of
// runs, the call's launch sequence captured once per (runs, steps, reorder
// phases and buffers) and replayed.
struct PersistCache {
    std::vector<pic_handle *> key;
    BatchRun *druns = nullptr;
    int *dstart = nullptr;
    unsigned *ctl = nullptr;
    int nf = 0, nm = 0;
    struct Graph {
        std::vector<long long> key;
        cudaGraphExec_t exec;
        long long launches;
    };
    std::vector<Graph> graphs;
    void release()
    {
        for (auto &g : graphs) cudaGraphExecDestroy(g.exec);
        graphs.clear();
        if (druns) cudaFree(druns);
        if (dstart) cudaFree(dstart);
        if (ctl) cudaFree(ctl);
        druns = nullptr;
        dstart = nullptr;
        ctl = nullptr;
        key.clear();
    }
};
static PersistCache g_persist;

// A handle that goes away takes the cached persistent sequence with it.
static void persist_forget(pic_handle *h)
{
    for (pic_handle *k : g_persist.key)
        if (k == h) {
            g_persist.release();
            return;
        }
}


// A handle that goes away takes the cached batch with it.
static void batch_forget(pic_handle *h)
{
    std::lock_guard<std::mutex> lk(g_batch_mu);
    for (pic_handle *k : g_batch.key)
        if (k == h) {
            g_batch.release();
            break;
        }
    persist_forget(h);
}

// Runs per group: the batch is split into kBatchGroups groups of about equal
// particle count, each stepped by its own four launches on its own stream, so
// that the phases of different groups overlap (one group's field phase with
// another's mover) as separate runs' step graphs do.
constexpr int kBatchGroups = 4;

static BatchRun batch_run_of(pic_handle *h)
{
    BatchRun R;
    std::memset(&R, 0, sizeof(R));
    R.g = h->g;
    R.p[0] = h->p32[0];
    R.p[1] = h->p32[1];
    R.bk = h->bricks;
    for (int k = 0; k < 3; k++) {
        R.E[k] = (float *)h->E[k];
        R.B[k] = (float *)h->B[k];
        R.J[k] = (float *)h->J[k];
    }
    R.err = h->err;
    R.cur = h->cur;
    R.fb[0] = (h->g.nx + 31) / 32;
    R.fb[1] = (h->g.ny + 7) / 8;
    R.fb[2] = h->g.dims == 3 ? h->g.nz : 1;
    return R;
}

// Upload the group's descriptors and work lists; capture its step graph the
// first time.
static int batch_group_prepare(BatchGroup &G, bool fresh)
{
    const int n = (int)G.runs.size();
    pic_handle *h0 = G.runs[0];
    std::vector<BatchRun> runs((size_t)n);
    std::vector<int> starts(2 * ((size_t)n + 1), 0);
    int *fstart = starts.data(), *mstart = starts.data() + n + 1;
    for (int a = 0; a < n; a++) {
        runs[(size_t)a] = batch_run_of(G.runs[(size_t)a]);
        const BatchRun &R = runs[(size_t)a];
        fstart[a + 1] = fstart[a] + R.fb[0] * R.fb[1] * R.fb[2];
        mstart[a + 1] = mstart[a] + R.bk.ntiles;
    }
    if (fresh) {
        G.s = h0->s;
        G.nf = fstart[n];
        G.nm = mstart[n];
        if (cudaMalloc(&G.druns, sizeof(BatchRun) * (size_t)n) != cudaSuccess ||
            cudaMalloc(&G.dstart, sizeof(int) * starts.size()) != cudaSuccess)
            return PIC_ERR_OOM;
    }
    CK(cudaMemcpyAsync(G.druns, runs.data(), sizeof(BatchRun) * (size_t)n, cudaMemcpyHostToDevice, G.s));
    CK(cudaMemcpyAsync(G.dstart, starts.data(), sizeof(int) * starts.size(), cudaMemcpyHostToDevice, G.s));
    CK(cudaStreamSynchronize(G.s));
    if (!fresh) return PIC_OK;
    // one step of every run: B half, move + deposit, B half, E + fold + AddCurrent
    const int dims = h0->g.dims, fdtd = h0->g.fdtd;
    g_launches = 0;
    cudaGraph_t gr = nullptr;
    CK(cudaStreamBeginCapture(G.s, cudaStreamCaptureModeThreadLocal));
    launch_batch_bhalf(dims, fdtd, G.druns, G.dstart, n, G.nf, G.s);
    launch_batch_move(dims, h0->g.exact_charge != 0, G.druns, G.dstart + n + 1, n, G.nm, G.s);
    launch_batch_bhalf(dims, fdtd, G.druns, G.dstart, n, G.nf, G.s);
    launch_batch_efield(dims, G.druns, G.dstart, n, G.nf, G.s);
    G.step_kernels = g_launches;
    const cudaError_t e = cudaStreamEndCapture(G.s, &gr);
    const cudaError_t ei = e == cudaSuccess ? cudaGraphInstantiate(&G.ge, gr, 0) : e;
    if (gr) cudaGraphDestroy(gr);
    if (ei != cudaSuccess) {
        G.ge = nullptr;
        return cuda_status(ei);
    }
    return PIC_OK;
}

static int step_many_batched(pic_handle *const *hs, int32_t n, int32_t nsteps)
{
    std::lock_guard<std::mutex> lk(g_batch_mu);
    for (int32_t a = 0; a < n; a++) CK(cudaStreamSynchronize(hs[a]->s));
    BatchCache &C = g_batch;
    const bool same = !C.groups.empty() && C.key.size() == (size_t)n && std::equal(C.key.begin(), C.key.end(), hs);
    if (!same) {
        C.release();
        // largest first, dealt to the lightest group
        std::vector<int32_t> order((size_t)n);
        for (int32_t a = 0; a < n; a++) order[(size_t)a] = a;
        std::stable_sort(order.begin(), order.end(),
                         [&](int32_t x, int32_t y) { return hs[x]->capacity > hs[y]->capacity; });
        const int ng = n < kBatchGroups ? (int)n : kBatchGroups;
        C.groups.resize((size_t)ng);
        std::vector<long long> load((size_t)ng, 0);
        for (int32_t a : order) {
            size_t gi = 0;
            for (size_t q = 1; q < load.size(); q++)
                if (load[q] < load[gi]) gi = q;
            C.groups[gi].runs.push_back(hs[a]);
            load[gi] += hs[a]->capacity;
        }
        C.key.assign(hs, hs + n);
    }
    for (BatchGroup &G : C.groups) {
        for (pic_handle *h : G.runs)
            for (int k = 0; k < 3; k++) CK(cudaMemsetAsync(h->J[k], 0, field_bytes(h), G.runs[0]->s));
        const int r = batch_group_prepare(G, !same);
        if (r) {
            C.release();
            return r;
        }
    }
    for (int32_t i = 0; i < nsteps; i++)
        for (BatchGroup &G : C.groups) {
            CK(cudaGraphLaunch(G.ge, G.s));
            G.runs[0]->launches += G.step_kernels;
            for (size_t a = 0; a < G.runs.size(); a++) {
                pic_handle *h = G.runs[a];
                h->t += 1;
                if (h->cfg.reorder_period > 0 && (h->t % h->cfg.reorder_period) == 0) {
                    g_launches = 0;
                    launch_reorder_f32(h->g, h->p32[h->cur], h->p32[h->cur ^ 1], h->cnt, h->capacity, h->bricks,
                                       h->err, G.s);
                    launch_batch_flip(G.druns, (int)a, G.s);
                    h->launches += g_launches;
                    h->cur ^= 1;
                }
            }
        }
    for (BatchGroup &G : C.groups) CK(cudaStreamSynchronize(G.s));
    int first = PIC_OK;
    for (int32_t a = 0; a < n; a++) {
        const int q = finish(hs[a]);
        if (q && !first) first = q;
    }
    return first;
}

extern "C" {

int pic_version(void) { return 10000; }

const char *pic_error_string(int code)
{
    switch (code) {
        case PIC_OK: return "ok";
        case PIC_ERR_INVALID: return "invalid argument or configuration";
        case PIC_ERR_OOM: return "device memory allocation failed";
        case PIC_ERR_OVERFLOW: return "particle capacity exceeded";
        case PIC_ERR_NAN: return "non-finite value";
        case PIC_ERR_TIMEOUT: return "bounded device wait timed out";
        case PIC_ERR_CUDA: return "CUDA runtime error";
        case PIC_ERR_RANGE: return "particle outside the ghost frame of the grid";
        case PIC_ERR_NOGPU: return "no CUDA device";
        default: return "unknown error";
    }
}

void pic_destroy(pic_handle *h)
{
    if (h) batch_forget(h);
    if (!h) return;
    if (h->s) cudaStreamSynchronize(h->s);
    if (h->cs) cudaStreamSynchronize(h->cs);
    for (auto &row : h->graph)
        for (auto &ge : row)
            if (ge) cudaGraphExecDestroy(ge);
    for (int b = 0; b < 2; b++) {
        if (h->ev_copied[b]) cudaEventDestroy(h->ev_copied[b]);
        if (h->ev_done[b]) cudaEventDestroy(h->ev_done[b]);
    }
    for (void *p : h->allocs) cudaFree(p);
    if (h->cs) cudaStreamDestroy(h->cs);
    if (h->s) cudaStreamDestroy(h->s);
    delete h;
}

int pic_create(const pic_config *cfg, pic_handle **out)
{
    if (!cfg || !out) return PIC_ERR_INVALID;
    *out = nullptr;
    const pic_config &c = *cfg;
    if (c.dims != 2 && c.dims != 3) return PIC_ERR_INVALID;
    if (c.geom != PIC_GEOM_CARTESIAN && c.geom != PIC_GEOM_CYLINDRICAL) return PIC_ERR_INVALID;
    // the cylindrical step: 3D, no current filter; the reference's FP64 form
    // or the FP32 cell-relative one, each with the theta-gridded or the modal
    // (m = 0, 1) field solve.  The rank holding the axis has it at x = 3.5
    // (rmin = rshift = -0.5, cyl_common.F90:23); a slab away from the axis
    // starts at least 2.5 cells out, so that every radius its stencils use,
    // ghosts included, is positive.
    if (c.geom == PIC_GEOM_CYLINDRICAL &&
        (c.dims != 3 || c.curr_filter != 0 || (c.ny % 2) != 0 || (c.inc_axis != 0 && c.inc_axis != 1) ||
         (c.inc_axis ? c.rmin != -0.5 : (c.slab_x == 0 || !(c.rmin >= 2.5)))))
        return PIC_ERR_INVALID;
    if (c.cyl_modes != 0 && (c.geom != PIC_GEOM_CYLINDRICAL || c.cyl_modes != 2 || c.ny < 4)) return PIC_ERR_INVALID;
    // the slab form: the Cartesian step (FP64 or FP32) or the FP64
    // theta-gridded cylindrical one with its x faces on neighbouring ranks
    // (no current filter: its passes would need a halo exchange per pass);
    // 2 = the high x face is the outer radius of a cylinder
    if (c.slab_x < 0 || c.slab_x > 2 || (c.slab_x != 0 && c.curr_filter != 0) ||
        (c.slab_x == 2 && c.geom != PIC_GEOM_CYLINDRICAL) ||
        (c.slab_x != 0 && c.geom == PIC_GEOM_CYLINDRICAL && (c.precision != PIC_PREC_FP64 || c.cyl_modes != 0)))
        return PIC_ERR_INVALID;
    // the exact-order current: FP64 Cartesian, two sorted records per slot
    if (c.exact_current != 0 && (c.exact_current != 1 || c.geom != PIC_GEOM_CARTESIAN ||
                                 c.precision != PIC_PREC_FP64 || c.capacity >= (1ll << 31)))
        return PIC_ERR_INVALID;
    if (c.fdtd != PIC_FDTD_YEE && c.fdtd != PIC_FDTD_LEHE) return PIC_ERR_INVALID;
    if (c.fp64_tiles < -1 || c.fp64_tiles > 1) return PIC_ERR_INVALID;
    if (c.exact_charge != 0 && (c.exact_charge != 1 || c.precision != PIC_PREC_FP32 || c.geom != PIC_GEOM_CARTESIAN))
        return PIC_ERR_INVALID;
    if (c.precision != PIC_PREC_FP64 && c.precision != PIC_PREC_FP32) return PIC_ERR_INVALID;
    if (c.nx < 5 || c.ny < 5 || (c.dims == 3 && c.nz < 5)) return PIC_ERR_INVALID;
    if (c.nflvr < 1 || c.nflvr > PIC_MAX_FLVR) return PIC_ERR_INVALID;
    if (!(c.c > 0.0 && c.c < 1.0) || c.capacity < 1 || c.capacity >= (1ll << 32) - 1) return PIC_ERR_INVALID;
    if (c.curr_filter < 0 || c.reorder_period < 0) return PIC_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return PIC_ERR_NOGPU;
    }
    pic_handle *h = new pic_handle();
    h->cfg = c;
    h->fp32 = c.precision == PIC_PREC_FP32;
    GridP &g = h->g;
    std::memset(&g, 0, sizeof(g));
    g.dims = c.dims;
    g.nx = c.nx;
    g.ny = c.ny;
    g.nz = c.dims == 3 ? c.nz : 1;
    g.mx = c.nx + 5;
    g.my = c.ny + 5;
    g.mz = c.dims == 3 ? c.nz + 5 : 1;
    g.fdtd = c.fdtd;
    g.sy = g.mx;
    g.sz = (long long)g.mx * g.my;
    g.ncell = g.sz * g.mz;
    div_magic((unsigned)g.mx, g.mx_magic, g.mx_shift);
    div_magic((unsigned)g.my, g.my_magic, g.my_shift);
    if (g.ncell >= (1ll << kFlvShift) - 1 || g.mx > 4096 || g.my > 4096) {
        delete h;
        return PIC_ERR_INVALID;
    }
    g.c = c.c;
    g.h = (c.c * 0.5) * 1.0;   // fld_halfc, vars.F90:221
    g.fc = c.c * 1.0;          // fldc, vars.F90:220
    g.sqc = c.c * c.c;         // vars.F90:223
    g.cinv = 1.0 / c.c;        // vars.F90:222
    g.qi = c.qi;
    for (int d = 0; d < 3; d++) g.bext[d] = c.bext[d];
    if (c.geom == PIC_GEOM_CYLINDRICAL) cyl_lehe_coefficients(c.c, c.ny, g.lehe);
    else lehe_coefficients(c.dims, c.c, g.lehe);
    g.geom = c.geom;
    // a cylinder's x faces: the axis and the outer radius have no neighbour;
    // a slab exchanges the others
    g.closed_x = c.geom != PIC_GEOM_CYLINDRICAL ? 0
                 : c.slab_x == 0                ? 3
                                                : (c.inc_axis ? 1 : 0) | (c.slab_x == 2 ? 2 : 0);
    g.inc_axis = c.geom == PIC_GEOM_CYLINDRICAL && c.inc_axis;
    g.rmin = c.rmin;
    g.x_external = c.slab_x != 0;
    g.exact_charge = c.exact_charge != 0;
    g.qm[0] = 0.0;
    for (int f = 1; f <= PIC_MAX_FLVR; f++) g.qm[f] = f <= c.nflvr ? c.qm[f] : 0.0;
    g.c_f = (float)g.c;
    g.sqc_f = (float)g.sqc;
    g.cinv_f = (float)g.cinv;
    g.qi_f = (float)g.qi;
    for (int d = 0; d < 3; d++) g.bext_f[d] = (float)g.bext[d];
    for (int f = 0; f <= PIC_MAX_FLVR; f++) g.qm_half_f[f] = (float)g.qm[f] * 0.5f;
    // subdomains.F90:52-67
    g.xmin = 3.0;
    g.xmax = (double)(g.mx - 2);
    g.ymin = 3.0;
    g.ymax = (double)(g.my - 2);
    g.zmin = c.dims == 3 ? 3.0 : 1.0;
    g.zmax = c.dims == 3 ? (double)(g.mz - 2) : 2.0;
    g.xlen = g.xmax - g.xmin;
    g.ylen = g.ymax - g.ymin;
    g.zlen = g.zmax - g.zmin;
    h->capacity = c.capacity;

    int r = PIC_OK;
    if (cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking) != cudaSuccess) r = PIC_ERR_CUDA;
    const size_t fb = field_bytes(h);
    for (int k = 0; k < 3 && !r; k++) {
        if ((r = dalloc(h, (char **)&h->E[k], fb))) break;
        if ((r = dalloc(h, (char **)&h->B[k], fb))) break;
        if ((r = dalloc(h, (char **)&h->J[k], fb))) break;
    }
    if (!r && c.curr_filter > 0) r = dalloc(h, (char **)&h->Jtmp, fb);
    if (!r && c.cyl_modes == 2) {
        h->modal = true;
        const size_t nm = (size_t)g.mx * 3 * (size_t)g.mz, esz = h->fp32 ? sizeof(float) : sizeof(double);
        for (int k = 0; k < 3 && !r; k++)
            if ((r = dalloc(h, (char **)&h->Em[k], nm * esz)) || (r = dalloc(h, (char **)&h->Bm[k], nm * esz)) ||
                (r = dalloc(h, (char **)&h->Jm[k], nm * esz)))
                break;
        for (int k = 0; k < 3 && !r; k++) {
            cudaMemsetAsync(h->Em[k], 0, nm * esz, h->s);
            cudaMemsetAsync(h->Bm[k], 0, nm * esz, h->s);
            cudaMemsetAsync(h->Jm[k], 0, nm * esz, h->s);
        }
    }
    if (!r) r = alloc_particles(h);
    if (!r && h->fp32) {
        // bricks sized for the configured fill (capacity / interior cells)
        Bricks &bk = h->bricks;
        if (!choose_bricks(g, (double)h->capacity / ((double)g.nx * g.ny * g.nz), c.brick, bk)) r = PIC_ERR_INVALID;
        const size_t nt = (size_t)bk.ntiles;
        if (r || (r = dalloc(h, &bk.tile_start, nt + 1)) || (r = dalloc(h, &bk.box, 8 * nt)) ||
            (r = dalloc(h, &bk.count, nt + 1)) || (r = dalloc(h, &bk.cursor, nt)) ||
            (r = dalloc(h, &bk.bid, (size_t)h->capacity)) || (r = dalloc(h, &bk.src, (size_t)h->capacity)) ||
            (r = dalloc(h, &bk.scan_tmp, scan_tmp_len(nt + 1))) ||
            (r = dalloc(h, &bk.wmax_bits, 1))) {
        }
        // the node averages of the Cartesian tiled mover, computed once per
        // move instead of by every brick for its box
        if (!r && g.geom == PIC_GEOM_CARTESIAN &&
            !(r = dalloc(h, (char **)&bk.nodeA, (size_t)g.ncell * sizeof(float4))))
            r = dalloc(h, (char **)&bk.nodeB, (size_t)g.ncell * sizeof(float2));
    }
    if (!r) r = dalloc(h, &h->cnt, 1);
    if (!r) r = dalloc(h, &h->err, 1);
    if (!r && c.slab_x) r = dalloc(h, &h->slab_sent, 2);
    if (!r) {
        SortScratch &sc = h->sc;
        sc.ntiles = sort_tiles(h->capacity);
        sc.scan_tmp_len = scan_tmp_len(256 * sc.ntiles);
        // radix-sort keys and indices: the FP64 reorder only
        const size_t nk = h->fp32 ? 1 : (size_t)h->capacity;
        if ((r = dalloc(h, &sc.key[0], nk)) || (r = dalloc(h, &sc.key[1], nk)) || (r = dalloc(h, &sc.idx[0], nk)) ||
            (r = dalloc(h, &sc.idx[1], nk)) || (r = dalloc(h, &sc.hist, 256 * sc.ntiles)) ||
            (r = dalloc(h, &sc.scan_tmp, sc.scan_tmp_len))) {
        }
    }
    // the tiles of the FP64 movers (faster than the per-particle mover's
    // global FP64 atomics on every grid measured: 0.15 against 0.26 ms per
    // move on the 256^2 grid of 2.1 M particles, 44 against 69 ms on
    // 512 x 256 x 256); the exact-order current keeps the per-particle
    // mover, whose records it sorts anyway
    if (!r && (c.geom == PIC_GEOM_CARTESIAN || c.geom == PIC_GEOM_CYLINDRICAL) && c.precision == PIC_PREC_FP64 &&
        !c.exact_current && c.fp64_tiles >= 0) {
        Tiles64 &T = h->t64;
        choose_tiles64(g, T);
        if (!(r = dalloc(h, &T.range, 2 * (size_t)T.H * (size_t)T.D * (size_t)T.ntiles)) &&
            !(r = dalloc(h, &T.box, 8 * (size_t)T.ntiles)) && !(r = dalloc(h, &T.np, 1)) &&
            !(r = dalloc(h, &T.qmax, 1)))
            h->tiled64 = true;
    }
    if (!r && c.exact_current) {
        SegRecords &R = h->rec;
        h->exact = true;
        R.n2 = 2 * h->capacity;
        R.sc.ntiles = sort_tiles(R.n2);
        R.sc.scan_tmp_len = scan_tmp_len(256 * R.sc.ntiles);
        const size_t ne = g.dims == 3 ? 12 : 8;
        if ((r = dalloc(h, &R.sc.key[0], (size_t)R.n2)) || (r = dalloc(h, &R.sc.key[1], (size_t)R.n2)) ||
            (r = dalloc(h, &R.sc.idx[0], (size_t)R.n2)) || (r = dalloc(h, &R.sc.idx[1], (size_t)R.n2)) ||
            (r = dalloc(h, &R.sc.hist, 256 * R.sc.ntiles)) || (r = dalloc(h, &R.sc.scan_tmp, R.sc.scan_tmp_len)) ||
            (r = dalloc(h, &R.val, ne * (size_t)R.n2)) || (r = dalloc(h, &R.vecj, ne * (size_t)g.ncell)) ||
            (r = dalloc(h, &R.count, 1))) {
        }
    }
    if (!r) {
        h->diag_blocks = field_energy_blocks(g);
        if (!(r = dalloc(h, &h->diag_partials, 2 * (size_t)h->diag_blocks))) r = dalloc(h, &h->diag_out, 64);
    }
    if (!r) {
        std::vector<double> X, P;
        maxbolt_table(h->ntab, X, P);
        if (!(r = dalloc(h, &h->tab_x, h->ntab)) && !(r = dalloc(h, &h->tab_p, h->ntab))) {
            cudaMemcpy(h->tab_x, X.data(), X.size() * sizeof(double), cudaMemcpyHostToDevice);
            cudaMemcpy(h->tab_p, P.data(), P.size() * sizeof(double), cudaMemcpyHostToDevice);
        }
    }
    if (!r) {
        for (int k = 0; k < 3; k++) {
            cudaMemsetAsync(h->E[k], 0, fb, h->s);
            cudaMemsetAsync(h->B[k], 0, fb, h->s);
            cudaMemsetAsync(h->J[k], 0, fb, h->s);
        }
        cudaMemsetAsync(h->cnt, 0, sizeof(Counters), h->s);
        cudaMemsetAsync(h->err, 0, sizeof(int), h->s);
        r = finish(h);
    }
    if (r) {
        pic_destroy(h);
        return r;
    }
    *out = h;
    return PIC_OK;
}

void *pic_stream(pic_handle *h) { return h ? (void *)h->s : nullptr; }

int pic_load_fields(pic_handle *h, const double *Ex, const double *Ey, const double *Ez, const double *Bx,
                    const double *By, const double *Bz)
{
    if (!h) return PIC_ERR_INVALID;
    const double *src[6] = {Ex, Ey, Ez, Bx, By, Bz};
    void *dst[6] = {h->E[0], h->E[1], h->E[2], h->B[0], h->B[1], h->B[2]};
    const size_t n = (size_t)h->g.ncell;
    if (h->fp32) {
        int r = ensure_stage(h);
        if (r) return r;
    }
    int seq = 0;   // running chunk number: staging buffer seq % 2
    for (int k = 0; k < 6; k++) {
        if (!src[k]) continue;
        if (!h->fp32) {
            CK(cudaMemcpyAsync(dst[k], src[k], n * sizeof(double), cudaMemcpyHostToDevice, h->s));
        } else {
            int r = load_array_f32(h, src[k], (float *)dst[k], (long long)n, seq);
            if (r) return r;
        }
    }
    if (h->modal) {   // the modes m = 0, 1 of the loaded fields; E, B become their synthesis
        if (h->fp32) modal_load<float>(h);
        else modal_load<double>(h);
    }
    int r = sync_both(h);
    if (r) return r;
    return finish(h);
}

int pic_load_current(pic_handle *h, const double *Jx, const double *Jy, const double *Jz)
{
    if (!h) return PIC_ERR_INVALID;
    const double *src[3] = {Jx, Jy, Jz};
    const size_t n = (size_t)h->g.ncell;
    if (h->fp32) {
        int r = ensure_stage(h);
        if (r) return r;
    }
    int seq = 0;   // running chunk number: staging buffer seq % 2
    for (int k = 0; k < 3; k++) {
        if (!src[k]) continue;
        if (!h->fp32) {
            CK(cudaMemcpyAsync(h->J[k], src[k], n * sizeof(double), cudaMemcpyHostToDevice, h->s));
        } else {
            int r = load_array_f32(h, src[k], (float *)h->J[k], (long long)n, seq);
            if (r) return r;
        }
    }
    int r = sync_both(h);
    if (r) return r;
    return finish(h);
}

int pic_fetch_fields(pic_handle *h, double *Ex, double *Ey, double *Ez, double *Bx, double *By, double *Bz, double *Jx,
                     double *Jy, double *Jz)
{
    if (!h) return PIC_ERR_INVALID;
    double *dst[9] = {Ex, Ey, Ez, Bx, By, Bz, Jx, Jy, Jz};
    void *src[9] = {h->E[0], h->E[1], h->E[2], h->B[0], h->B[1], h->B[2], h->J[0], h->J[1], h->J[2]};
    const size_t n = (size_t)h->g.ncell;
    if (h->fp32) {
        int r = ensure_stage(h);
        if (r) return r;
    }
    int seq = 0;   // running chunk number: staging buffer seq % 2
    for (int k = 0; k < 9; k++) {
        if (!dst[k]) continue;
        if (!h->fp32) {
            CK(cudaMemcpyAsync(dst[k], src[k], n * sizeof(double), cudaMemcpyDeviceToHost, h->s));
        } else {
            int r = fetch_array_f32(h, (const float *)src[k], dst[k], (long long)n, seq);
            if (r) return r;
        }
    }
    int r = sync_both(h);
    if (r) return r;
    return finish(h);
}

int pic_particle_count(pic_handle *h, int64_t *used)
{
    if (!h || !used) return PIC_ERR_INVALID;
    long long u = 0;
    CK(cudaMemcpyAsync(&u, &h->cnt->used, sizeof(long long), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    *used = u;
    return PIC_OK;
}

int pic_load_particles(pic_handle *h, int64_t n, const double *q, const double *x, const double *y, const double *z,
                       const double *u, const double *v, const double *w, const int32_t *flv)
{
    if (!h || n < 0 || n > h->capacity || (n > 0 && (!q || !x || !y || !z || !u || !v || !w || !flv)))
        return PIC_ERR_INVALID;
    const double *src[7] = {q, x, y, z, u, v, w};
    if (!h->fp32) {
        PartF64 &p = h->p64[h->cur];
        double *dst[7] = {p.q, p.x, p.y, p.z, p.u, p.v, p.w};
        for (int k = 0; k < 7; k++)
            if (n) CK(cudaMemcpyAsync(dst[k], src[k], (size_t)n * sizeof(double), cudaMemcpyHostToDevice, h->s));
        if (n) CK(cudaMemcpyAsync(p.flv, flv, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, h->s));
    } else if (n > 0) {
        // chunk k: copies on the copy stream into staging buffer k%2 while
        // chunk k-1 converts on h->s
        int r = ensure_stage(h);
        if (r) return r;
        const long long chunk = stage_particle_chunk(h);
        int k = 0;
        for (long long o = 0; o < n; o += chunk, k++) {
            const int b = k & 1;
            const long long m = (n - o) < chunk ? (n - o) : chunk;
            const PartF64 t = stage_particles(h, b, chunk);
            double *dst[7] = {t.q, t.x, t.y, t.z, t.u, t.v, t.w};
            CK(cudaStreamWaitEvent(h->cs, h->ev_done[b], 0));
            for (int a = 0; a < 7; a++)
                CK(cudaMemcpyAsync(dst[a], src[a] + o, (size_t)m * sizeof(double), cudaMemcpyHostToDevice, h->cs));
            CK(cudaMemcpyAsync(t.flv, flv + o, (size_t)m * sizeof(int32_t), cudaMemcpyHostToDevice, h->cs));
            CK(cudaEventRecord(h->ev_copied[b], h->cs));
            CK(cudaStreamWaitEvent(h->s, h->ev_copied[b], 0));
            PartF32 d = h->p32[h->cur];
            d.key += o; d.dx += o; d.dy += o; if (d.dz) d.dz += o;
            d.ux += o; d.uy += o; d.uz += o; d.w += o;
            launch_f64_to_f32(h->g, t, d, m, h->err, h->s);
            CK(cudaEventRecord(h->ev_done[b], h->s));
        }
        r = sync_both(h);
        if (r) return r;
    }
    Counters c0 = {};
    c0.used = n;
    c0.np = n;
    CK(cudaMemcpyAsync(h->cnt, &c0, sizeof(Counters), cudaMemcpyHostToDevice, h->s));
    set_sorted(h, false);
    return finish(h);
}

int pic_fetch_particles(pic_handle *h, int64_t *nout, double *q, double *x, double *y, double *z, double *u, double *v,
                        double *w, int32_t *flv)
{
    if (!h) return PIC_ERR_INVALID;
    int64_t n = 0;
    int r = pic_particle_count(h, &n);
    if (r) return r;
    if (nout) *nout = n;
    double *dst[7] = {q, x, y, z, u, v, w};
    if (!h->fp32) {
        PartF64 &p = h->p64[h->cur];
        const double *src[7] = {p.q, p.x, p.y, p.z, p.u, p.v, p.w};
        for (int k = 0; k < 7; k++)
            if (dst[k] && n) CK(cudaMemcpyAsync(dst[k], src[k], (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, h->s));
        if (flv && n) CK(cudaMemcpyAsync(flv, p.flv, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, h->s));
    } else if (n > 0) {
        // chunk k: converts on h->s into staging buffer k%2 while chunk k-1
        // copies out on the copy stream
        r = ensure_stage(h);
        if (r) return r;
        const long long chunk = stage_particle_chunk(h);
        int k = 0;
        for (long long o = 0; o < n; o += chunk, k++) {
            const int b = k & 1;
            const long long m = (n - o) < chunk ? (n - o) : chunk;
            const PartF64 t = stage_particles(h, b, chunk);
            PartF32 sp = h->p32[h->cur];
            sp.key += o; sp.dx += o; sp.dy += o; if (sp.dz) sp.dz += o;
            sp.ux += o; sp.uy += o; sp.uz += o; sp.w += o;
            CK(cudaStreamWaitEvent(h->s, h->ev_copied[b], 0));
            launch_f32_to_f64(h->g, sp, t, m, h->s);
            CK(cudaEventRecord(h->ev_done[b], h->s));
            CK(cudaStreamWaitEvent(h->cs, h->ev_done[b], 0));
            const double *src[7] = {t.q, t.x, t.y, t.z, t.u, t.v, t.w};
            for (int a = 0; a < 7; a++)
                if (dst[a]) CK(cudaMemcpyAsync(dst[a] + o, src[a], (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, h->cs));
            if (flv) CK(cudaMemcpyAsync(flv + o, t.flv, (size_t)m * sizeof(int32_t), cudaMemcpyDeviceToHost, h->cs));
            CK(cudaEventRecord(h->ev_copied[b], h->cs));
        }
        r = sync_both(h);
        if (r) return r;
    }
    return finish(h);
}

int pic_init_weibel(pic_handle *h, double epc, double density, double drift, double temp_ion, double temp_elc,
                    uint32_t seed)
{
    if (!h || !(epc > 0) || h->cfg.nflvr < 2) return PIC_ERR_INVALID;
    WeibelParams w;
    w.epc = epc;
    w.density = density;
    w.drift = drift;
    w.temp[0] = temp_ion;
    w.temp[1] = temp_elc;
    w.seed = seed;
    w.sgn_out = nullptr;
    // init_prtl.F90:190: Nprtl = epc * (x2-x1)*(y2-y1)*(z2-z1), truncated
    const double vol = (double)h->g.nx * (double)h->g.ny * (h->g.dims == 3 ? (double)h->g.nz : 1.0);
    w.ntrial = (long long)(epc * vol);
    if (w.ntrial <= 0 || 2 * w.ntrial >= (1ll << 32)) return PIC_ERR_INVALID;
    const PartF64 *p64 = h->fp32 ? nullptr : &h->p64[h->cur];
    const PartF32 *p32 = h->fp32 ? &h->p32[h->cur] : nullptr;
    CK(cudaMemsetAsync(h->cnt, 0, sizeof(Counters), h->s));
    set_sorted(h, false);
    int r = launch_weibel(h->g, w, h->tab_x, h->tab_p, h->ntab, p64, p32, h->cnt, h->sc, h->capacity, h->err, h->s);
    if (r) return r;
    return finish(h);
}

// --- phases --------------------------------------------------------------

int pic_update_b_half(pic_handle *h)
{
    if (!h) return PIC_ERR_INVALID;
    if (h->modal) {
        if (h->fp32) modal_bhalf<float>(h);
        else modal_bhalf<double>(h);
    } else if (h->g.geom == PIC_GEOM_CYLINDRICAL && h->fp32) {
        float *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_cyl_bhalf<float>(h->g, E, B, h->s);
    } else if (h->g.geom == PIC_GEOM_CYLINDRICAL) {
        double *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_cyl_bhalf(h->g, E, B, h->s);
    } else if (h->fp32) {
        float *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_bhalf<float>(h->g, E, B, h->s);
    } else {
        double *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_bhalf<double>(h->g, E, B, h->s);
    }
    return finish_phase(h);
}

int pic_reset_current(pic_handle *h)
{
    if (!h) return PIC_ERR_INVALID;
    for (int k = 0; k < 3; k++) CK(cudaMemsetAsync(h->J[k], 0, field_bytes(h), h->s));
    return finish_phase(h);
}

int pic_move_deposit(pic_handle *h)
{
    if (!h) return PIC_ERR_INVALID;
    for (int k = 0; k < 3; k++) CK(cudaMemsetAsync(h->J[k], 0, field_bytes(h), h->s));
    if (h->g.geom == PIC_GEOM_CYLINDRICAL && h->fp32) {
        float *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        if (h->sorted)
            launch_cyl_move_deposit_f32_tiled(h->g, h->p32[h->cur], h->bricks, E, B, J, h->err, h->s);
        else
            launch_cyl_move_deposit_f32(h->g, h->p32[h->cur], h->cnt, E, B, J, h->err, h->s);
    } else if (h->g.geom == PIC_GEOM_CYLINDRICAL) {
        double *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_cyl_move_deposit(h->g, h->p64[h->cur], h->cnt, E, B, J, h->err, h->s,
                                h->tiled64 && h->sorted ? &h->t64 : nullptr);
    } else if (h->fp32) {
        float *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        if (h->sorted)
            launch_move_deposit_f32_tiled(h->g, h->p32[h->cur], h->bricks, h->cnt, E, B, J, h->err, h->s);
        else
            launch_move_deposit_f32(h->g, h->p32[h->cur], h->cnt, E, B, J, h->err, h->s);
    } else {
        double *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        if (h->tiled64 && h->sorted)
            launch_move_deposit_f64_tiled(h->g, h->p64[h->cur], h->cnt, h->t64, E, B, J, h->err, h->s);
        else
            launch_move_deposit_f64(h->g, h->p64[h->cur], h->cnt, E, B, J, h->err, h->s,
                                    h->exact ? &h->rec : nullptr);
    }
    return finish_phase(h);
}

int pic_exchange_particles(pic_handle *h)
{
    if (!h || h->g.x_external) return PIC_ERR_INVALID;   // a slab exchanges through pic_slab_pack_particles
    if (!h->fp32) launch_exchange_f64(h->g, h->p64[h->cur], h->cnt, h->sc, h->capacity, h->err, h->s);
    return finish_phase(h);
}

int pic_update_e(pic_handle *h)
{
    if (!h) return PIC_ERR_INVALID;
    if (h->modal) {
        if (h->fp32) modal_update_e<float>(h);
        else modal_update_e<double>(h);
    } else if (h->g.geom == PIC_GEOM_CYLINDRICAL && h->fp32) {
        float *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_cyl_efield<float>(h->g, 0, E, B, J, h->s);
    } else if (h->g.geom == PIC_GEOM_CYLINDRICAL) {
        double *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_cyl_efield(h->g, 0, E, B, J, h->s);
    } else if (h->fp32) {
        float *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_efield<float>(h->g, 0, E, B, J, h->s);
    } else {
        double *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_efield<double>(h->g, 0, E, B, J, h->s);
    }
    return finish_phase(h);
}

int pic_fold_current(pic_handle *h)
{
    if (!h) return PIC_ERR_INVALID;
    if (h->g.geom == PIC_GEOM_CYLINDRICAL && h->fp32) {
        float *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_cyl_fold<float>(h->g, J, h->s);
    } else if (h->g.geom == PIC_GEOM_CYLINDRICAL) {
        double *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_cyl_fold(h->g, J, h->s);
    } else if (h->fp32) {
        float *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_fold<float>(h->g, J, h->s);
    } else {
        double *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_fold<double>(h->g, J, h->s);
    }
    return finish_phase(h);
}

int pic_filter_current(pic_handle *h)
{
    if (!h || h->g.geom == PIC_GEOM_CYLINDRICAL) return PIC_ERR_INVALID;
    if (!h->Jtmp) {
        int r = dalloc(h, (char **)&h->Jtmp, field_bytes(h));
        if (r) return r;
    }
    for (int k = 0; k < h->cfg.curr_filter; k++) {
        if (h->fp32) {
            float *E[3], *B[3], *J[3];
            field_ptrs(h, E, B, J);
            launch_filter<float>(h->g, J, (float *)h->Jtmp, h->s);
        } else {
            double *E[3], *B[3], *J[3];
            field_ptrs(h, E, B, J);
            launch_filter<double>(h->g, J, (double *)h->Jtmp, h->s);
        }
    }
    return finish_phase(h);
}

int pic_add_current(pic_handle *h)
{
    if (!h) return PIC_ERR_INVALID;
    if (h->modal) {
        if (h->fp32) modal_add_current<float>(h);
        else modal_add_current<double>(h);
    } else if (h->g.geom == PIC_GEOM_CYLINDRICAL && h->fp32) {
        float *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_cyl_efield<float>(h->g, 2, E, B, J, h->s);
    } else if (h->g.geom == PIC_GEOM_CYLINDRICAL) {
        double *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_cyl_efield(h->g, 2, E, B, J, h->s);
    } else if (h->fp32) {
        float *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_efield<float>(h->g, 2, E, B, J, h->s);
    } else {
        double *E[3], *B[3], *J[3];
        field_ptrs(h, E, B, J);
        launch_efield<double>(h->g, 2, E, B, J, h->s);
    }
    return finish_phase(h);
}

int pic_bc_reflect_x(pic_handle *h, int32_t side, double pos)
{
    if (!h || h->fp32 || h->g.geom != PIC_GEOM_CARTESIAN || h->g.x_external || (side != 0 && side != 1))
        return PIC_ERR_INVALID;
    double *E[3], *B[3], *J[3];
    field_ptrs(h, E, B, J);
    launch_wall_reflect(h->g, h->p64[h->cur], h->cnt, J, side, pos, h->capacity, h->s);
    return finish_phase(h);
}

int pic_bc_conducting_x(pic_handle *h, int32_t side, double pos)
{
    if (!h || h->fp32 || h->g.geom != PIC_GEOM_CARTESIAN || h->g.x_external || (side != 0 && side != 1))
        return PIC_ERR_INVALID;
    double *E[3], *B[3], *J[3];
    field_ptrs(h, E, B, J);
    launch_wall_conducting(h->g, E, side, pos, h->s);
    return finish_phase(h);
}

int pic_bc_reflect_y(pic_handle *h, int32_t side, double pos)
{
    if (!h || h->fp32 || h->g.geom != PIC_GEOM_CARTESIAN || (side != 0 && side != 1)) return PIC_ERR_INVALID;
    double *E[3], *B[3], *J[3];
    field_ptrs(h, E, B, J);
    launch_wall_reflect_y(h->g, h->p64[h->cur], h->cnt, J, side, pos, h->capacity, h->s);
    return finish_phase(h);
}

int pic_bc_conducting_y(pic_handle *h, int32_t side, double pos)
{
    if (!h || h->fp32 || h->g.geom != PIC_GEOM_CARTESIAN || (side != 0 && side != 1)) return PIC_ERR_INVALID;
    double *E[3], *B[3], *J[3];
    field_ptrs(h, E, B, J);
    launch_wall_conducting_y(h->g, E, side, pos, h->s);
    return finish_phase(h);
}

int pic_bc_remove(pic_handle *h, int32_t face, double pos)
{
    if (!h || h->fp32 || h->g.geom != PIC_GEOM_CARTESIAN || face < 1 || face > 6 || (h->g.dims == 2 && face > 4) ||
        (h->g.x_external && face <= 2))
        return PIC_ERR_INVALID;
    launch_wall_remove(h->g, h->p64[h->cur], h->cnt, face, pos, h->capacity, h->s);
    return finish_phase(h);
}

int pic_bc_attenuate(pic_handle *h, int32_t faces, const double *pos, const double *scale)
{
    if (!h || h->fp32 || h->g.geom != PIC_GEOM_CARTESIAN || h->g.x_external || !pos || !scale || faces < 0 ||
        faces > 63 || (h->g.dims == 2 && (faces & 48)))
        return PIC_ERR_INVALID;
    for (int n = 0; n < 6; n++)
        if (((faces >> n) & 1) && !(scale[n] > 0.0)) return PIC_ERR_INVALID;
    double *E[3], *B[3], *J[3];
    field_ptrs(h, E, B, J);
    launch_bc_attenuate(h->g, E, B, faces, pos, scale, h->s);
    return finish_phase(h);
}

int pic_bc_attenuate_flow(pic_handle *h, int32_t face, double pos, double thickness, double scale,
                          const double *bflow, const double *drift)
{
    if (!h || h->fp32 || h->g.geom != PIC_GEOM_CARTESIAN || face < 1 || face > 4 || !bflow || !drift ||
        !(scale > 0.0) || !(thickness >= 0.0) || (h->g.x_external && face <= 2))
        return PIC_ERR_INVALID;
    double *E[3], *B[3], *J[3];
    field_ptrs(h, E, B, J);
    launch_bc_attenuate_flow(h->g, E, B, face, pos, thickness, scale, bflow, drift, h->s);
    return finish_phase(h);
}

int pic_bc_open_x(pic_handle *h, int32_t side, double pos)
{
    if (!h || h->fp32 || h->g.geom != PIC_GEOM_CARTESIAN || h->g.x_external || (side != 0 && side != 1))
        return PIC_ERR_INVALID;
    double *E[3], *B[3], *J[3];
    field_ptrs(h, E, B, J);
    launch_bc_open_fld_x(h->g, E, B, side, pos, h->s);
    return finish_phase(h);
}

int pic_bc_open_prtl_x(pic_handle *h, int32_t side, double pos)
{
    if (!h || h->fp32 || h->g.geom != PIC_GEOM_CARTESIAN || h->g.x_external || (side != 0 && side != 1))
        return PIC_ERR_INVALID;
    if (!h->open_col) {
        const int r = dalloc(h, &h->open_col, 2 * (size_t)h->g.my * (size_t)h->g.mz);
        if (r) return r;
    }
    SortScratch &sc = h->sc;
    launch_bc_open_prtl_x(h->g, h->p64[h->cur], h->cnt, side, pos, h->open_col, sc.key[0], sc.hist, sc.scan_tmp,
                          sc.scan_tmp + sc.scan_tmp_len - 1, h->capacity, h->err, h->s);
    return finish_phase(h);
}

int pic_bc_pml(pic_handle *h, int32_t faces, const double *pos, const double *thickness)
{
    if (!h || h->g.geom != PIC_GEOM_CARTESIAN || h->g.x_external || h->modal || faces < 0 || faces > 63 ||
        (h->g.dims == 2 && (faces & 0x30)) || (faces && (!pos || !thickness)))
        return PIC_ERR_INVALID;
    for (int f = 0; f < 6; f++)
        if (((faces >> f) & 1) && !(thickness[f] > 0.0 && std::fabs(pos[f]) < 1e9)) return PIC_ERR_INVALID;
    const GridP &g = h->g;
    const size_t rows = (size_t)g.mx + g.my + g.mz;
    std::vector<double> coef(6 * rows);
    std::vector<uint8_t> flag(rows);
    h->pml_on = faces != 0 && pml_tables(g, faces, pos, thickness, coef.data(), flag.data());
    if (!h->pml_on) return PIC_OK;
    if (!h->pml_psi) {   // InitPMLArr: zeroed on first use
        const size_t bytes = 12 * (size_t)g.ncell * (h->fp32 ? sizeof(float) : sizeof(double));
        int r = dalloc(h, &h->pml_coef, 6 * rows);
        if (!r) r = dalloc(h, &h->pml_flag, rows);
        if (!r) r = dalloc(h, reinterpret_cast<uint8_t **>(&h->pml_psi), bytes);
        if (r) {
            h->pml_on = false;
            return r;
        }
        CK(cudaMemsetAsync(h->pml_psi, 0, bytes, h->s));
    }
    CK(cudaMemcpyAsync(h->pml_coef, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, h->s));
    CK(cudaMemcpyAsync(h->pml_flag, flag.data(), flag.size(), cudaMemcpyHostToDevice, h->s));
    return finish(h);   // the host tables go out of scope
}

static int pml_phase(pic_handle *h, int which)
{
    if (!h || h->g.geom != PIC_GEOM_CARTESIAN || h->g.x_external || h->modal) return PIC_ERR_INVALID;
    if (!h->pml_on) return PIC_OK;
    const GridP &g = h->g;
    PmlP P;
    int off = 0;
    const int m[3] = {g.mx, g.my, g.mz};
    for (int a = 0; a < 3; a++) {
        P.coef[a] = h->pml_coef + 6 * (size_t)off;
        P.flag[a] = h->pml_flag + off;
        off += m[a];
    }
    P.fc = g.fc;
    if (h->fp32) {
        float *E[3], *B[3], *J[3], *psi[6];
        field_ptrs(h, E, B, J);
        for (int c = 0; c < 6; c++) psi[c] = (float *)h->pml_psi + (size_t)(which == 0 ? 6 + c : c) * g.ncell;
        launch_pml<float>(g, P, which, E, B, psi, h->s);
    } else {
        double *E[3], *B[3], *J[3], *psi[6];
        field_ptrs(h, E, B, J);
        for (int c = 0; c < 6; c++) psi[c] = (double *)h->pml_psi + (size_t)(which == 0 ? 6 + c : c) * g.ncell;
        launch_pml<double>(g, P, which, E, B, psi, h->s);
    }
    return finish_phase(h);
}

int pic_bc_pml_b(pic_handle *h) { return pml_phase(h, 0); }
int pic_bc_pml_e(pic_handle *h) { return pml_phase(h, 1); }

int pic_bc_inflow_reflect(pic_handle *h, double pos, double drift_x)
{
    if (!h || h->fp32 || h->g.geom != PIC_GEOM_CARTESIAN || h->g.x_external || !(fabs(drift_x) < 1e300))
        return PIC_ERR_INVALID;
    double *E[3], *B[3], *J[3];
    field_ptrs(h, E, B, J);
    launch_bc_inflow_reflect(h->g, h->p64[h->cur], h->cnt, J, pos, drift_x, h->capacity, h->err, h->s);
    return finish_phase(h);
}

// Philox-4x32-10 on the host (the draw of the injection's Poisson count).
static void host_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c0 = n0;
        c1 = (uint32_t)p1;
        c2 = n2;
        c3 = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

int pic_bc_inflow(pic_handle *h, const pic_inflow *inj)
{
    if (!h || !inj || h->fp32 || h->g.geom != PIC_GEOM_CARTESIAN || h->g.x_external) return PIC_ERR_INVALID;
    const GridP &g = h->g;
    const int side = inj->face;
    if (side < 1 || side > (g.dims == 3 ? 6 : 4) || inj->nspecies < 1 || inj->nspecies > 4 || !(inj->epc > 0.0) ||
        !(inj->density >= 0.0) || !(inj->vmax >= 0.0) || !(inj->speed >= 0.0))
        return PIC_ERR_INVALID;
    for (int sp = 0; sp < inj->nspecies; sp++)
        if (inj->flv[sp] < 1 || inj->flv[sp] > h->cfg.nflvr || !(inj->temp[sp] >= 0.0)) return PIC_ERR_INVALID;
    // SetInjDomain (bc_inflow.F90:191-235) on one rank: the borders of the
    // rank are 0 and n, local = global - 0 + 3; the other axes span
    // xmin..xmax (subdomains.F90:52-66)
    InflowParams f;
    f.x1 = 3.0;
    f.x2 = g.mx - 2;
    f.y1 = 3.0;
    f.y2 = g.my - 2;
    f.z1 = g.dims == 3 ? 3.0 : 1.0;
    f.z2 = g.dims == 3 ? (double)(g.mz - 2) : 2.0;
    const double pos = inj->pos, vc = inj->vmax * g.c, shift = inj->speed * g.c;
    const double n3[3] = {(double)g.nx, (double)g.ny, (double)g.nz};
    double *lo[3] = {&f.x1, &f.y1, &f.z1}, *hi[3] = {&f.x2, &f.y2, &f.z2};
    const int ax = (side - 1) / 2;
    if (side % 2 == 1) {
        *lo[ax] = fmax(pos - shift, 0.0) - 0.0 + 3;
        *hi[ax] = fmin(pos + vc, n3[ax]) - 0.0 + 3;
    } else {
        *lo[ax] = fmax(pos - vc, 0.0) - 0.0 + 3;
        *hi[ax] = fmin(pos + shift, n3[ax]) - 0.0 + 3;
    }
    long long n = (long long)(inj->epc * fmax(0.0, f.x2 - f.x1) * fmax(0.0, f.y2 - f.y1) * fmax(0.0, f.z2 - f.z1));
    if (n <= 0) return PIC_OK;
    if (n < 1000) {
        // GetIntPoissonDist (prob_dist.F90:194-216) with mean n
        const uint32_t ctr[4] = {0xFFFFFFFFu, inj->call, 0u, 0u}, key[2] = {inj->seed, 0x494E4A43u};
        uint32_t r[4];
        host_philox(ctr, key, r);
        const double r1 = (double)((((uint64_t)r[0] << 32) | r[1]) >> 11) * (1.0 / 9007199254740992.0);
        const double mean = (double)n;
        double sum = exp(-mean), sum_logn = 0.0;
        const double log_mean = log(mean);
        long long k = 0;
        while (sum < r1) {
            k = k + 1;
            sum_logn = sum_logn + log((double)k);
            sum = sum + exp(-mean + (double)k * log_mean - sum_logn);
            if (k > 10000) break;
        }
        n = k;
        if (n == 0) return PIC_OK;
    }
    if (n >= (1ll << 31)) return PIC_ERR_INVALID;
    f.density = inj->density;
    for (int d = 0; d < 3; d++) f.drift[d] = inj->drift[d];
    f.c = g.c;
    f.pos = pos;
    f.side = side;
    f.dims = g.dims;
    f.nsp = inj->nspecies;
    for (int sp = 0; sp < 4; sp++) {
        f.flv[sp] = sp < inj->nspecies ? inj->flv[sp] : 0;
        f.temp[sp] = sp < inj->nspecies ? inj->temp[sp] : 0.0;
        f.charge[sp] = sp < inj->nspecies ? inj->charge[sp] : 0.0;
    }
    f.seed = inj->seed;
    f.call = inj->call;
    f.ntrial = n;
    int r = launch_inflow(g, f, h->tab_x, h->tab_p, h->ntab, h->p64[h->cur], h->cnt, h->sc, h->capacity, h->err, h->s);
    if (r) return r;
    return finish_phase(h);
}

int pic_set_sync(pic_handle *h, int32_t sync)
{
    if (!h) return PIC_ERR_INVALID;
    h->sync = sync != 0;
    return h->sync ? finish(h) : PIC_OK;
}

int pic_slab_face_len(pic_handle *h, int64_t *n)
{
    if (!h || !n || !h->g.x_external) return PIC_ERR_INVALID;
    *n = 9ll * h->g.my * h->g.mz;
    return PIC_OK;
}

extern "C++" {
template <typename T>
static void slab_fields(pic_handle *h, int32_t which, bool pack, double *a, double *b)
{
    T *E[3], *B[3], *J[3];
    field_ptrs(h, E, B, J);
    T *const *F = which == 0 ? E : which == 1 ? B : J;
    if (pack) launch_slab_pack_fields<T>(h->g, which, F, a, b, h->s);
    else launch_slab_unpack_fields<T>(h->g, which, F, a, b, h->s);
}
}

int pic_slab_pack_fields(pic_handle *h, int32_t which, double *to_left, double *to_right)
{
    if (!h || !h->g.x_external || which < 0 || which > 2 || !to_left || !to_right) return PIC_ERR_INVALID;
    if (h->fp32) slab_fields<float>(h, which, true, to_left, to_right);
    else slab_fields<double>(h, which, true, to_left, to_right);
    return finish_phase(h);
}

int pic_slab_unpack_fields(pic_handle *h, int32_t which, const double *from_left, const double *from_right)
{
    if (!h || !h->g.x_external || which < 0 || which > 2 || !from_left || !from_right) return PIC_ERR_INVALID;
    if (h->fp32) slab_fields<float>(h, which, false, const_cast<double *>(from_left), const_cast<double *>(from_right));
    else slab_fields<double>(h, which, false, const_cast<double *>(from_left), const_cast<double *>(from_right));
    return finish_phase(h);
}

int pic_slab_pack_particles(pic_handle *h, double *out, int64_t cap, int64_t *n_right, int64_t *n_left)
{
    if (!h || !h->g.x_external || !out || cap < 0 || !n_right || !n_left) return PIC_ERR_INVALID;
    if (h->fp32)
        launch_slab_pack_f32(h->g, h->p32[h->cur], h->cnt, out, cap, h->sc.hist, h->sc.scan_tmp,
                             h->sc.scan_tmp + h->sc.scan_tmp_len - 1, h->slab_sent, h->capacity, h->err, h->s);
    else
        launch_exchange_f64(h->g, h->p64[h->cur], h->cnt, h->sc, h->capacity, h->err, h->s, out, cap, h->slab_sent);
    uint32_t sent[2] = {0, 0};
    *n_right = 0;
    *n_left = 0;
    CK(cudaMemcpyAsync(sent, h->slab_sent, sizeof(sent), cudaMemcpyDeviceToHost, h->s));
    // the counts size the transfers, so this call waits in either sync mode
    // and checks the device error word like a synchronous call: an outbox or
    // capacity overflow (nothing moved, the count unchanged) returns
    // PIC_ERR_OVERFLOW with zero counts instead of counts no buffer holds
    const int r = finish(h);
    if (r != PIC_OK) return r;
    if ((int64_t)sent[1] > cap) return PIC_ERR_OVERFLOW;
    *n_right = sent[0];
    *n_left = (int64_t)sent[1] - (int64_t)sent[0];
    return PIC_OK;
}

int pic_slab_pack_particles_fixed(pic_handle *h, double *to_left, double *to_right, int64_t cap)
{
    if (!h || !h->g.x_external || !to_left || !to_right || cap < 0) return PIC_ERR_INVALID;
    launch_slab_pack_fixed(h->g, h->fp32, h->p64[h->cur], h->p32[h->cur], h->cnt, h->sc, to_left, to_right, cap,
                           h->slab_sent, h->capacity, h->err, h->s);
    return finish_phase(h);
}

int pic_slab_unpack_particles_fixed(pic_handle *h, const double *from_left, const double *from_right, int64_t cap)
{
    if (!h || !h->g.x_external || !from_left || !from_right || cap < 0) return PIC_ERR_INVALID;
    launch_slab_append_fixed(h->g, h->fp32, h->p64[h->cur], h->p32[h->cur], h->cnt, from_left, from_right, cap,
                             h->capacity, h->err, h->s);
    return finish_phase(h);
}

int pic_slab_unpack_particles(pic_handle *h, const double *in, int64_t n)
{
    if (!h || !h->g.x_external || n < 0 || (n > 0 && !in)) return PIC_ERR_INVALID;
    if (h->fp32) launch_slab_append_f32(h->g, h->p32[h->cur], h->cnt, in, n, h->capacity, h->err, h->s);
    else launch_slab_append(h->g, h->p64[h->cur], h->cnt, in, n, h->capacity, h->err, h->s);
    return finish_phase(h);
}

int pic_reorder(pic_handle *h)
{
    if (!h) return PIC_ERR_INVALID;
    if (h->fp32) launch_reorder_f32(h->g, h->p32[h->cur], h->p32[h->cur ^ 1], h->cnt, h->capacity, h->bricks, h->err, h->s);
    else
        launch_reorder_f64(h->g, h->p64[h->cur], h->p64[h->cur ^ 1], h->cnt, h->sc, h->capacity, h->err, h->s,
                           h->tiled64 ? &h->t64 : nullptr);
    h->cur ^= 1;
    set_sorted(h, h->fp32 || h->tiled64);
    return finish_phase(h);
}

int pic_set_step(pic_handle *h, int64_t t)
{
    if (!h) return PIC_ERR_INVALID;
    h->t = t;
    return PIC_OK;
}

int pic_step(pic_handle *h, int32_t nsteps)
{
    // a slab's step has exchanges with its neighbours between the phases
    if (!h || nsteps < 0 || h->g.x_external) return PIC_ERR_INVALID;
    // J must be zero when a deposit starts; inside the loop the E update
    // consumes and clears it.
    for (int k = 0; k < 3; k++) CK(cudaMemsetAsync(h->J[k], 0, field_bytes(h), h->s));
    if (h->profiling) {
        const long long before = [&] { long long n = 0; for (long long v : h->phase_launches) n += v; return n; }();
        int r = step_profiled(h, nsteps);
        long long after = 0;
        for (long long v : h->phase_launches) after += v;
        h->launches += after - before;
        if (r) return r;
        return finish(h);
    }
    for (int32_t i = 0; i < nsteps; i++) {
        int r = enqueue_graph_step(h);
        if (r) return r;
    }
    return finish(h);
}

int pic_step_batched(pic_handle *const *hs, int32_t n, int32_t nsteps)
{
    if (!hs || n < 1 || nsteps < 0) return PIC_ERR_INVALID;
    for (int32_t a = 0; a < n; a++)
        if (!hs[a] || hs[a]->g.x_external) return PIC_ERR_INVALID;
    if (!batchable(hs, n)) return PIC_ERR_INVALID;
    if (nsteps == 0) return PIC_OK;
    return step_many_batched(hs, n, nsteps);
}

static int step_persistent(pic_handle *const *hs, int32_t n, int32_t nsteps, unsigned spin_limit, int force_timeout)
{
    std::lock_guard<std::mutex> lk(g_batch_mu);
    PersistCache &P = g_persist;
    pic_handle *h0 = hs[0];
    cudaStream_t s = h0->s;
    for (int32_t a = 0; a < n; a++) CK(cudaStreamSynchronize(hs[a]->s));
    if (!(P.key.size() == (size_t)n && std::equal(P.key.begin(), P.key.end(), hs))) {
        P.release();
        std::vector<int> starts(2 * ((size_t)n + 1), 0);
        int *fstart = starts.data(), *mstart = starts.data() + n + 1;
        for (int32_t a = 0; a < n; a++) {
            const BatchRun R = batch_run_of(hs[a]);
            fstart[a + 1] = fstart[a] + R.fb[0] * ((R.fb[1] + kPersistFieldRows - 1) / kPersistFieldRows) * R.fb[2];
            mstart[a + 1] = mstart[a] + R.bk.ntiles;
        }
        if (cudaMalloc(&P.druns, sizeof(BatchRun) * (size_t)n) != cudaSuccess ||
            cudaMalloc(&P.dstart, sizeof(int) * starts.size()) != cudaSuccess ||
            cudaMalloc(&P.ctl, sizeof(unsigned) * (3 + 4 * (size_t)n)) != cudaSuccess) {
            P.release();
            return PIC_ERR_OOM;
        }
        CK(cudaMemcpyAsync(P.dstart, starts.data(), sizeof(int) * starts.size(), cudaMemcpyHostToDevice, s));
        P.nf = fstart[n];
        P.nm = mstart[n];
        P.key.assign(hs, hs + n);
    }
    // the descriptors as they are now (each run's current particle buffer)
    {
        std::vector<BatchRun> runs((size_t)n);
        for (int32_t a = 0; a < n; a++) runs[(size_t)a] = batch_run_of(hs[a]);
        CK(cudaMemcpyAsync(P.druns, runs.data(), sizeof(BatchRun) * (size_t)n, cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));
    }
    // the graph of this call: keyed by the steps, the test switches and every
    // run's reorder phase and current buffer
    std::vector<long long> key = {nsteps, (long long)spin_limit, force_timeout};
    for (int32_t a = 0; a < n; a++) {
        const pic_handle *h = hs[a];
        key.push_back(h->cfg.reorder_period > 0 ? h->t % h->cfg.reorder_period : 0);
        key.push_back(h->cur);
    }
    cudaGraphExec_t ge = nullptr;
    long long launches = 0;
    for (auto &g : P.graphs)
        if (g.key == key) {
            ge = g.exec;
            launches = g.launches;
        }
    // the host-side step counters and buffers advance as the sequence does
    std::vector<long long> t((size_t)n);
    std::vector<int> cur((size_t)n);
    for (int32_t a = 0; a < n; a++) {
        t[(size_t)a] = hs[a]->t;
        cur[(size_t)a] = hs[a]->cur;
    }
    auto enqueue = [&]() {
        long long launches = 0;
        for (int32_t done = 0; done < nsteps;) {
            int span = nsteps - done;
            for (int32_t a = 0; a < n; a++) {
                const int per = hs[a]->cfg.reorder_period;
                if (per > 0) span = std::min(span, (int)(per - t[(size_t)a] % per));
            }
            for (int32_t a = 0; a < n; a++)
                for (int k = 0; k < 3 && done == 0; k++) cudaMemsetAsync(hs[a]->J[k], 0, field_bytes(hs[a]), s);
            g_launches = 0;
            launch_ensemble_persistent(h0->g.dims, h0->g.fdtd, h0->g.exact_charge != 0, P.druns, P.dstart,
                                       P.dstart + n + 1, n, span, P.ctl, spin_limit, force_timeout, s);
            launches += g_launches;
            for (int32_t a = 0; a < n; a++) {
                pic_handle *h = hs[a];
                t[(size_t)a] += span;
                if (h->cfg.reorder_period > 0 && t[(size_t)a] % h->cfg.reorder_period == 0) {
                    g_launches = 0;
                    const int c = cur[(size_t)a];
                    launch_reorder_f32(h->g, h->p32[c], h->p32[c ^ 1], h->cnt, h->capacity, h->bricks, h->err, s);
                    launch_batch_flip(P.druns, (int)a, s);
                    launches += g_launches;
                    cur[(size_t)a] ^= 1;
                }
            }
            done += span;
        }
        return launches;
    };
    if (!ge) {
        cudaGraph_t gr = nullptr;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        launches = enqueue();
        const cudaError_t e = cudaStreamEndCapture(s, &gr);
        const cudaError_t ei = e == cudaSuccess ? cudaGraphInstantiate(&ge, gr, 0) : e;
        if (gr) cudaGraphDestroy(gr);
        if (ei != cudaSuccess) return cuda_status(ei);
        P.graphs.push_back({key, ge, launches});
    } else {
        // the host-side counters advance as the captured sequence does
        for (int32_t done = 0; done < nsteps;) {
            int span = nsteps - done;
            for (int32_t a = 0; a < n; a++) {
                const int per = hs[a]->cfg.reorder_period;
                if (per > 0) span = std::min(span, (int)(per - t[(size_t)a] % per));
            }
            for (int32_t a = 0; a < n; a++) {
                t[(size_t)a] += span;
                const int per = hs[a]->cfg.reorder_period;
                if (per > 0 && t[(size_t)a] % per == 0) cur[(size_t)a] ^= 1;
            }
            done += span;
        }
    }
    CK(cudaGraphLaunch(ge, s));
    for (int32_t a = 0; a < n; a++) {
        hs[a]->t = t[(size_t)a];
        hs[a]->cur = cur[(size_t)a];
    }
    h0->launches += launches;
    unsigned status = 0;
    CK(cudaMemcpyAsync(&status, P.ctl + 2, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (status & PIC_DEVERR_TIMEOUT) return PIC_ERR_TIMEOUT;
    int first = PIC_OK;
    for (int32_t a = 0; a < n; a++) {
        const int q = finish(hs[a]);
        if (q && !first) first = q;
    }
    return first;
}

int pic_step_persistent(pic_handle *const *hs, int32_t n, int32_t nsteps, uint32_t spin_limit, int32_t force_timeout)
{
    if (!hs || n < 1 || nsteps < 0) return PIC_ERR_INVALID;
    for (int32_t a = 0; a < n; a++)
        if (!hs[a] || hs[a]->g.x_external || hs[a]->s == nullptr) return PIC_ERR_INVALID;
    if (!batchable(hs, n)) return PIC_ERR_INVALID;
    if (nsteps == 0) return PIC_OK;
    // about one second of polls (each sleeps 200 ns) unless the caller sets it
    return step_persistent(hs, n, nsteps, spin_limit ? spin_limit : 4000000u, force_timeout != 0);
}

int pic_step_many(pic_handle *const *hs, int32_t n, int32_t nsteps)
{
    if (!hs || n < 0 || nsteps < 0) return PIC_ERR_INVALID;
    bool eager = false;
    for (int32_t a = 0; a < n; a++) {
        if (!hs[a] || hs[a]->g.x_external) return PIC_ERR_INVALID;
        eager = eager || hs[a]->profiling;
    }
    if (eager) {
        for (int32_t a = 0; a < n; a++) {
            int r = pic_step(hs[a], nsteps);
            if (r) return r;
        }
        return PIC_OK;
    }
    for (int32_t a = 0; a < n; a++)
        for (int k = 0; k < 3; k++) CK(cudaMemsetAsync(hs[a]->J[k], 0, field_bytes(hs[a]), hs[a]->s));
    for (int32_t i = 0; i < nsteps; i++)
        for (int32_t a = 0; a < n; a++) {
            int r = enqueue_graph_step(hs[a]);
            if (r) return r;
        }
    int first = PIC_OK;
    for (int32_t a = 0; a < n; a++) {
        int r = finish(hs[a]);
        if (r && !first) first = r;
    }
    return first;
}

int pic_diagnostics(pic_handle *h, double masse, double *out, int32_t nout)
{
    if (!h || !out || nout < 4) return PIC_ERR_INVALID;
    const GridP &g = h->g;
    if (!h->rho) {
        int r;
        if ((r = dalloc(h, &h->rho, (size_t)g.ncell)) || (r = dalloc(h, &h->rho_pos, (size_t)g.ncell))) return r;
    }
    CK(cudaMemsetAsync(h->diag_out, 0, 64 * sizeof(double), h->s));
    launch_field_energy(g, h->E, h->B, h->fp32, h->diag_partials, h->diag_blocks, h->diag_out, h->s);
    if (h->fp32) {
        const float *E[3] = {(const float *)h->E[0], (const float *)h->E[1], (const float *)h->E[2]};
        launch_gauss_f32(g, h->p32[h->cur], h->cnt, E, h->rho, h->rho_pos, h->diag_out + 2, h->s);
        launch_particle_energy_f32(g, h->p32[h->cur], h->cnt, masse, h->diag_out + 4, h->s);
    } else {
        const double *E[3] = {(const double *)h->E[0], (const double *)h->E[1], (const double *)h->E[2]};
        launch_gauss_f64(g, h->p64[h->cur], h->cnt, E, h->rho, h->rho_pos, h->diag_out + 2, h->s);
        launch_particle_energy_f64(g, h->p64[h->cur], h->cnt, masse, h->diag_out + 4, h->s);
    }
    double tmp[64];
    CK(cudaMemcpyAsync(tmp, h->diag_out, sizeof(tmp), cudaMemcpyDeviceToHost, h->s));
    int r = finish(h);
    const int n = nout < 4 + h->cfg.nflvr ? nout : 4 + h->cfg.nflvr;
    for (int i = 0; i < n; i++) out[i] = tmp[i];
    return r;
}

int pic_solve_gauss(pic_handle *h, double tol, int32_t max_iter, int32_t *iters, double *rel_residual,
                    double *rho_mean)
{
    if (!h || h->g.geom != PIC_GEOM_CARTESIAN || h->g.x_external || !(tol > 0.0) || max_iter < 1) return PIC_ERR_INVALID;
    const GridP &g = h->g;
    if (!h->rho) {
        int r;
        if ((r = dalloc(h, &h->rho, (size_t)g.ncell)) || (r = dalloc(h, &h->rho_pos, (size_t)g.ncell))) return r;
    }
    if (h->fp32) launch_rho_f32(g, h->p32[h->cur], h->cnt, h->rho, h->rho_pos, h->s);
    else launch_rho_f64(g, h->p64[h->cur], h->cnt, h->rho, h->rho_pos, h->s);
    int it = 0;
    double rr = 0.0, mean = 0.0;
    const int rc = solve_gauss(g, h->E, h->fp32, h->rho, tol, max_iter, h->s, &it, &rr, &mean);
    if (iters) *iters = it;
    if (rel_residual) *rel_residual = rr;
    if (rho_mean) *rho_mean = mean;
    if (rc != PIC_OK) return rc;
    return finish(h);
}

int pic_profile(pic_handle *h, int32_t enable)
{
    if (!h) return PIC_ERR_INVALID;
    h->profiling = enable != 0;
    return PIC_OK;
}

int pic_phase_times(pic_handle *h, double *ms, int64_t *launches, int32_t n, int64_t *steps)
{
    if (!h || n < 0) return PIC_ERR_INVALID;
    for (int i = 0; i < n && i < PIC_PHASE_COUNT; i++) {
        if (ms) ms[i] = h->phase_ms[i];
        if (launches) launches[i] = h->phase_launches[i];
    }
    if (steps) *steps = h->prof_steps;
    for (int i = 0; i < PIC_PHASE_COUNT; i++) {
        h->phase_ms[i] = 0;
        h->phase_launches[i] = 0;
    }
    h->prof_steps = 0;
    return PIC_OK;
}

int pic_launch_count(pic_handle *h, int64_t *launches)
{
    if (!h || !launches) return PIC_ERR_INVALID;
    *launches = h->launches;
    h->launches = 0;
    return PIC_OK;
}

int pic_device_errors(pic_handle *h, int32_t *bits)
{
    if (!h || !bits) return PIC_ERR_INVALID;
    int b = 0;
    CK(cudaMemcpyAsync(&b, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->s));
    CK(cudaMemsetAsync(h->err, 0, sizeof(int), h->s));
    CK(cudaStreamSynchronize(h->s));
    *bits = b;
    return PIC_OK;
}

}  // extern "C"

namespace pic {
int weibel_with_signs(pic_handle *h, double epc, double density, double drift, double temp_ion, double temp_elc,
                      uint32_t seed, double *sgn, PartF64 *view, long long *n)
{
    if (!h || h->fp32 || !sgn || !view || !n || !(epc > 0) || h->cfg.nflvr < 2) return PIC_ERR_INVALID;
    WeibelParams w;
    w.epc = epc;
    w.density = density;
    w.drift = drift;
    w.temp[0] = temp_ion;
    w.temp[1] = temp_elc;
    w.seed = seed;
    w.sgn_out = sgn;
    const double vol = (double)h->g.nx * (double)h->g.ny * (h->g.dims == 3 ? (double)h->g.nz : 1.0);
    w.ntrial = (long long)(epc * vol);
    if (w.ntrial <= 0 || 2 * w.ntrial >= (1ll << 32)) return PIC_ERR_INVALID;
    CK(cudaMemsetAsync(h->cnt, 0, sizeof(Counters), h->s));
    set_sorted(h, false);
    int r = launch_weibel(h->g, w, h->tab_x, h->tab_p, h->ntab, &h->p64[h->cur], nullptr, h->cnt, h->sc, h->capacity,
                          h->err, h->s);
    if (r) return r;
    if ((r = finish(h))) return r;
    int64_t used = 0;
    if ((r = pic_particle_count(h, &used))) return r;
    *view = h->p64[h->cur];
    *n = used;
    return PIC_OK;
}
}  // namespace pic
