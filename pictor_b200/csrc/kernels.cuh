// kernels.cuh -- host launchers of the device kernels (one declaration per
// kernel family; definitions in fields.cu, mover.cu, mover_f32.cu, bricks.cu,
// particles.cu, cyl.cu, diag.cu).
#pragma once

#include "common.cuh"

namespace pic {

// Particle arrays in the reference layout (vars.F90:43-45).
struct PartF64 {
    double *q, *x, *y, *z, *u, *v, *w;
    int32_t *flv;
};

// FP32 cell-relative particles: key = (flv << 28) | linear ghosted cell index;
// offsets in [0,1) from the cell's lower corner; momenta gamma*v/c; w = q.
// In 2D dz is not stored (the out-of-plane position never enters the 2D step).
struct PartF32 {
    uint32_t *key;
    float *dx, *dy, *dz, *ux, *uy, *uz, *w;
};

constexpr int kFlvShift = 28;
constexpr uint32_t kCellMask = (1u << kFlvShift) - 1u;

// fields.cu
template <typename T> void launch_bhalf(const GridP &g, T *const E[3], T *const B[3], cudaStream_t s);
template <typename T> void launch_efield(const GridP &g, int mode, T *const E[3], T *const B[3], T *const J[3], cudaStream_t s);
template <typename T> void launch_fold(const GridP &g, T *const J[3], cudaStream_t s);
template <typename T> void launch_filter(const GridP &g, T *const J[3], T *tmp, cudaStream_t s);

// cyl.cu (cylindrical FP64 form)
template <typename T>
void launch_cyl_bhalf(const GridP &g, T *const E[3], T *const B[3], cudaStream_t s);
template <typename T>
void launch_cyl_efield(const GridP &g, int mode, T *const E[3], T *const B[3], T *const J[3], cudaStream_t s);
template <typename T>
void launch_cyl_fold(const GridP &g, T *const J[3], cudaStream_t s);
// modal.cu: the cylindrical field solve on azimuthal modes m = 0, 1 (arrays (mx, 3, mz))
template <typename T>
void launch_modal_bhalf(const GridP &g, T *const Em[3], T *const Bm[3], cudaStream_t s);
template <typename T>
void launch_modal_efield(const GridP &g, int mode, T *const Em[3], T *const Bm[3], T *const Jm[3], cudaStream_t s);
template <typename T>
void launch_modal_synth(const GridP &g, T *const Fm[3], T *const F[3], cudaStream_t s);
template <typename T>
void launch_modal_project(const GridP &g, T *const F[3], T *const Fm[3], cudaStream_t s);
struct Tiles64;
void launch_cyl_move_deposit(const GridP &g, const PartF64 &p, const Counters *cnt, double *const E[3],
                             double *const B[3], double *const J[3], int *err, cudaStream_t s,
                             const Tiles64 *T = nullptr);
void launch_cyl_move_deposit_f32(const GridP &g, const PartF32 &p, const Counters *cnt, float *const E[3],
                                 float *const B[3], float *const J[3], int *err, cudaStream_t s);

// mover.cu
struct SegRecords;
// rec == nullptr: the current goes to J by FP64 atomics; otherwise it is
// summed in the reference's order (pic_config.exact_current, see mover.cu).
// first (device, may be null): move the slots [*first, used) only.
void launch_move_deposit_f64(const GridP &g, const PartF64 &p, const Counters *cnt, double *const E[3],
                             double *const B[3], double *const J[3], int *err, cudaStream_t s,
                             SegRecords *rec = nullptr, const long long *first = nullptr);
// mover_f64_tiled.cu: the FP64 mover after a reorder, one CTA per tile of H
// row segments of W consecutive cells (x in [1 + sx W, 1 + (sx+1) W), rows
// j0 .. j0 + H - 1, plane k; the tiles cover the ghosted grid), whose
// particles the cell-order reorder leaves in H slot ranges.
constexpr int kTile64SmemBytes = 110 * 1024;   // node box + FP64 current box of one tile (2 CTAs per SM)
constexpr int kTile64MaxRows = 8;
struct Tiles64 {
    uint32_t *range;              // 2 H per tile: first and past-the-end slot of each row segment
    int *box;                     // 8 per tile: lo[3], hi[3] of the cells its particles occupy (1-based)
    long long *np;                // the live count at the reorder: slots past it were appended since
    unsigned long long *qmax;     // bits of max |q| over the live particles at the reorder (>= 0 doubles
                                  // order as their bit patterns): the bound of the fixed-point current box
    int W, H, nsx, ntiles;        // W cells per row segment, H rows per tile
    int D;                        // z planes per tile (3D; H D row segments, at most kTile64MaxRows)
    int jfirst;                   // rows of the first row group (H, or 2: the low ghost rows alone, so
                                  // that the next groups start at the first interior row)
    int smem_bytes;
};
void choose_tiles64(const GridP &g, Tiles64 &T);
// After a reorder: the tiles' slot ranges from the sorted keys, the boxes.
void launch_tiles64_after_reorder(const GridP &g, const uint32_t *keys, const Counters *cnt, Tiles64 &T,
                                  cudaStream_t s);
void launch_move_deposit_f64_tiled(const GridP &g, const PartF64 &p, const Counters *cnt, const Tiles64 &T,
                                   double *const E[3], double *const B[3], double *const J[3], int *err,
                                   cudaStream_t s);
// mover_f32.cu: per-particle FP32 mover (any particle order)
void launch_move_deposit_f32(const GridP &g, const PartF32 &p, const Counters *cnt, float *const E[3],
                             float *const B[3], float *const J[3], int *err, cudaStream_t s);
// Bricks of the FP32 form: blocks of t[0] x t[1] x t[2] interior cells, nb[d]
// per axis, x fastest.  After a reorder the particles of brick b occupy slots
// [tile_start[b], tile_start[b+1]); box[8b..8b+5] holds the lower and upper
// cell bounds (relative to the brick centre 3 + nb*t + t/2, unwrapped) of
// where the brick's particles are, which the tiled mover reads and rewrites.
constexpr int kBrickSmemBytes = 64 * 1024;   // dynamic shared memory of the tiled mover (node + current box)
struct Bricks {
    uint32_t *tile_start;   // ntiles + 1
    int *box;               // 8 per brick
    uint32_t *count;        // ntiles + 1 (scan input)
    uint32_t *cursor;       // ntiles
    uint32_t *bid;          // brick id per particle slot (capacity); slot scratch of the in-brick order
    uint32_t *src;          // source slot of every brick-grouped slot (capacity)
    uint32_t *scan_tmp;
    uint32_t *wmax_bits;    // max |w| of the live particles (FP32 bits), set by the reorder
    float4 *nodeA;          // node-averaged Ex, Ey, Ez, Bx (+ bext) at every interior node, or null
    float2 *nodeB;          // node-averaged By, Bz (+ bext); both written before each tiled move
    int t[3], nb[3], ntiles;
    unsigned int tmagic[3];   // x / t[d] = fast_div(x, tmagic[d], tshift[d]) for t[d] >= 2 (div_magic)
    int tshift[3];
    int smem_floats;
};
// Shared words of a mover box of C cells: (C+1) nodes per axis x 6 field
// components and (C+3) current cells per axis x 3 components of jw words
// (1: 32-bit fixed point, 2: 64-bit).
__host__ __device__ inline long long box_floats(int dims, int cx, int cy, int cz, int jw = 1)
{
    const long long nn = (long long)(cx + 1) * (cy + 1) * (dims == 3 ? cz + 1 : 1);
    const long long nj = (long long)(cx + 3) * (cy + 3) * (dims == 3 ? cz + 3 : 1);
    return 6 * nn + 3 * jw * nj;
}
// Words per current entry of a mover box: 64-bit fixed point for the
// cylindrical form, whose weights grow with the radius (a 32-bit scale set by
// the largest weight leaves too few bits for the currents near the axis).
__host__ __device__ inline int box_current_words(const GridP &g) { return g.geom == PIC_GEOM_CYLINDRICAL ? 2 : 1; }
constexpr int kBoxAxisMax = 64;   // cells per axis of a mover box
// Brick shape: `req` (all > 0) if given, else about 4096 particles per brick
// at ppc particles per cell.  Returns false if the brick plus one cell on
// each side would not fit the mover's shared memory.
bool choose_bricks(const GridP &g, double ppc, const int req[3], Bricks &bk);
// Tiled FP32 mover: one CTA per brick.
// One run of a batch of FP32 runs stepped by shared kernels (one launch per
// phase for all runs).  `cur` is the run's current particle buffer; a
// reorder of the run flips it on the device (launch_batch_flip).
struct BatchRun {
    GridP g;
    PartF32 p[2];
    Bricks bk;
    float *E[3], *B[3], *J[3];
    int *err;
    int cur;
    int fb[3];   // blocks of the (32, 8) interior tiling of the field kernels
};
// Work lists: run r owns field items [fstart[r], fstart[r+1]) and bricks
// [mstart[r], mstart[r+1]).
void launch_batch_bhalf(int dims, int fdtd, const BatchRun *runs, const int *fstart, int n, int total, cudaStream_t s);
void launch_batch_efield(int dims, const BatchRun *runs, const int *fstart, int n, int total, cudaStream_t s);
void launch_batch_move(int dims, bool exact_charge, const BatchRun *runs, const int *mstart, int n, int total,
                       cudaStream_t s);
void launch_batch_flip(BatchRun *runs, int r, cudaStream_t s);
// Field work items of the persistent ensemble step: 32 x (8 kPersistFieldRows)
// interior cells (kPersistFieldRows blocks of the field kernels' tiling).
constexpr int kPersistFieldRows = 4;
// ensemble.cu: the persistent ensemble step, nsteps steps of the n runs in one
// launch; ctl holds 3 + 4 n counters (zeroed by the launcher).
void launch_ensemble_persistent(int dims, int fdtd, bool exact_charge, const BatchRun *runs, const int *fstart,
                                const int *mstart, int n, int nsteps, unsigned *ctl, unsigned spin_limit,
                                int force_timeout, cudaStream_t s);
void launch_move_deposit_f32_tiled(const GridP &g, const PartF32 &p, const Bricks &bk, const Counters *cnt,
                                   float *const E[3], float *const B[3], float *const J[3], int *err, cudaStream_t s);
// cyl.cu: tiled FP32 cylindrical mover, one CTA per brick (+ the axis current)
void launch_cyl_move_deposit_f32_tiled(const GridP &g, const PartF32 &p, const Bricks &bk, float *const E[3],
                                       float *const B[3], float *const J[3], int *err, cudaStream_t s);

// particles.cu
struct SortScratch {
    uint32_t *key[2];
    uint32_t *idx[2];
    uint32_t *hist;       // 256 * ntiles
    uint32_t *scan_tmp;   // partial sums of the scan
    size_t ntiles;
    size_t scan_tmp_len;
};
size_t sort_tiles(long long capacity);
size_t scan_tmp_len(size_t n);
// Stable LSD radix sort of sc.key[0] (with the slot index as payload) over
// the first *used keys, each < 2^nbits; returns r with the result in
// sc.key[r] / sc.idx[r].
int radix_sort_keys(SortScratch &sc, const long long *used, int nbits, cudaStream_t s);
int sort_key_bits(long long ncell);
// Exact-order deposit of the FP64 form: the two zigzag segments of particle n
// are records 2n and 2n+1 (key = the cell of the segment, ncell for none;
// NE values each, structure of arrays: val[e * n2 + r]); sorted by cell
// (stable, so a cell's records stay in particle order), summed per cell into
// vecj[e * ncell + cell] in that order, and assembled into J in the loop
// order of ReduceCurrentMatrix.
struct SegRecords {
    SortScratch sc;       // sized for n2 keys; sc.key[0] receives the record keys
    double *val;          // NE * n2
    double *vecj;         // NE * ncell
    long long *count;     // device: 2 * used
    long long n2;         // 2 * capacity
};
// Exchange (wrap) of the reference layout: holes + append in AppendParticles order.
// Slab form (g.x_external): the x leavers go to `out` (out_cap particles of 8
// doubles) and sent_counts (device) receives {right-bound, right + left-bound}.
void launch_exchange_f64(const GridP &g, PartF64 &p, Counters *cnt, SortScratch &sc, long long capacity, int *err,
                         cudaStream_t s, double *out = nullptr, long long out_cap = 0, uint32_t *sent_counts = nullptr);
// bc.cu: walls along x (src/bc/bc_reflect.F90 on one rank), FP64 reference layout
void launch_wall_reflect(const GridP &g, PartF64 &p, const Counters *cnt, double *const J[3], int side, double pos,
                         long long capacity, cudaStream_t s);
void launch_wall_conducting(const GridP &g, double *const E[3], int side, double pos, cudaStream_t s);
void launch_wall_reflect_y(const GridP &g, PartF64 &p, const Counters *cnt, double *const J[3], int side, double pos,
                           long long capacity, cudaStream_t s);
void launch_wall_conducting_y(const GridP &g, double *const E[3], int side, double pos, cudaStream_t s);
void launch_wall_remove(const GridP &g, PartF64 &p, const Counters *cnt, int face, double pos, long long capacity,
                        cudaStream_t s);
// bc.cu: field faces of EnforceBC_Final (bc.F90:292-340): 'attn' faces
// (Attenuate_EM_Vacuum), an 'iflw' face with a uniform flow
// (Attenuate_EM_Flow), 'open' faces along x (OpenBC_Fld_Left/Right)
void launch_bc_attenuate(const GridP &g, double *const E[3], double *const B[3], int faces, const double *pos,
                         const double *sc, cudaStream_t s);
void launch_bc_attenuate_flow(const GridP &g, double *const E[3], double *const B[3], int side, double pos, double dl,
                              double sc, const double *b, const double *v, cudaStream_t s);
void launch_bc_open_fld_x(const GridP &g, double *const E[3], double *const B[3], int side, double pos, cudaStream_t s);
// bc.cu: RefPrtlFluidFrameRight (bc_inflow.F90:62-121) with its current
void launch_bc_inflow_reflect(const GridP &g, PartF64 &p, const Counters *cnt, double *const J[3], double pos,
                              double drift, long long capacity, int *err, cudaStream_t s);
// bc.cu: an 'open' particle face along x (OpenBC_Prtl_Left/Right, bc.F90:478-621)
void launch_bc_open_prtl_x(const GridP &g, PartF64 &p, Counters *cnt, int side, double pos, double *col,
                           uint32_t *flag, uint32_t *counts, uint32_t *scan_tmp, uint32_t *total, long long capacity,
                           int *err, cudaStream_t s);
// pml.cu: the convolutional PML (bc_pml.F90).  Per axis and 1-based index a
// (a = 1..m): coef[axis][6 (a-1) + 0..2] = a, b, c at position a - 3 (the E
// update), [+3..5] at a - 3 + 0.5 (the B update); flag bits below.
constexpr uint8_t kPmlInside = 1;       // a - 3 strictly between the axis's pml_pos_ind
constexpr uint8_t kPmlBeyond = 2;       // a - 3 beyond the axis's layers (zeroed)
constexpr uint8_t kPmlBeyondHalf = 4;   // a - 3 + 0.5 beyond them
struct PmlP {
    const double *coef[3];
    const uint8_t *flag[3];
    double fc;
};
// Host: the tables of (mx + my + mz) rows (6 doubles and one flag each, x
// rows first); false when the whole grid lies inside (no_pml_this_domain).
bool pml_tables(const GridP &g, int faces, const double *pos, const double *thickness, double *coef, uint8_t *flag);
// which 0: UpdateMagFld_PML + halo(B); 1: UpdateElcFld_PML + halo(E)
template <typename T>
void launch_pml(const GridP &g, const PmlP &P, int which, T *const E[3], T *const B[3], T *const psi[6], cudaStream_t s);
// slab.cu: x faces of a slab (fields and particles), see pic_slab_* in the C ABI
template <typename T>
void launch_slab_pack_fields(const GridP &g, int which, T *const F[3], double *to_left, double *to_right, cudaStream_t s);
template <typename T>
void launch_slab_unpack_fields(const GridP &g, int which, T *const F[3], const double *from_left,
                               const double *from_right, cudaStream_t s);
// the FP32 form's x leavers (slab.cu): to the outbox, and the inbox appended
void launch_slab_pack_f32(const GridP &g, PartF32 &p, const Counters *cnt, double *out, long long out_cap,
                          uint32_t *counts, uint32_t *scan_tmp, uint32_t *total, uint32_t *sent, long long capacity,
                          int *err, cudaStream_t s);
void launch_slab_append_f32(const GridP &g, PartF32 &p, Counters *cnt, const double *in, long long n,
                            long long capacity, int *err, cudaStream_t s);
// slab.cu: the x leavers through fixed-size boxes (cap + 1 records of 8
// doubles, record 0 the count), with no count on the host
void launch_slab_pack_fixed(const GridP &g, bool fp32, PartF64 &p64, PartF32 &p32, Counters *cnt, SortScratch &sc,
                            double *to_left, double *to_right, long long cap, uint32_t *sent, long long capacity,
                            int *err, cudaStream_t s);
void launch_slab_append_fixed(const GridP &g, bool fp32, PartF64 &p64, PartF32 &p32, Counters *cnt,
                              const double *from_left, const double *from_right, long long cap, long long capacity,
                              int *err, cudaStream_t s);
void launch_slab_append(const GridP &g, PartF64 &p, Counters *cnt, const double *in, long long n, long long capacity,
                        int *err, cudaStream_t s);
// Stable cell-key reorder (ReorderPrtlArr).  The payload is gathered into
// `out`, after which the caller swaps `p` and `out`.
void launch_reorder_f64(const GridP &g, const PartF64 &p, const PartF64 &out, Counters *cnt, SortScratch &sc,
                        long long capacity, int *err, cudaStream_t s, Tiles64 *tiles = nullptr);
// Reorder of the FP32 form (bricks.cu): live particles grouped by brick into
// `out`, after which the caller swaps `p` and `out`.
void launch_reorder_f32(const GridP &g, const PartF32 &p, const PartF32 &out, Counters *cnt, long long capacity,
                        const Bricks &bk, int *err, cudaStream_t s);
// Reference layout <-> FP32 cell-relative conversion.
void launch_f64_to_f32(const GridP &g, const PartF64 &in, const PartF32 &out, long long n, int *err, cudaStream_t s);
void launch_f32_to_f64(const GridP &g, const PartF32 &in, const PartF64 &out, long long n, cudaStream_t s);
void launch_array_f64_to_f32(const double *in, float *out, long long n, cudaStream_t s);
void launch_array_f32_to_f64(const float *in, double *out, long long n, cudaStream_t s);
// Device Weibel loader.
struct WeibelParams {
    double epc, density, drift, temp[2];
    uint32_t seed;
    long long ntrial;
    double *sgn_out;   // optional (FP64 layout): +-1, the sign of each particle's beam drift
};
// Weibel loader into the FP64 buffers of handle h with the beam-drift sign of
// every particle in sgn (device, capacity entries); returns the particles'
// device view and count (used by the adjoint engine, adjoint.cu).
int weibel_with_signs(pic_handle *h, double epc, double density, double drift, double temp_ion, double temp_elc,
                      uint32_t seed, double *sgn, PartF64 *view, long long *n);
int launch_weibel(const GridP &g, const WeibelParams &w, const double *table_x, const double *table_p, int ntable,
                  const PartF64 *p64, const PartF32 *p32, Counters *cnt, SortScratch &sc, long long capacity,
                  int *err, cudaStream_t s);
// Particle injection at an 'iflw' face (InjectNewPrtl, bc_inflow.F90:134-256):
// the trial region (local coordinates), the trial count, a uniform density
// and drift, up to four species per accepted position.
struct InflowParams {
    double x1, x2, y1, y2, z1, z2;
    double density, drift[3], c, pos;
    int side, dims, nsp;
    int flv[4];
    double temp[4], charge[4];
    uint32_t seed, call;
    long long ntrial;
};
int launch_inflow(const GridP &g, const InflowParams &f, const double *X, const double *P, int nt, PartF64 &p,
                  Counters *cnt, SortScratch &sc, long long capacity, int *err, cudaStream_t s);
void scan_exclusive_u32(const uint32_t *in, uint32_t *out, size_t n, uint32_t *tmp, uint32_t *total, cudaStream_t s);

// diag.cu
void launch_field_energy(const GridP &g, const void *const E[3], const void *const B[3], bool fp32, double *partials,
                         int nblocks, double *out2, cudaStream_t s);
int field_energy_blocks(const GridP &g);
void launch_particle_energy_f64(const GridP &g, const PartF64 &p, const Counters *cnt, double masse, double *out,
                                cudaStream_t s);
void launch_particle_energy_f32(const GridP &g, const PartF32 &p, const Counters *cnt, double masse, double *out,
                                cudaStream_t s);
void launch_rho_f64(const GridP &g, const PartF64 &p, const Counters *cnt, double *rho, double *rho_pos, cudaStream_t s);
void launch_rho_f32(const GridP &g, const PartF32 &p, const Counters *cnt, double *rho, double *rho_pos, cudaStream_t s);
// poisson.cu: E = -grad(phi) with the node divergence equal to rho minus its
// mean (FP64 conjugate gradients); returns a PIC status
int solve_gauss(const GridP &g, void *const E[3], bool fp32, const double *rho, double tol, int max_iter,
                cudaStream_t s, int *iters, double *rel_res, double *rho_mean);
void launch_gauss_f64(const GridP &g, const PartF64 &p, const Counters *cnt, const double *const E[3], double *rho,
                      double *rho_pos, double *out2, cudaStream_t s);
void launch_gauss_f32(const GridP &g, const PartF32 &p, const Counters *cnt, const float *const E[3], double *rho,
                      double *rho_pos, double *out2, cudaStream_t s);

}  // namespace pic
