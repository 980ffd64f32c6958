/*
 * pictor_b200.h -- C ABI of the B200 (sm_100a) particle-in-cell step.
 *
 * The reference has no plugin API: src/MAIN.F90 calls argument-less Fortran
 * subroutines under `#ifdef gpu` (MAIN.F90:20-28, 53-55, 67-69, 91-93,
 * 113-116, 128-130, 161-163, 173-175, 189-191, 223-233, 250-252, 263-265)
 * that work on module globals (vars.F90, src/var_gpu.F90).  Each entry point
 * below replaces one of those subroutines; a Fortran module binds them with
 * ISO_C_BINDING (pictor_b200/fortran/pictor_b200_gpu.F90).  Plain pointers
 * and sizes only.
 *
 * Layout on the host side is the reference's: fields are column-major
 * (mx,my,mz) double arrays with 2 low and 3 high ghost layers (mx = nx+5,
 * mz = 1 in 2D; src/comm/subdomains/subdomains.F90:42-50); particles are the
 * SoA q,x,y,z,u,v,w (double) + flv (int32) of vars.F90:43-45 with absolute
 * local cell coordinates, interior [3, m-2), 2D z in [1,2) and flv = 0 marking
 * a hole.
 *
 * Every call returns PIC_OK (0) or a negative PIC_ERR_* code; the Fortran shim
 * maps a nonzero code to the reference's Abort(code)
 * (src/comm/communication.F90:96-102).  One host thread drives a handle; the
 * library owns all device memory and its CUDA stream.
 */
#ifndef PICTOR_B200_H
#define PICTOR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PIC_MAX_FLVR 15

enum {
    PIC_OK = 0,
    PIC_ERR_INVALID = -1,   /* bad argument or configuration                   */
    PIC_ERR_OOM = -2,       /* device allocation failed                        */
    PIC_ERR_OVERFLOW = -3,  /* particle capacity exceeded (cf. particles_gpu.F90:21, Abort(12)) */
    PIC_ERR_NAN = -4,       /* non-finite value met                             */
    PIC_ERR_TIMEOUT = -5,   /* a bounded device wait gave up                   */
    PIC_ERR_CUDA = -6,      /* CUDA runtime error                              */
    PIC_ERR_RANGE = -7,     /* particle outside the ghost frame of the grid    */
    PIC_ERR_NOGPU = -8      /* no CUDA device                                  */
};

enum { PIC_GEOM_CARTESIAN = 0, PIC_GEOM_CYLINDRICAL = 1 };
enum { PIC_FDTD_YEE = 0, PIC_FDTD_LEHE = 1 };
/* PIC_PREC_FP64: the reference layout and arithmetic (drop-in).
   PIC_PREC_FP32: FP32 particles with cell-relative positions and FP32 fields. */
enum { PIC_PREC_FP64 = 0, PIC_PREC_FP32 = 1 };

/* Runtime form of parameters.F90 + the setup's species table.  Replaces the
   compile-time module parameters read by the GPU kernels (src/var_gpu.F90). */
typedef struct {
    int32_t nx, ny, nz;          /* interior cells (parameters.F90:6-8); nz ignored in 2D  */
    int32_t dims;                /* 2 or 3 (Makefile THREE_DIMS)                          */
    int32_t geom;                /* PIC_GEOM_*                                             */
    int32_t fdtd;                /* PIC_FDTD_* (Makefile FDTD=Lehe)                       */
    int32_t precision;           /* PIC_PREC_*                                             */
    int32_t nflvr;               /* species count (vars.F90:92)                           */
    double c;                    /* Courant number (parameters.F90:20)                    */
    double qi;                   /* charge unit from InitScale (initialise.F90:46)        */
    double bext[3];              /* Bx_ext0, By_ext0, Bz_ext0 (vars.F90:25)               */
    double qm[PIC_MAX_FLVR + 1]; /* flvrqm, index 1..nflvr (vars.F90:87)                  */
    int32_t reorder_period;      /* prtl_reorder_period (parameters.F90:71); 0 = never    */
    int32_t curr_filter;         /* passes of the (1/4,1/2,1/4) filter (parameters.F90:22) */
    int64_t capacity;            /* particle slots on the device (gpu_prtl_arr_size)      */
    /* cylindrical (geom = PIC_GEOM_CYLINDRICAL): r of the first interior x cell
       (xborders(procxind) + rshift, cyl_common.F90:23) and whether the axis is
       in the domain (parameters.F90:65). */
    double rmin;
    int32_t inc_axis;
    /* FP32 form: brick shape in interior cells (the unit of the reorder and
       of one CTA of the mover); 0 = chosen from the fill (capacity / cells).
       No counterpart in the reference, whose reorder is per cell. */
    int32_t brick[3];
    /* cylindrical: 0 = the reference's theta-gridded field solve; 2 = the
       field solve on azimuthal modes m = 0, 1 (the theta-gridded scheme
       projected onto them; particles still gather from and deposit onto the
       ny theta cells).  No counterpart in the reference. */
    int32_t cyl_modes;
    /* 1 = this handle is one slab of a domain split along x (the reference's
       MPI decomposition with the x neighbours on other ranks): the kernels
       leave the x ghost layers to the pic_slab_* exchanges and particles
       leaving through the x faces to pic_slab_pack_particles; y and z stay
       periodic on the slab.  Cartesian (FP64 or FP32) or cylindrical (FP64,
       theta-gridded: a slab of radii; inc_axis on the slab holding the axis,
       whose low face then has no neighbour, rmin >= 2.5 on the others), no
       current filter.  2 = the same for the cylindrical slab whose high face
       is the outer radius (no neighbour: leavers are dropped, its ghosts are
       neither packed nor unpacked).  0 = one domain. */
    int32_t slab_x;
    /* FP64 Cartesian form: 1 = sum the current in the reference's serial
       order (each cell's VecJ entries in particle order, then the cells onto
       the edges in the loop order of ReduceCurrentMatrix,
       movdep_routines.F90:243-311), so that J and every later phase equal
       the serial CPU build bit for bit and a run is reproducible; costs a
       sort of two records per particle each step.  0 = FP64 atomics into J
       (the sums differ from the serial build's in the last bits). */
    int32_t exact_current;
    /* FP64 form (Cartesian or cylindrical) after a reorder: 0 or 1 = the
       mover by tiles of cells (node and current boxes in shared memory); -1
       = one thread per particle with global atomics.  Positions and momenta are the same
       either way; the current differs in the order of its sums. */
    int32_t fp64_tiles;
    /* FP32 Cartesian form, 3D: 1 = each zigzag segment's current is its
       exact line integral of the bilinear weights (the cross term q dx dy dz
       / 12 of Villasenor and Buneman), so charge is conserved exactly and the
       Gauss residual stays at FP32 round-off; 0 = the reference's weights
       (products of segment-midpoint weights, vars.F90:343-355), which the
       FP64 form keeps: the FP32 form then differs from it by precision only.
       No counterpart in the reference. */
    int32_t exact_charge;
    int32_t reserved[3];
} pic_config;

typedef struct pic_handle pic_handle;

/* Library version, for the Fortran side to check at InitAll_gpu. */
int pic_version(void);

/* Create / destroy a simulation handle.  Replaces InitAll_gpu's allocations
   (src/init/initialise_gpu.F90:9-150). */
int pic_create(const pic_config *cfg, pic_handle **out);
void pic_destroy(pic_handle *h);

/* Host <-> device copies (InitAll_gpu, CopyGPUDataToHostForOutput
   src/mem/particles_gpu.F90:569-581).  Field arrays are (mx,my,mz)
   column-major doubles; any pointer may be NULL to skip that array. */
int pic_load_fields(pic_handle *h, const double *Ex, const double *Ey, const double *Ez,
                    const double *Bx, const double *By, const double *Bz);
int pic_fetch_fields(pic_handle *h, double *Ex, double *Ey, double *Ez,
                     double *Bx, double *By, double *Bz, double *Jx, double *Jy, double *Jz);
/* Current host -> device, as smoothen_current_gpu_OnHost does around the
   host filter (src/maxwell/fields_gpu.F90:120-131). */
int pic_load_current(pic_handle *h, const double *Jx, const double *Jy, const double *Jz);
int pic_load_particles(pic_handle *h, int64_t n, const double *q, const double *x, const double *y,
                       const double *z, const double *u, const double *v, const double *w,
                       const int32_t *flv);
/* Writes the used_prtl_arr_size slots (holes included); *n receives the count.
   Host arrays must hold pic_particle_count() entries. */
int pic_fetch_particles(pic_handle *h, int64_t *n, double *q, double *x, double *y, double *z,
                        double *u, double *v, double *w, int32_t *flv);
int pic_particle_count(pic_handle *h, int64_t *used);

/* Generate the Weibel set-up (setup_weibel.F90:17-61; init_prtl.F90:177-221;
   prob_dist.F90:13-70,223-254) on the device, with Philox-4x32-10 keyed by
   seed in place of gfortran's random_number.  epc = trials per cell per call,
   density = acceptance threshold, drift = beam |v| along x, temp = 2kT/mc^2. */
int pic_init_weibel(pic_handle *h, double epc, double density, double drift,
                    double temp_ion, double temp_elc, uint32_t seed);

/* Phases of one time step, in MAIN.F90 order. */
int pic_update_b_half(pic_handle *h);      /* UpdateBfieldHalfGPU + SendRecvFlds(B)  (em_update_gpu.F90:44) */
int pic_move_deposit(pic_handle *h);       /* MoveDepositPrtlGPU (movdep_gpu.F90:14-49)                     */
int pic_exchange_particles(pic_handle *h); /* ExchangePrtlGPU + AppendParticles (loadprtlout.F90:13-106, comm_prtl.F90:11-30) */
int pic_update_e(pic_handle *h);           /* UpdateEfieldGPU + SendRecvFlds(E) (em_update_gpu.F90:12-42)    */
int pic_fold_current(pic_handle *h);       /* UpdateCurrentsAllEdgesGPU / UpdateCurrentAllFaces (comm_fld.F90:15-72) */
int pic_add_current(pic_handle *h);        /* AddCurrentGPU + EMfldExchangeGPU (em_update_gpu.F90:92-109)    */
int pic_reset_current(pic_handle *h);      /* ResetCurrentGPU (fields_gpu.F90:61-65)                        */
int pic_reorder(pic_handle *h);            /* ReorderPrtlGPU / ReorderPrtlArr (mem_prtl.F90:166-301)        */
/* Current filter passes (smoothen_current, current.F90:19-163). */
int pic_filter_current(pic_handle *h);

/* Walls along x (src/bc/bc_reflect.F90 on one rank), for setups whose
   bc_face(1) (side 0, left) or bc_face(2) (side 1, right) is a wall at
   `pos` cells from the first interior cell.  pic_bc_reflect_x:
   RefBC_Prtl_Left/Right — particles beyond the wall mirrored with u
   reversed, the current beyond it folded back (EnforceBC_PostMovDep,
   MAIN.F90:77: after pic_move_deposit, before pic_exchange_particles).
   pic_bc_conducting_x: CondBC_Fld_Left/Right — Ey, Ez zeroed beyond the
   wall (EnforceBC_Final, MAIN.F90:209: after pic_add_current).  The FP64
   Cartesian single domain; the phase API, not pic_step. */
int pic_bc_reflect_x(pic_handle *h, int32_t side, double pos);
int pic_bc_conducting_x(pic_handle *h, int32_t side, double pos);
/* The y faces (bc_face(3) side 0 bottom, bc_face(4) side 1 top):
   RefBC_Prtl_Bottom/Top with their current fold (bc_reflect.F90:79-128) and
   CondBC_Fld_Bottom/Top (Ex, Ez zeroed, :11-41); also on a slab. */
int pic_bc_reflect_y(pic_handle *h, int32_t side, double pos);
int pic_bc_conducting_y(pic_handle *h, int32_t side, double pos);
/* A face of type 'remv' (bc.F90:258-283, RemovePrtl_Left/Right of
   bc_open.F90:8-62): the particles beyond the wall at `pos` on face 1..6
   (x, y, z; low, high) become holes; called where EnforceBC_PostMovDep
   calls it.  FP64 Cartesian. */
int pic_bc_remove(pic_handle *h, int32_t face, double pos);
/* Field faces of EnforceBC_Final (bc.F90:292-340) besides 'cond'; FP64
   Cartesian single domain, called after pic_add_current (MAIN.F90:209).
   pic_bc_attenuate: the faces of type 'attn' (SetBC_Fld, bc.F90:24-52) —
   Attenuate_EM_Vacuum with AttenFactorVacuum (bc_attenuate.F90:151-290):
   bit n-1 of `faces` marks bc_face(n) (1, 2 x; 3, 4 y; 5, 6 z, 3D only),
   pos[n-1] its pos_fld and scale[n-1] its attn_scale (SetBC_Fld default 4);
   every field component outside the attenuating faces is scaled by
   1 - min(1, (d / scale)^3) at its staggered position.
   pic_bc_attenuate_flow: face 1..4 of type 'iflw' (SetBC_InflowFld,
   bc.F90:163-205) — Attenuate_EM_Flow (bc_attenuate.F90:16-131) for a
   uniform flow: MagFld = bflow[3], DriftVelocity = drift[3]; the layer of
   `thickness` (attn_thickness, default 1) beside pos relaxes E to -v x B and
   B to bflow with the scale length `scale` (attn_scale, default 4).
   pic_bc_open_x: an 'open' field face along x (OpenBC_Fld_Left side 0,
   OpenBC_Fld_Right side 1, bc.F90:411-469). */
int pic_bc_attenuate(pic_handle *h, int32_t faces, const double *pos, const double *scale);
int pic_bc_attenuate_flow(pic_handle *h, int32_t face, double pos, double thickness, double scale,
                          const double *bflow, const double *drift);
int pic_bc_open_x(pic_handle *h, int32_t side, double pos);
/* An 'open' particle face along x (OpenBC_Prtl_Left side 0, OpenBC_Prtl_Right
   side 1, bc.F90:478-621, with dx = 1 as EnforceBC_Final calls them,
   :333-334): the particles beyond the face at `pos` become holes; every
   particle within one cell inside it is mirrored across the face and
   appended in slot order (InsertNewPrtl), its u lowered by gamma v0, v0 the
   mean x velocity of flavours 1 and 2 in its (j, k) column of that layer
   (OpenBC_MeanPrtlSpeed), taken <= 0 on the right face and >= 0 on the left.
   The column sums are FP64 atomics, so v0 (and the copies' u) can differ from
   the serial sum in the last bit.  PIC_ERR_OVERFLOW (nothing appended) when
   the copies do not fit in the capacity. */
int pic_bc_open_prtl_x(pic_handle *h, int32_t side, double pos);
/* Faces of type 'pml' (SetBC_Fld, bc.F90:45-50): the convolutional PML of
   bc_pml.F90 with SetPMLParameters' profile (n = 4, kappa_max = 1,
   sigma_max = 1, alpha_max = 9e-4).  pic_bc_pml sets the faces: bit n-1 of
   `faces` marks bc_face(n) (1, 2 x; 3, 4 y; 5, 6 z, 3D only) at pos[n-1]
   (pos_fld, cells from the first interior cell) with thickness[n-1]
   (attn_thickness, SetBC_Fld default 4); the twelve auxiliary grids
   (pml_E_psi1/2, pml_B_psi1/2) are zeroed on the first call and kept by later
   ones (moved faces); faces = 0 switches the PML off.  pic_bc_pml_b is
   UpdateMagFld_PML + SendRecvFlds(B), called after the second
   pic_update_b_half (MAIN.F90:103-105); pic_bc_pml_e is UpdateElcFld_PML +
   SendRecvFlds(E), called after pic_update_e (:108-110).  Both do nothing
   while the grid lies inside the faces (no_pml_this_domain).  FP64 or FP32
   Cartesian single domain. */
int pic_bc_pml(pic_handle *h, int32_t faces, const double *pos, const double *thickness);
int pic_bc_pml_b(pic_handle *h);
int pic_bc_pml_e(pic_handle *h);
/* Particle injection at a face of type 'iflw' (SetBC_InflowPrtl, bc.F90:67-153):
   InjectNewPrtl (bc_inflow.F90:134-256) with 'rndm' placement, called where
   EnforceBC_PostMovDep calls InflowBC_Prtl (bc.F90:240, after
   pic_move_deposit).  The trial region is SetInjDomain's: along the face's
   axis from pos - speed c (or pos - vmax c) to pos + vmax c (or pos + speed
   c), clipped to the grid, the full interior across; epc times its volume
   trials (a Poisson draw of that mean below 1000), each at a uniform random
   position, accepted with probability `density` and only in the layer the
   flow emptied in one step (beyond pos + drift c on the face's side); each
   accepted position gets one particle per species (flv, charge, a
   Maxwellian of temperature temp boosted by the drift: GetVelGamma_MaxBolt
   and AddDriftVel, prob_dist.F90:13-30, 223-254), appended in trial order.
   The setup's density and drift functions are uniform here; the random
   numbers are Philox-4x32-10 keyed by seed, with `call` distinct per call
   (the step).  FP64 Cartesian single domain; PIC_ERR_OVERFLOW (nothing
   appended) past the capacity. */
typedef struct pic_inflow {
    int32_t face;          /* bc_face index 1..6 (2D: 1..4) */
    double pos;            /* bc_face(face)%pos_prtl, cells from the first interior cell */
    double speed;          /* bc_face(face)%speed (InjSpeed), a fraction of c per step */
    double vmax;           /* the flow's DriftVmax (SetBC_InflowFld default 1) */
    double epc;            /* trials per cell of unit density */
    double density;        /* Den, in [0, 1] */
    double drift[3];       /* DriftVelocity, in units of c */
    int32_t nspecies;      /* phase-space properties injected at each position, 1..4 */
    int32_t flv[4];
    double temp[4];        /* Temperature of each */
    double charge[4];      /* FlvrCharge(flv) * fraction of each */
    uint32_t seed, call;
} pic_inflow;
int pic_bc_inflow(pic_handle *h, const pic_inflow *inj);
/* RefPrtlFluidFrameRight (bc_inflow.F90:62-121), which InflowBC_Prtl runs
   before injecting when bc_face(2) is an 'iflw' particle face with 'rndm'
   placement: every particle beyond the injector at pos (bc_face(2)%pos_prtl)
   moved by the flow's drift (x > pos + 3 + drift_x c, local) is reflected
   in the frame moving with the flow (ReflectPrtlMovingFrameX), mirrored
   across that layer, and the current of the move added to J
   (DepositCurrentPIC, deposit.F90:11-103; FP64 atomics).  FP64 Cartesian. */
int pic_bc_inflow_reflect(pic_handle *h, double pos, double drift_x);

/* Slab form (pic_config.slab_x = 1).  A slab's step is the phase sequence
   with exchanges between the slabs (comm_fld.F90:15-130, loadprtlout.F90:
   13-106, comm_prtl.F90:11-66 across ranks); the caller moves the buffers
   (device pointers) between neighbouring slabs, the left neighbour of the
   first slab being the last one:
     pic_update_b_half; B faces | pic_move_deposit; pic_slab_pack_particles,
     particles, pic_slab_unpack_particles (from the left, then from the
     right) | pic_update_b_half; B faces | pic_update_e | J faces;
     pic_fold_current; pic_add_current; E faces | pic_reorder every period.
   Face buffers hold pic_slab_face_len doubles each: component-major layers
   of my * mz values.  pack_fields(which: 0 E, 1 B, 2 J) fills to_left and
   to_right (J: the ghost current, which it zeroes); unpack_fields takes what
   the left neighbour packed to its right (from_left) and what the right one
   packed to its left (from_right), copied into the ghosts (E, B) or added to
   the interior layers (J).  pack_particles removes the particles that left
   through the x faces and writes them to `out` (8 doubles each: q, x, y, z,
   u, v, w, flv, positions in the receiver's coordinates): n_right bound
   right first, then n_left bound left; y and z leavers wrap on the slab.
   pack_particles waits for its work in either sync mode (the counts size the
   transfers) and returns the device errors like a synchronous call:
   PIC_ERR_OVERFLOW, with both counts 0 and no particle moved, if more than
   `cap` leave or the appended particles would pass the capacity.  pic_step,
   pic_step_many and pic_exchange_particles refuse a slab.  The FP32 form
   uses the same buffers (its fields and particles converted to and from
   doubles exactly): its mover leaves an x leaver in the ghost cell beside
   the face, and the particles a slab receives between two reorders are
   moved one per thread after the bricks. */
int pic_slab_face_len(pic_handle *h, int64_t *n);
/* sync = 0: the phase entry points (pic_update_b_half ... pic_reorder and
   the pic_slab_* calls) only enqueue their work on the handle's stream
   (pic_stream) and report launch errors; device errors surface at the next
   synchronous call or pic_device_errors.  For a host that orders its own
   transfers on that stream (the slab exchanges).  sync = 1 (the default)
   waits for the queued work and returns its device errors. */
int pic_set_sync(pic_handle *h, int32_t sync);
int pic_slab_pack_fields(pic_handle *h, int32_t which, double *to_left, double *to_right);
int pic_slab_unpack_fields(pic_handle *h, int32_t which, const double *from_left, const double *from_right);
int pic_slab_pack_particles(pic_handle *h, double *out, int64_t cap, int64_t *n_right, int64_t *n_left);
int pic_slab_unpack_particles(pic_handle *h, const double *in, int64_t n);
/* The same exchange with the counts on the device, so that a slab's step
   never waits on the host: each direction's particles go in a box of
   cap + 1 records of 8 doubles (record 0 holds the count in its first word,
   the particles follow), and the boxes travel whole (a fixed size each
   step).  pic_slab_pack_particles_fixed fills to_left and to_right (all
   leavers or, when they exceed cap in total, none: the device error word
   gets PIC_DEVERR_OVERFLOW and both counts are 0); the neighbours' boxes
   go to pic_slab_unpack_particles_fixed, which appends from the left, then
   from the right, and ignores the box of a face without neighbour.  Both
   only enqueue their work under pic_set_sync(h, 0). */
int pic_slab_pack_particles_fixed(pic_handle *h, double *to_left, double *to_right, int64_t cap);
int pic_slab_unpack_particles_fixed(pic_handle *h, const double *from_left, const double *from_right, int64_t cap);

/* nsteps full steps of MAIN.F90:42-284 (reorder every reorder_period steps,
   counted from the handle's step counter), captured once as a CUDA graph. */
int pic_step(pic_handle *h, int32_t nsteps);
int pic_set_step(pic_handle *h, int64_t t);

/* The batched form of pic_step for an ensemble of independent runs (no
   counterpart in the reference, which runs one simulation per job): nsteps
   steps of each of the n handles, enqueued step by step across the handles,
   each on its own stream, so that the step graphs of small runs execute
   concurrently on the GPU.  All handles must belong to the current device.
   Returns the first error of any handle; handles in profiling mode are
   stepped one after the other. */
int pic_step_many(pic_handle *const *hs, int32_t n, int32_t nsteps);

/* The same ensemble step as one persistent kernel per span of steps: every
   phase of every run, for the steps up to the next reorder of any run, in a
   single launch whose CTAs (three per SM) take the work items (the B half
   step's blocks of 32 x 8 cells, the mover's bricks, the second B half step,
   the E update) in order from one counter; an item first waits until its
   run has finished the phase it depends on, so each run steps at its own
   pace and the phases of different runs overlap.  The reorders due between
   spans run on the device between the launches; the whole sequence of the
   call is captured as one CUDA graph (kept for the next call with the same
   runs, steps and reorder phases).  Requires what pic_step_batched requires.
   Every wait gives up after spin_limit polls (0: a default of about one
   second) and the call then returns PIC_ERR_TIMEOUT; force_timeout = 1 makes
   the first mover item wait for a count that is never reached (a test of
   that bound: the runs' state is then undefined, the GPU stays usable). */
int pic_step_persistent(pic_handle *const *hs, int32_t n, int32_t nsteps, uint32_t spin_limit,
                        int32_t force_timeout);

/* The same ensemble step with one launch per phase for a group of runs:
   the runs are split into up to four groups of about equal particle count;
   each group's B half step, mover, B half step and E update are single
   launches over all of its runs (work items: (32, 8) blocks of every run's
   interior, and every run's bricks), captured as one CUDA graph per group on
   the group's stream.  Requires FP32 runs of one dimensionality and FDTD,
   all reordered at least once (their bricks valid), without the current
   filter; returns PIC_ERR_INVALID otherwise. */
int pic_step_batched(pic_handle *const *hs, int32_t n, int32_t nsteps);

/* The initial electrostatic field, FP64 on the device (no counterpart in the
   reference, whose setups start from a neutral plasma with E = 0 or set the
   fields themselves; north_star keeps this solve in FP64 for the FP32 form
   too).  The particles' CIC charge density rho at the nodes (the rho of the
   Gauss residual of pic_diagnostics) minus its mean (returned in *rho_mean,
   a uniform neutralising background on the periodic grid) is the right-hand
   side of -L phi = rho - mean, L the periodic 7-point (2D: 5-point) Laplacian
   of the interior nodes, solved by conjugate gradients to a relative residual
   of `tol` in at most max_iter iterations; E is replaced by -grad(phi)
   (Ex(i) = phi(i) - phi(i+1) at i + 1/2, ghosts as periodic images, Ez = 0
   in 2D), whose node divergence (CalcDivE, savedata_routines.F90:310-348) is
   rho - mean; B is left as it is.  *iters and *rel_residual report the
   solve.  Cartesian single domain, FP64 or FP32 fields.  PIC_ERR_TIMEOUT when
   max_iter runs out before tol (E then holds the last iterate). */
int pic_solve_gauss(pic_handle *h, double tol, int32_t max_iter, int32_t *iters, double *rel_residual,
                    double *rho_mean);
/* Diagnostics (savedata_routines.F90:265-348), FP64 accumulation on device:
   out[0] = sum |B|^2, out[1] = sum |E|^2 over the interior (CalcFldEnergy),
   out[2] = max |divE - rho| over interior nodes, out[3] = max |rho_+|,
   out[4..4+nflvr-1] = kinetic energy per species (CalcPrtlEnergy). */
int pic_diagnostics(pic_handle *h, double masse, double *out, int32_t nout);

/* Device error word accumulated by the kernels since the last call (bit set of
   PIC_DEVERR_*); cleared by the call. */
enum { PIC_DEVERR_RANGE = 1, PIC_DEVERR_OVERFLOW = 2, PIC_DEVERR_NAN = 4, PIC_DEVERR_SUBSTEP = 8,
       PIC_DEVERR_TIMEOUT = 16 };
int pic_device_errors(pic_handle *h, int32_t *bits);

/* Phases of pic_step, in step order. */
enum {
    PIC_PHASE_BHALF1 = 0, /* UpdateBfieldHalf + halo before the push     */
    PIC_PHASE_MOVE,       /* MoveDepositPrtl                               */
    PIC_PHASE_EXCHANGE,   /* particle wrap (FP64 layout)                   */
    PIC_PHASE_BHALF2,     /* second UpdateBfieldHalf + halo                */
    PIC_PHASE_EFIELD,     /* UpdateEfield + fold + AddCurrent + halo       */
    PIC_PHASE_REORDER,    /* ReorderPrtl (every reorder_period steps)      */
    PIC_PHASE_COUNT
};
/* Profiling (the reference's per-phase timers, MAIN.F90:440-452 and
   communication.F90:69-94, on the device): while enabled, pic_step launches
   phases eagerly with a CUDA event pair around each; pic_phase_times returns
   the summed milliseconds and kernel launches per phase and the number of
   profiled steps, then resets them. */
int pic_profile(pic_handle *h, int32_t enable);
int pic_phase_times(pic_handle *h, double *ms, int64_t *launches, int32_t n, int64_t *steps);
/* Kernels launched by pic_step since the last call (graph or eager). */
int pic_launch_count(pic_handle *h, int64_t *launches);

/* Field energy without any device allocation (no counterpart in the
   reference).  For callers that cannot call cudaMalloc at this point: hosts
   whose memory pool owns all of the GPU's memory, or that must not let a
   library allocate/free (cudaFree synchronizes the device) between their own
   steps.  Inputs are caller-owned DEVICE arrays in the reference layout
   ((nx+5, ny+5, nz+5 or 1) column-major FP64); out2 is a DEVICE pointer that
   receives the sum of Bx^2 + By^2 + Bz^2 and the sum of Ex^2 + Ey^2 + Ez^2
   over the interior cells 3..m-3 of each axis.  Work is enqueued on `stream`
   (a cudaStream_t, NULL for the default stream); synchronize before reading
   out2.  The reduction's partial sums use one fixed array of 148*8 pairs in
   the library's device memory, shared by every call: calls that overlap on
   the GPU race.  Each call looks up that array's device address in the
   current context.  Returns PIC_ERR_INVALID for bad sizes. */
int pic_field_energy_noalloc(const double *Ex, const double *Ey, const double *Ez,
                             const double *Bx, const double *By, const double *Bz,
                             int32_t nx, int32_t ny, int32_t nz, int32_t dims,
                             double *out2, void *stream);

/* ---------------------------------------------------------------------------
   The differentiable form (no counterpart in the reference): a 2D Cartesian
   periodic Yee run whose objective is the time-integrated magnetic energy
   J = sum over steps t of 1/2 sum over cells |B_t|^2, with hand-written
   adjoint kernels for the field updates, the push and the deposit.  The
   forward step is the step of this library (FP64 or FP32 per
   cfg->precision; dims 2, geom Cartesian, fdtd Yee, no current filter) on
   interior arrays with periodic indices and particles in fixed slots.
   --------------------------------------------------------------------------- */
typedef struct pic_adjoint pic_adjoint;
int pic_adj_create(const pic_config *cfg, pic_adjoint **out);
void pic_adj_destroy(pic_adjoint *a);
/* Initial particles from the Weibel loader of pic_init_weibel (same seed, same
   particles), recording each particle's beam-drift sign for the parameter
   gradients.  Fields start at zero. */
int pic_adj_init_weibel(pic_adjoint *a, double epc, double density, double drift, double temp_ion, double temp_elc,
                        uint32_t seed, int64_t *n);
/* Initial particles from host arrays in the reference layout (x, y in ghosted
   1-based cell units, z in [1,2)); drift_sign may be NULL (parameter
   gradients are then zero). */
int pic_adj_load_particles(pic_adjoint *a, int64_t n, const double *q, const double *x, const double *y,
                           const double *z, const double *u, const double *v, const double *w, const int32_t *flv,
                           const double *drift_sign);
int pic_adj_fetch_particles(pic_adjoint *a, int64_t *n, double *q, double *x, double *y, double *z, double *u,
                            double *v, double *w, int32_t *flv, double *drift_sign);
/* nsteps steps from the initial state, keeping the state every
   checkpoint_every steps; *objective = J. */
int pic_adj_forward(pic_adjoint *a, int32_t nsteps, int32_t checkpoint_every, double *objective);
/* Branches of the forward mover for the following pic_adj_forward calls:
   0 free (default); 1 record the discrete decisions of every particle and
   step (start and end cells, the side of the relay point's clamp, the
   periodic wrap); 2 replay the recorded ones (same particle count, at most
   the recorded step count), which makes the run a smooth function of the
   initial state whose derivative at the recorded run is the adjoint's:
   central differences of replayed runs check the gradient without the jumps
   of the zigzag current.  The reverse sweep always recomputes freely. */
int pic_adj_branches(pic_adjoint *a, int32_t mode);
/* Reverse sweep of the last forward run (each segment between checkpoints is
   recomputed): dJ/d(initial u, v, w, x, y) per particle (host arrays of n, any
   may be NULL) and dparam[0] = dJ/d drift, dparam[1..2] = dJ/d temperature of
   flavours 1 and 2 (the loader's Maxwell temperatures temp[0..1]). */
int pic_adj_gradient(pic_adjoint *a, double drift, const double *temp, double *du, double *dv, double *dw, double *dx,
                     double *dy, double *dparam);

/* Text for an error code. */
const char *pic_error_string(int code);

/* Stream the handle launches on (cudaStream_t as void*), for callers that
   order their own device work after the library's. */
void *pic_stream(pic_handle *h);

#ifdef __cplusplus
}
#endif
#endif
