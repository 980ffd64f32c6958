/*
 * pictor_oracle.h -- CPU restatement (FP64, serial) of PICTOR's Cartesian
 * particle-in-cell time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * in pictor_b200/ is compared against.  Nothing in the product links it,
 * loads it or calls it; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py do.
 *
 * Parity status: the reference is Fortran (h5pfc + mpi_f08 + HDF5) and ships
 * no tests, golden vectors or fixtures, and no Fortran compiler exists in
 * this image, so this restatement cannot be checked against outputs of the
 * reference itself: parity against the reference is UNPINNED.  The
 * restatement is pinned instead to hand-derived known-answer vectors
 * (single-particle zigzag deposits, Boris gyration, Philox-4x32-10 published
 * vectors, Yee/Lehe stencil values) committed under tests/golden/.
 *
 * Layout conventions follow the reference exactly: fields are column-major
 * (mx,my,mz) arrays with 2 low and 3 high ghost layers (mx = nx+5;
 * src/comm/subdomains/subdomains.F90:42-50), indices are 1-based in the
 * comments and 0-based in memory; particle positions are absolute local cell
 * coordinates with the interior in [3, m-2) (subdomains.F90:52-67).
 */
#ifndef PICTOR_ORACLE_H
#define PICTOR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_FLVR 8

typedef struct {
    int dims;               /* 2 or 3 (Makefile THREE_DIMS / -DtwoD)            */
    int nx, ny, nz;         /* interior cells (nz ignored in 2D)                */
    int mx, my, mz;         /* nx+5, ny+5, nz+5 (mz=1 in 2D)                    */
    int fdtd;               /* 0 = Yee (em_update.F90), 1 = Lehe (em_update_lehe.F90) */
    int nflvr;              /* number of species                               */
    double c;               /* Courant number, parameters.F90:20               */
    double qi;              /* InitScale charge unit, initialise.F90:46         */
    double bext[3];         /* Bx_ext0, By_ext0, Bz_ext0 (vars.F90:25)          */
    double flvrqm[ORC_MAX_FLVR + 1]; /* q/m per flavour, index 1..nflvr         */
} orc_grid;

/* Particle SoA in the reference layout (vars.F90:43-45). */
typedef struct {
    double *q, *x, *y, *z, *u, *v, *w;
    int32_t *flv;
    int64_t used;           /* used_prtl_arr_size                              */
    int64_t capacity;       /* prtl_arr_size                                   */
} orc_particles;

typedef struct {
    double *Ex, *Ey, *Ez, *Bx, *By, *Bz, *Jx, *Jy, *Jz;
} orc_fields;

/* Fill mx,my,mz from nx,ny,nz,dims. */
void orc_grid_init(orc_grid *g);

/* em_update.F90 / em_update_lehe.F90 */
void orc_update_b_half(const orc_grid *g, orc_fields *f);
void orc_update_e(const orc_grid *g, orc_fields *f);
void orc_add_current(const orc_grid *g, orc_fields *f);
/* Lehe coefficients (em_update_lehe.F90:8-25): out[0..8] =
   alpha_x, alpha_y, alpha_z, beta_xy, beta_xz, beta_yx, beta_yz, beta_zx, beta_zy,
   out[9..11] = delta_x, delta_y, delta_z. */
void orc_lehe_coefficients(const orc_grid *g, double out[12]);

/* comm_fld.F90 SendRecvFlds on a single periodic rank. */
void orc_send_recv_flds(const orc_grid *g, double *Fx, double *Fy, double *Fz);
/* comm_fld.F90 UpdateCurrentAllFaces on a single periodic rank. */
void orc_update_current_all_faces(const orc_grid *g, double *Jx, double *Jy, double *Jz);
/* current.F90 smoothen_current (curr_filter passes of MovingAverageFilter). */
void orc_filter_current(const orc_grid *g, double *Jx, double *Jy, double *Jz, int passes);
/* current.F90 ResetCurrent */
void orc_reset_current(const orc_grid *g, orc_fields *f);

/* movdep.F90 MoveDepositPrtl (gather, Boris push, zigzag deposit, reduce). */
void orc_move_deposit(const orc_grid *g, orc_particles *p, orc_fields *f);

/* loadprtlout.F90 LoadPrtlOutliers + comm_prtl.F90 AppendParticles on a single
   periodic rank.  Returns 0, or -1 when the particle capacity is exceeded. */
int orc_exchange_particles(const orc_grid *g, orc_particles *p);
/* Walls along x on one rank (xborders = 0), src/bc/bc_reflect.F90: pos in
   cells from the first interior cell (bc_face%pos_prtl / pos_fld).
   RefBC_Prtl_Left/Right (:135-155): specular reflection of the particles
   beyond the wall and ReflCurrentLeft/Right (:195-237) of the current;
   CondBC_Fld_Left/Right (:43-72): tangential E zeroed beyond the wall. */
void orc_refl_prtl_left(const orc_grid *g, orc_particles *p, orc_fields *f, double pos);
void orc_refl_prtl_right(const orc_grid *g, orc_particles *p, orc_fields *f, double pos);
void orc_cond_fld_left(const orc_grid *g, orc_fields *f, double pos);
void orc_cond_fld_right(const orc_grid *g, orc_fields *f, double pos);
/* The y faces (bc_reflect.F90:11-41 CondBC_Fld_Top/Bottom, :79-128
   RefBC_Prtl_Top/Bottom with their own current fold). */
void orc_refl_prtl_bottom(const orc_grid *g, orc_particles *p, orc_fields *f, double pos);
void orc_refl_prtl_top(const orc_grid *g, orc_particles *p, orc_fields *f, double pos);
void orc_cond_fld_bottom(const orc_grid *g, orc_fields *f, double pos);
void orc_cond_fld_top(const orc_grid *g, orc_fields *f, double pos);
/* RemovePrtl_Left / RemovePrtl_Right (bc_open.F90:8-62) for face 1..6 (x, y,
   z; low, high): the particles beyond bc_pos_local(face, pos) = pos + 3
   (bc.F90:350-363) become holes. */
void orc_remove_prtl(const orc_grid *g, orc_particles *p, int face, double pos);
/* Field faces of EnforceBC_Final (bc.F90:292-340): Attenuate_EM_Vacuum
   (bc_attenuate.F90:151-290), Attenuate_EM_Flow with a uniform flow
   (:16-131), OpenBC_Fld_Left/Right (bc.F90:411-469). */
void orc_attn_vacuum(const orc_grid *g, orc_fields *f, int faces, const double *pos, const double *scale);
void orc_attn_flow(const orc_grid *g, orc_fields *f, int side, double pos, double dl, double scale, const double *b,
                   const double *v);
void orc_open_fld_right(const orc_grid *g, orc_fields *f, double pos);
void orc_open_fld_left(const orc_grid *g, orc_fields *f, double pos);
/* OpenBC_Prtl_Left (side 0) / Right (side 1), bc.F90:478-621, layer width dx. */
int orc_open_prtl(const orc_grid *g, orc_particles *p, int side, double pos, double dx);
/* InjectNewPrtl (bc_inflow.F90:134-256) for a uniform density and drift. */
typedef struct {
    int32_t face;
    double pos, speed, vmax, epc, density, drift[3];
    int32_t nspecies, flv[4];
    double temp[4], charge[4];
    uint32_t seed, call;
} orc_inflow;
int64_t orc_inject(const orc_grid *g, orc_particles *p, const orc_inflow *f);
/* RefPrtlFluidFrameRight (bc_inflow.F90:62-121) with DepositCurrentPIC. */
void orc_refl_fluid_right(const orc_grid *g, orc_particles *p, orc_fields *f, double pos, double vx);
/* Convolutional PML (bc_pml.F90): bit n-1 of `faces` marks bc_face(n) as
   'pml' at pos[n-1] with attn_thickness thickness[n-1] (SetBC_Fld default 4),
   with SetPMLParameters' profile (n = 4, kappa_max = 1, sigma_max = 1,
   alpha_max = 9e-4); psiE / psiB are pml_E_psi1 x, y, z, pml_E_psi2 x, y, z
   and the same for B, each a zeroed ghosted grid.  orc_pml_b is
   UpdateMagFld_PML (:146-264), called after the second B half step;
   orc_pml_e is UpdateElcFld_PML (:83-144), after the E update.  Neither
   refreshes the halo: SendRecvFlds follows each in MAIN.F90:104-110. */
typedef struct {
    int32_t faces;
    double pos[6], thickness[6];
    double *psiE[6], *psiB[6];
} orc_pml;
void orc_pml_b(const orc_grid *g, orc_fields *f, orc_pml *p);
void orc_pml_e(const orc_grid *g, orc_fields *f, orc_pml *p);

/* mem_prtl.F90 ReorderPrtlArr: stable counting sort by cell key; holes dropped.
   If perm is non-NULL it receives, for each output slot, the input slot. */
void orc_reorder(const orc_grid *g, orc_particles *p, int64_t *perm);

/* One time step of src/MAIN.F90:42-284 (single rank, periodic, curr_filter=0,
   no setup hooks).  t is the step counter used by the reorder period test. */
int orc_step(const orc_grid *g, orc_particles *p, orc_fields *f, int t, int reorder_period);
/* orc_step with curr_filter passes of the current filter (MAIN.F90:156-165). */
int orc_step_filtered(const orc_grid *g, orc_particles *p, orc_fields *f, int t, int reorder_period, int curr_filter);

/* savedata_routines.F90 CalcFldEnergy (sums, not halved): out[0]=sum|B|^2,
   out[1]=sum|E|^2 over the interior 3..m-3. */
void orc_field_energy(const orc_grid *g, const orc_fields *f, double out[2]);
/* OpenMP build: 1 = sum each cell's current in particle order, bit for bit
   the serial build's result at any thread count; 0 (default) = thread
   slices as the reference's OPEN_MP path.  No effect in the serial build. */
void orc_set_exact_order(int on);
/* savedata_routines.F90 CalcPrtlEnergy: energy[flv-1] per species. */
void orc_particle_energy(const orc_grid *g, const orc_particles *p, double masse, double massi, double *energy);
/* L-infinity norm over interior nodes of divE - rho, with divE as in
   savedata_routines.F90:329-348 (backward differences) and rho the CIC
   deposit of q*qi at nodes folded periodically.  rho_max receives max|rho| of
   the positive species alone (a scale for the residual). */
double orc_gauss_residual(const orc_grid *g, const orc_fields *f, const orc_particles *p, double *rho_max);

/* Philox-4x32-10 (Salmon et al., SC'11). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double orc_u01(uint32_t hi, uint32_t lo);

/* Weibel loader: two InitPrtl calls as in setup_weibel.F90:23-24, positions
   by init_prtl.F90:177-221, momenta by prob_dist.F90:13-70,223-254.
   The gfortran random_number stream is replaced by Philox-4x32-10 keyed by
   seed.  Returns the number of particles written, or -1 on overflow. */
typedef struct {
    int dims, nx, ny, nz;
    double epc;             /* trials per unit volume per call                  */
    double density;         /* acceptance threshold Den() (setup_weibel:46-49) */
    double drift;           /* |v| of the beams along x (beta if <1, gamma if >1) */
    double temp_ion, temp_elc; /* Temp = 2 kT/mc^2 per species (prob_dist:12)    */
    uint32_t seed;
} orc_weibel;
int64_t orc_load_weibel(const orc_weibel *w, orc_particles *p);
/* The Maxwell-Boltzmann inverse-CDF tables of prob_dist.F90:34-54 (N=10000). */
void orc_maxbolt_table(int n, double *x_table, double *pdf_table);

/* ---- cylindrical (r, theta, z), pictor_oracle_cyl.c ---------------------
   x = r (axis at x = 3.5), y = theta (ny cells over 2 pi), z; 3D only.
   fdtd selects the B update: 0 = cyl_em_update.F90, 1 = cyl_em_update_lehe.F90. */
void orc_cyl_params(const orc_grid *g, double out[4]);    /* dtheta, ax_perm_area, 1/dtheta, rshift */
void orc_cyl_update_b_half(const orc_grid *g, orc_fields *f);
void orc_cyl_update_e(const orc_grid *g, orc_fields *f);
void orc_cyl_add_current(const orc_grid *g, orc_fields *f);
void orc_cyl_send_recv_flds(const orc_grid *g, double *Fx, double *Fy, double *Fz);
void orc_cyl_fold(const orc_grid *g, double *Jx, double *Jy, double *Jz);
void orc_cyl_move_deposit(const orc_grid *g, orc_particles *p, orc_fields *f);
int orc_cyl_exchange(const orc_grid *g, orc_particles *p);
int orc_cyl_step(const orc_grid *g, orc_particles *p, orc_fields *f, int t, int reorder_period);
int64_t orc_cyl_load_uniform(const orc_grid *g, int npx, int npy, int npz, double density, double temp, double charge,
                             int flv, uint32_t seed, orc_particles *p);
void orc_cyl_field_energy(const orc_grid *g, const orc_fields *f, double out[2]);
extern int orc_cyl_max_substeps;
extern int64_t orc_cyl_substep_overruns;

#ifdef __cplusplus
}
#endif
#endif
