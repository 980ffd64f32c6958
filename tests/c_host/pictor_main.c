/*
 * pictor_main.c -- a compiled host for libpictor_b200 that makes the calls
 * of the reference's main loop (src/MAIN.F90:42-284, the `#ifdef gpu`
 * branch) in its order, through the C ABI of include/pictor_b200.h:
 *
 *   InitAll_gpu                  pic_create + pic_load_particles
 *   do t = 1, nsteps
 *     UpdateBfieldHalfGPU        pic_update_b_half
 *     MoveDepositPrtlGPU         pic_move_deposit
 *     ExchangePrtlGPU            pic_exchange_particles
 *     UpdateBfieldHalfGPU        pic_update_b_half
 *     UpdateEfieldGPU            pic_update_e
 *     UpdateCurrentsAllEdgesGPU  pic_fold_current
 *     smoothen_current_gpu       pic_filter_current
 *     AddCurrentGPU              pic_add_current
 *     CopyGPUDataToHostForOutput pic_fetch_fields + pic_fetch_particles (every
 *                                `output` steps, into the host arrays)
 *     ResetCurrentGPU            pic_reset_current
 *     ReorderPrtlGPU             pic_reorder (every `period` steps)
 *   end do
 *
 * The single periodic rank of a setup such as setup_weibel.F90, whose
 * EnforceBC_*, PostMovDep, PreAddCurrent and Finalsubroutines hooks do
 * nothing.  Input and output are raw little-endian files:
 *   in:  int64 n, then q, x, y, z, u, v, w (n doubles each), flv (n int32)
 *   out: the same for the fetched particles, then Ex, Ey, Ez, Bx, By, Bz
 *        ((nx+5)(ny+5)(nz+5 or 1) doubles each, column-major) of the last
 *        fetch, which the host makes after the last step.
 * Usage: pictor_main dims nx ny nz c qi nsteps period output exact in out
 * Exit status 0, or the failing call's PIC_ERR_* code as a positive number.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "pictor_b200.h"

#define CALL(x)                                                                  \
    do {                                                                         \
        int rc_ = (x);                                                           \
        if (rc_ != PIC_OK) {                                                     \
            fprintf(stderr, "%s: %s (%d)\n", #x, pic_error_string(rc_), rc_);    \
            return -rc_;                                                         \
        }                                                                        \
    } while (0)

static int read_all(FILE *f, void *p, size_t bytes) { return fread(p, 1, bytes, f) == bytes ? 0 : -1; }

int main(int argc, char **argv)
{
    if (argc != 13) {
        fprintf(stderr, "usage: %s dims nx ny nz c qi nsteps period output exact in out\n", argv[0]);
        return 64;
    }
    pic_config cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.dims = atoi(argv[1]);
    cfg.nx = atoi(argv[2]);
    cfg.ny = atoi(argv[3]);
    cfg.nz = atoi(argv[4]);
    cfg.c = atof(argv[5]);
    cfg.qi = atof(argv[6]);
    const int nsteps = atoi(argv[7]);
    const int period = atoi(argv[8]);
    const int output = atoi(argv[9]);
    cfg.exact_current = atoi(argv[10]);
    cfg.geom = PIC_GEOM_CARTESIAN;
    cfg.fdtd = PIC_FDTD_YEE;
    cfg.precision = PIC_PREC_FP64;
    cfg.nflvr = 2;              /* AllocatePrtlVars: flavour 1 ions, 2 electrons */
    cfg.qm[1] = 1.0;            /* mi = me: pair plasma */
    cfg.qm[2] = -1.0;
    cfg.reorder_period = 0;     /* the host calls the reorder itself */
    cfg.inc_axis = 1;

    FILE *fi = fopen(argv[11], "rb");
    if (!fi) return 66;
    int64_t n = 0;
    if (read_all(fi, &n, sizeof n) || n < 0) return 65;
    cfg.capacity = 2 * n + 65536;
    double *a[7];
    for (int k = 0; k < 7; k++) {
        a[k] = (double *)malloc((size_t)cfg.capacity * sizeof(double));
        if (!a[k] || read_all(fi, a[k], (size_t)n * sizeof(double))) return 65;
    }
    int32_t *flv = (int32_t *)malloc((size_t)cfg.capacity * sizeof(int32_t));
    if (!flv || read_all(fi, flv, (size_t)n * sizeof(int32_t))) return 65;
    fclose(fi);

    pic_handle *h = NULL;
    CALL(pic_create(&cfg, &h));
    CALL(pic_load_particles(h, n, a[0], a[1], a[2], a[3], a[4], a[5], a[6], flv));
    const size_t nf = (size_t)(cfg.nx + 5) * (size_t)(cfg.ny + 5) * (size_t)(cfg.dims == 3 ? cfg.nz + 5 : 1);
    double *F[6];
    for (int k = 0; k < 6; k++) {
        F[k] = (double *)calloc(nf, sizeof(double));
        if (!F[k]) return 70;
    }
    int64_t got = n;
    for (int t = 1; t <= nsteps; t++) {
        CALL(pic_update_b_half(h));
        CALL(pic_move_deposit(h));
        CALL(pic_exchange_particles(h));
        CALL(pic_update_b_half(h));
        CALL(pic_update_e(h));
        CALL(pic_fold_current(h));
        CALL(pic_filter_current(h));
        CALL(pic_add_current(h));
        if ((output > 0 && t % output == 0) || t == nsteps) {
            int64_t cnt = 0;
            CALL(pic_particle_count(h, &cnt));
            if (cnt > cfg.capacity) return 71;
            CALL(pic_fetch_fields(h, F[0], F[1], F[2], F[3], F[4], F[5], NULL, NULL, NULL));
            CALL(pic_fetch_particles(h, &got, a[0], a[1], a[2], a[3], a[4], a[5], a[6], flv));
        }
        CALL(pic_reset_current(h));
        if (period > 0 && t % period == 0) CALL(pic_reorder(h));
    }
    pic_destroy(h);

    FILE *fo = fopen(argv[12], "wb");
    if (!fo) return 73;
    fwrite(&got, sizeof got, 1, fo);
    for (int k = 0; k < 7; k++) fwrite(a[k], sizeof(double), (size_t)got, fo);
    fwrite(flv, sizeof(int32_t), (size_t)got, fo);
    for (int k = 0; k < 6; k++) fwrite(F[k], sizeof(double), nf, fo);
    fclose(fo);
    return 0;
}
