/*
 * Oracle harness (test infrastructure only).
 *
 * Drives the reference solver's own, unmodified functions -- compiled from
 * the reference sources with the single-rank MPI and FFTW-API shims in
 * oracle/shim -- in place of the reference's main program (mhd.c) and its
 * hard-coded initial conditions (usrInitialize.c):
 *   - ref_setup():   initialize() from ./input in a work directory
 *                    (initialize.c:87-395);
 *   - ref_stage():   one RK3 stage, calling the reference's functions in the
 *                    order of the stage loop body at mhd.c:154-199;
 *   - ref_steps():   whole RK3 steps, with either a fixed dt (rkInit only) or
 *                    the reference's CFL update (mhd.c:201-206);
 *   - ref_check_divb(): max|dBx/dx + dBy/dy| as checkDivB (mhd.c:342-367).
 * Built as oracle/_ref/libmhdref.so (driven from Python with ctypes) and as
 * oracle/_ref/mhd_ref, a command-line timer used as the CPU baseline.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>
#include <math.h>

#include "macros.h"
#include "parameter.h"
#include "initialize.h"
#include "timeAdvance.h"
#include "parallel.h"
#include "calcDerivs.h"
#include "calcRHS.h"
#include "filtering.h"

extern real constDiffDivB;

/* Work directory holding ./input; initialize() reads it from the cwd. */
int ref_setup(const char *workdir)
{
    char old[4096];
    if (!getcwd(old, sizeof old)) return 1;
    if (chdir(workdir) != 0) return 2;
    constDiffDivB = 2.0; /* initialize.c:154 scales this global in place */
    initialize();
    if (chdir(old) != 0) return 3;
    return 0;
}

long ref_nvar(void) { return NVAR; }
long ref_nx(void) { return (long)nx; }
long ref_ny(void) { return (long)ny; }

/* One RK3 stage: the reference's calls in the order of mhd.c:154-199. */
void ref_stage(int iRK)
{
    sendrecvHaloPointsX();
    derivX(NVAR, uu, uuHaloX0, uuHaloX1, dudx, 0, 0);
    derivY(NVAR, uu, dudy, 0);
    if (viscosity > 0) {
        derivXX(3, uu, uuHaloX0, uuHaloX1, d2udx2, 1, 1);
        derivYY(3, uu, d2udy2, 1);
    }
    if ((Hall == 1) || (resistivity > 0)) {
        derivXX(3, uu, uuHaloX0, uuHaloX1, d2Bdx2, 4, 4);
        derivYY(3, uu, d2Bdy2, 4);
    }
    if (divBcleaning == 1) {
        calcDivB();
        sendrecvHaloPointsdivBX();
        derivX(1, divB, divBHaloX0, divBHaloX1, ddivBdx, 0, 0);
        derivY(1, divB, ddivBdy, 0);
    }
    calcEfield();
    sendrecvHaloPointsEfieldX();
    derivX(3, Efield, EfieldHaloX0, EfieldHaloX1, dEdx, 0, 0);
    derivY(3, Efield, dEdy, 0);
    calcRHS();
    rkExecute(iRK);
    sendrecvHaloPointsX();
    filtering();
}

/*
 * Advance nsteps whole RK3 steps starting from the current uu.
 * dt_fixed > 0: every step uses dt_fixed (rkInit(dt_fixed)); with hyperbolic
 *   cleaning (divBcleaning==2) calcDt is still called before the first step
 *   and after every step, because it is what sets Ch/Cp (timeAdvance.c:107-112).
 * dt_fixed <= 0: the reference's own dt control -- dt = calcDt(dt) before the
 *   loop (mhd.c:58-63) and after every step (mhd.c:205-206).
 * Returns the wall seconds spent in the step loop; *dt_io carries dt in/out.
 */
double ref_steps(int nsteps, double dt_fixed, double *dt_io)
{
    double dt = dt_io ? *dt_io : 0.0;
    if (dt_fixed > 0) {
        if (divBcleaning == 2) (void)calcDt(dt_fixed);
        dt = dt_fixed;
    } else {
        dt = calcDt(dt);
    }
    rkInit(dt);
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (int s = 0; s < nsteps; s++) {
        for (int iRK = 0; iRK < 3; iRK++) ref_stage(iRK);
        if (dt_fixed > 0) {
            if (divBcleaning == 2) (void)calcDt(dt_fixed);
            dt = dt_fixed;
        } else {
            dt = calcDt(dt);
        }
        rkInit(dt);
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (dt_io) *dt_io = dt;
    return (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
}

/* max|dudx[BX] + dudy[BY]|, as checkDivB (mhd.c:342-367), which also leaves
 * the values in divB. */
double ref_check_divb(void)
{
    real maxDivB = 0;
    for (size_t i = 0; i < iSize; i++)
        for (size_t j = 0; j < jSize; j++) {
            divB[IDXIJ(0, i, j)] = dudx[BX(i, j)] + dudy[BY(i, j)];
            real t = fabs(divB[IDXIJ(0, i, j)]);
            if (t > maxDivB) maxDivB = t;
        }
    return maxDivB;
}

/* Load uu from an output-format file: one double (time) then NVAR*nx*ny
 * doubles in C order [NVAR][nx][ny] (writeOutput.c:47-76). */
int ref_load_state(const char *path)
{
    FILE *fp = fopen(path, "rb");
    if (!fp) return 1;
    double t;
    size_t n = (size_t)NVAR * nx * ny;
    int ok = fread(&t, sizeof t, 1, fp) == 1 && fread(uu, sizeof(real), n, fp) == n;
    fclose(fp);
    return ok ? 0 : 2;
}

int ref_save_state(const char *path, double t)
{
    FILE *fp = fopen(path, "wb");
    if (!fp) return 1;
    size_t n = (size_t)NVAR * nx * ny;
    int ok = fwrite(&t, sizeof t, 1, fp) == 1 && fwrite(uu, sizeof(real), n, fp) == n;
    fclose(fp);
    return ok ? 0 : 2;
}

#ifdef ORACLE_MAIN
/* Write every page of the reference's per-stage arrays once (they are
 * outputs, overwritten before they are read in each stage), so that the
 * first timed step runs on resident memory as every later step of the
 * reference's own loop does, instead of paying the first-touch page faults
 * of ~60 field-sized arrays. */
static void pretouch(void)
{
    size_t plane = iSize * jSize;
    real *full[] = {dudx, dudy, dudt};
    real *three[] = {d2udx2, d2udy2, d2Bdx2, d2Bdy2, Efield, dEdx, dEdy};
    real *one[] = {divB, ddivBdx, ddivBdy};
    for (size_t k = 0; k < sizeof full / sizeof *full; k++)
        if (full[k]) memset(full[k], 0, arrSize * sizeof(real));
    for (size_t k = 0; k < sizeof three / sizeof *three; k++)
        if (three[k]) memset(three[k], 0, 3 * plane * sizeof(real));
    for (size_t k = 0; k < sizeof one / sizeof *one; k++)
        if (one[k]) memset(one[k], 0, plane * sizeof(real));
}

/* mhd_ref <workdir> <state.dat> <nsteps> <dt> [out.dat [warmup [gofile]]]
 * Runs `warmup` untimed steps, then nsteps timed RK3 steps of the reference
 * from the given state (dt <= 0 uses the reference's CFL control) and prints
 * one JSON line with the timed step-loop seconds.  Used as the CPU baseline.
 * With `gofile`, it prints "READY" after the set-up and the warm-up (without
 * a warm-up: after writing every page of the stage arrays once, see
 * pretouch) and waits (at most 1800 s) until that file exists before the
 * timed steps, so that several concurrent processes time the same interval. */
int main(int argc, char **argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: %s workdir state.dat nsteps dt [out.dat|- [warmup [gofile]]]\n",
                argv[0]);
        return 2;
    }
    if (ref_setup(argv[1]) != 0) { fprintf(stderr, "setup failed\n"); return 1; }
    if (ref_load_state(argv[2]) != 0) { fprintf(stderr, "cannot read %s\n", argv[2]); return 1; }
    int nsteps = atoi(argv[3]);
    int warm = argc > 6 ? atoi(argv[6]) : 0;
    double dt = atof(argv[4]), dtio = 0.0;
    if (warm > 0) (void)ref_steps(warm, dt, &dtio);
    if (argc > 7) {
        if (warm <= 0) pretouch();
        printf("READY\n");
        fflush(stdout);
        struct timespec nap = {0, 1000000};
        int waited = 0;
        while (access(argv[7], F_OK) != 0) {
            if (++waited > 1800000) { fprintf(stderr, "no go file\n"); return 3; }
            nanosleep(&nap, NULL);
        }
    }
    double sec = ref_steps(nsteps, dt, &dtio);
    if (argc > 5 && strcmp(argv[5], "-") != 0) ref_save_state(argv[5], 0.0);
    double cells = (double)nx * (double)ny * (double)nsteps;
    printf("{\"nx\": %zu, \"ny\": %zu, \"steps\": %d, \"seconds\": %.6f, "
           "\"cell_updates_per_s\": %.6e, \"dt\": %.17g}\n",
           nx, ny, nsteps, sec, sec > 0 ? cells / sec : 0.0, dtio);
    return 0;
}
#endif
