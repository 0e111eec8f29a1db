/*
 * mhd_gpu_dropin.h -- the reference's own hot-path entry points, implemented
 * on the GPU (mhd2dcfdfftw_open_b200/csrc/dropin.c, archive
 * libmhdgpu_dropin.a, which calls libmhdgpu.so).
 *
 * Same names, signatures and effects as the reference's routines; they act on
 * the reference's global arrays and parameters (declared in the reference's
 * initialize.h:11-69 and defined by its initialize.c), so the reference's
 * driver mhd.c, with initialize.c, usrInitialize.c, writeOutput.c and
 * divBcleaning.c, links against this layer unchanged in place of
 * calcDerivs.o, calcRHS.o, filtering.o, timeAdvance.o and parallel.o.
 *
 * By default every call copies the global arrays it reads to the device and
 * the arrays it writes back to the host, so the host globals always hold
 * what the reference would hold (checkDivB and writeArray in mhd.c read them
 * directly).  Resident mode (below) keeps the arrays on the device instead.  The device work runs on one context created on the first call
 * from the globals that initialize() set (device 0, or MHDGPU_DEVICE).
 * Errors: these functions return void as the reference's do; a failure is
 * reported once on stderr and by mhdgpu_last_error().  Periodic x boundary
 * only (boundaryTypeX = 0).
 */
#ifndef MHD_GPU_DROPIN_H
#define MHD_GPU_DROPIN_H

#ifdef __cplusplus
extern "C" {
#endif

/* calcDerivs.h:6-15 (calcDerivs.c:9-150) */
void derivX(int nv, double *arrMain, double *arrHalo0, double *arrHalo1, double *arrDeriv,
            int iVarStartMain, int iVarStartHalo);
void derivXX(int nv, double *arrMain, double *arrHalo0, double *arrHalo1, double *arrDeriv,
             int iVarStartMain, int iVarStartHalo);
void derivY(int nv, double *arrMain, double *arrDeriv, int iVarStartMain);
void derivYY(int nv, double *arrMain, double *arrDeriv, int iVarStartMain);
/* calcRHS.h:4-6 (calcRHS.c:13-75) */
void calcRHS(void);
void calcDivB(void);
void calcEfield(void);
/* filtering.h:6 (filtering.c:98-102) */
void filtering(void);
/* timeAdvance.h:6-8 (timeAdvance.c:20-153) */
void rkInit(double dt);
void rkExecute(int iRK);
double calcDt(double dt0);
/* parallel.h:4-6 (parallel.c:4-189): the 2-point periodic halos, filled on
 * the host as the reference's single-rank exchange fills them */
void sendrecvHaloPointsX(void);
void sendrecvHaloPointsdivBX(void);
void sendrecvHaloPointsEfieldX(void);

/* Resident mode (no counterpart in the reference): 1 keeps the global arrays
 * on the device between calls -- each array is uploaded on its first use
 * only, results stay on the device and the halo exchanges become no-ops (the
 * kernels wrap periodically); 0 returns to copying on every call (and first
 * brings the host up to date).  MHDGPU_DROPIN_RESIDENT=1 in the environment
 * turns it on before the first call.  A driver then calls
 * mhdgpu_dropin_sync_host() before it reads globals itself (for mhd.c: before
 * each checkDivB/writeArray), and mhdgpu_dropin_sync_device() after it writes
 * globals itself once the run has started (they are uploaded again on next
 * use).  Changing a parameter global re-creates the context from the host
 * arrays: sync the host first. */
void mhdgpu_dropin_resident(int on);
void mhdgpu_dropin_sync_host(void);
void mhdgpu_dropin_sync_device(void);

#ifdef __cplusplus
}
#endif
#endif
