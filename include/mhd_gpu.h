/*
 * mhd_gpu.h -- C ABI of the B200 (sm_100a) implementation of the per-step
 * hot path of the 2-D compressible MHD solver MHD2DCFDFFTW.
 *
 * Two layers, both plain C (no C++ or torch types cross this boundary):
 *
 *  1. Handle-based API (mhdgpu_*): a context owns one 2-D periodic domain on
 *     one GPU -- the state uu[NVAR][nx][ny], dudtRK and the derivative arrays
 *     that the reference keeps as globals (initialize.h:11-69) -- and exposes
 *     the reference's operators on it, whole RK3 stages and steps.
 *  2. Drop-in layer: the reference's own entry points (derivX, derivY,
 *     calcRHS, filtering, rkExecute, calcDt, ...) with the reference's
 *     signatures, implemented over the reference's globals in
 *     mhd2dcfdfftw_open_b200/csrc/dropin.c.  Declared in mhd_gpu_dropin.h.
 *
 * Layout: every field array is C order [nfield][nx][ny] of doubles
 * (macros.h:4-24), y contiguous.  Variable order: rho, ux, uy, uz, Bx, By,
 * Bz, p (and psi with hyperbolic cleaning).
 *
 * Errors: every call returns an mhdgpu_status; nothing traps or exits.
 * mhdgpu_last_error() repeats the last non-OK status of the calling thread.
 */
#ifndef MHD_GPU_H
#define MHD_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* The 15 lines of the reference's `input` file, in their order
 * (input:1-15, parsed by readInput at initialize.c:456-525). */
typedef struct {
    int boundaryTypeX;   /* 0 periodic (supported), 1 open (rejected)      */
    double cfl;
    double Tmax;
    double dtOut;
    long nx;
    long ny;             /* even, power of two, 8..8192                    */
    double Lx;
    double Ly;
    double adiabaticIdx;
    int Hall;            /* enters the CFL speed and forces d2B (no E term) */
    double di;
    double resistivity;
    double viscosity;
    int divBcleaning;    /* 0 none, 1 diffusive, 2 hyperbolic (NVAR = 9)   */
    int outDivB;
} mhdgpu_params;

typedef enum {
    MHDGPU_OK = 0,
    MHDGPU_ERR_INVALID = 1,      /* bad argument or size                   */
    MHDGPU_ERR_UNSUPPORTED = 2,  /* configuration outside the GPU path     */
    MHDGPU_ERR_CUDA = 3,         /* a CUDA runtime call failed             */
    MHDGPU_ERR_NOMEM = 4,        /* device allocation failed               */
    MHDGPU_ERR_TIMEOUT = 5,      /* a bounded on-device wait ran out       */
    MHDGPU_ERR_NONFINITE = 6     /* the state holds NaN/Inf or rho,p <= 0  */
} mhdgpu_status;

/* Arrays of a context, named after the reference's globals
 * (initialize.h:19-27).  Field counts: NVAR for UU/DUDX/DUDY/DUDT/DUDTRK,
 * 3 for the second derivatives and the electric field, 1 for divB. */
typedef enum {
    MHDGPU_UU = 0, MHDGPU_DUDX, MHDGPU_DUDY, MHDGPU_D2UDX2, MHDGPU_D2UDY2,
    MHDGPU_D2BDX2, MHDGPU_D2BDY2, MHDGPU_DIVB, MHDGPU_DDIVBDX, MHDGPU_DDIVBDY,
    MHDGPU_EFIELD, MHDGPU_DEDX, MHDGPU_DEDY, MHDGPU_DUDT, MHDGPU_DUDTRK,
    MHDGPU_NARRAYS
} mhdgpu_array;

typedef struct mhdgpu_ctx mhdgpu_ctx;

/* --- lifetime (replaces initialize()/finalize(), initialize.c:87-419) --- */
int mhdgpu_read_input(const char *path, mhdgpu_params *out);
int mhdgpu_create(const mhdgpu_params *p, int device, mhdgpu_ctx **out);
void mhdgpu_destroy(mhdgpu_ctx *ctx);
int mhdgpu_last_error(void);
const char *mhdgpu_error_string(int status);
int mhdgpu_nvar(const mhdgpu_ctx *ctx);

/* --- host <-> device --------------------------------------------------- */
int mhdgpu_set_array(mhdgpu_ctx *ctx, int which, const double *host);
int mhdgpu_get_array(mhdgpu_ctx *ctx, int which, double *host);
/* device address of a context array (for callers that keep data resident) */
double *mhdgpu_device_array(mhdgpu_ctx *ctx, int which);
int mhdgpu_synchronize(mhdgpu_ctx *ctx);

/* --- operators on the context's arrays, mirroring the reference --------
 * Each replaces the reference routine cited; all run asynchronously on the
 * context's stream.                                                        */
/* derivX / derivXX (calcDerivs.c:9-72): out[v] = d/dx (d2/dx2) of
 * in[v + start], v < nv.  `in`/`out` are context arrays (mhdgpu_array). */
int mhdgpu_deriv_x(mhdgpu_ctx *ctx, int nv, int in, int start, int out, int order);
/* derivY / derivYY (calcDerivs.c:75-150) */
int mhdgpu_deriv_y(mhdgpu_ctx *ctx, int nv, int in, int start, int out, int order);
int mhdgpu_calc_efield(mhdgpu_ctx *ctx);   /* calcEfield, calcRHS.c:24-43 */
int mhdgpu_calc_divb(mhdgpu_ctx *ctx);     /* calcDivB, calcRHS.c:13-22 */
int mhdgpu_calc_rhs(mhdgpu_ctx *ctx);      /* calcRHS, calcRHS.c:46-75,498-544 */
int mhdgpu_rk_init(mhdgpu_ctx *ctx, double dt);      /* rkInit, timeAdvance.c:20-27 */
int mhdgpu_rk_execute(mhdgpu_ctx *ctx, int iRK);     /* rkExecute, timeAdvance.c:29-36 */
int mhdgpu_filtering(mhdgpu_ctx *ctx);     /* filtering, filtering.c:98-102 */
/* calcDt (timeAdvance.c:38-153); also sets Ch/Cp for hyperbolic cleaning */
int mhdgpu_calc_dt(mhdgpu_ctx *ctx, double dt0, double *dt_out);
/* checkDivB (mhd.c:342-367): max |dudx[Bx] + dudy[By]|, fills DIVB */
int mhdgpu_check_divb(mhdgpu_ctx *ctx, double *maxdivb);
int mhdgpu_get_cleaning_speeds(mhdgpu_ctx *ctx, double *Ch, double *Cp);

/* --- whole stages and steps ------------------------------------------- */
/* One RK3 stage, the body of mhd.c:154-199, through the operators above. */
int mhdgpu_stage(mhdgpu_ctx *ctx, int iRK);
/* nsteps RK3 steps.  dt_fixed > 0: fixed dt (calcDt still sets Ch/Cp with
 * hyperbolic cleaning); dt_fixed <= 0: the reference's CFL control
 * (mhd.c:58-63, 201-206).  *dt_io carries dt in and out. */
int mhdgpu_steps(mhdgpu_ctx *ctx, int nsteps, double dt_fixed, double *dt_io);
/* Same steps through the fused two-pass stage (x pass + y pass per stage). */
int mhdgpu_steps_fused(mhdgpu_ctx *ctx, int nsteps, double dt_fixed, double *dt_io);
/* A stream of independent states (no counterpart in the reference): for r <
 * nstates, the state (NVAR*nx*ny doubles, the uu layout) at h_in[r] is
 * advanced by nsteps fused steps, each from *dt_io as mhdgpu_steps_fused
 * would after mhdgpu_set_array(UU), and written to h_out[r] (no h_out[r] may
 * overlap an h_in[k], k > r; the same pointer may repeat within h_in and
 * within h_out).  Uploads and downloads run on
 * their own streams while the previous/next state steps; page-locked host
 * buffers let them overlap.  *dt_io returns the last state's dt.  Afterwards
 * the context holds the last state, as after mhdgpu_steps_fused. */
int mhdgpu_steps_fused_stream(mhdgpu_ctx *ctx, int nstates, const double *const *h_in,
                              double *const *h_out, int nsteps, double dt_fixed, double *dt_io);

/* Arithmetic of mhdgpu_steps_fused (no counterpart in the reference, which
 * computes in FP64 only).  MHDGPU_PRECISION_FP64 (the default) follows the
 * reference's numerics.  MHDGPU_PRECISION_MIXED keeps the state, dudtRK,
 * the RK3 update, the CFL time step and the right-hand sides of the compact
 * schemes in FP64, and runs the tridiagonal sweeps, the FFT butterflies and
 * the fluxes in FP32; the derivatives are stored as FP32 and the x and y
 * filters are applied as an FP32 change added to the FP64 state.  After
 * mixed steps the derivative arrays hold FP32 scratch (mhdgpu_check_divb then
 * returns MHDGPU_ERR_UNSUPPORTED until an FP64 step has run).  Mixed
 * precision needs the fused path: 16 <= ny <= 8192, a grid the fused x pass
 * tiles, and divBcleaning 0 or 2; otherwise MHDGPU_ERR_UNSUPPORTED. */
enum { MHDGPU_PRECISION_FP64 = 0, MHDGPU_PRECISION_MIXED = 1 };
int mhdgpu_set_precision(mhdgpu_ctx *ctx, int precision);

/* Autotuner of the fused x pass (no counterpart in the reference): times the
 * pass for each tile width this grid admits (8, 16, 32 columns per CTA; the
 * rows per CTA and the cluster size follow from it) at the context's current
 * precision, keeps the fastest and remembers it for contexts of the same
 * shape created later in this process (a shape already tuned in this
 * process keeps its width, so runs repeat bit for bit).  The state is only
 * read; the derivative arrays are overwritten.  *columns_out: the width
 * chosen (may be NULL); 0 when the context takes the chunked x pass (lines
 * of 1024 rows and more), which has no width to choose and was measured
 * faster than every width of the cluster pass there.
 * MHDGPU_ERR_UNSUPPORTED when the grid has no fused x pass. */
int mhdgpu_autotune(mhdgpu_ctx *ctx, int *columns_out);

/* --- diagnostics -------------------------------------------------------- */
/* total energy and cross helicity of the state (sums times dx*dy);
 * *finite = 0 if the state holds a NaN or an Inf.  (No counterpart in the
 * reference, which prints energies from its driver, mhd.c:292-299.) */
int mhdgpu_diagnostics(mhdgpu_ctx *ctx, double *energy, double *cross_helicity,
                       int *finite);
/* cells of the state holding a NaN or Inf, and finite cells whose density or
 * pressure is not positive (the reference carries on through such states:
 * its calcDt only drops their NaN speeds).  No counterpart in the reference. */
int mhdgpu_state_cells(mhdgpu_ctx *ctx, long *nonfinite, long *nonpositive);

/* --- allocation-free time step ---------------------------------------------
 * No counterpart in the reference.  The CFL time step of calcDt for callers
 * that cannot allocate device memory (a framework whose pool allocator owns
 * the device's memory, a service that fixes its footprint at start-up): no
 * context, no allocation, no host synchronisation.  d_uu: the state
 * [NVAR][nx][ny] on the current device; d_out: 3 device doubles receiving
 * dt (after the 2% hysteresis against dt0), Ch and Cp (hyperbolic cleaning,
 * else 0); stream: a cudaStream_t (NULL: the default stream), the call is
 * asynchronous on it.  Scratch is a fixed 96 KiB device array held by every
 * GPU that loads the library: nx*ny is limited to 33,554,432 cells, larger
 * grids return MHDGPU_ERR_INVALID.  Calls share that array: calls that
 * overlap on the GPU race and must be serialised by the caller.  The first
 * call on a device looks the array up with that device current; make it
 * before any stream capture begins.  States with NaN or non-positive
 * density give what the reference's calcDt gives (as mhdgpu_calc_dt does):
 * its MAX/MIN macros per cell and its running minimum over the cells.  Use
 * mhdgpu_diagnostics to detect a non-finite state. */
int mhdgpu_calc_dt_noalloc(const double *d_uu, const mhdgpu_params *p, double dt0,
                           double *d_out, void *stream);

/* --- instrumentation ---------------------------------------------------- */
/* the context's CUDA stream (a cudaStream_t), for callers that time or order
 * work around the library's launches */
void *mhdgpu_stream(mhdgpu_ctx *ctx);
/* number of kernels this context has launched so far */
long mhdgpu_launch_count(const mhdgpu_ctx *ctx);
/* Self-test of the bounded waits (no counterpart in the reference): runs a
 * kernel whose mbarrier wait is never satisfied, with a limit of
 * `milliseconds` (0 < ms <= 2000).  Returns MHDGPU_ERR_TIMEOUT, read from the
 * context's status flag exactly as a stalled TMA copy in the x kernels would
 * be reported; the flag is cleared and the context stays usable. */
int mhdgpu_selftest_wait(mhdgpu_ctx *ctx, double milliseconds);
/* enable (1) / disable (0) CUDA-event bracketing of every launch; enabling
 * clears the record */
int mhdgpu_profile(mhdgpu_ctx *ctx, int enable);
/* total device time, launch count and algorithmic bytes (what the launches
 * must read and write at least) recorded for a kernel class:
 * 0 x-line solver, 1 y spectral, 2 pointwise, 3 reductions,
 * 4 fused x pass (x derivatives on long lines), 5 fused y pass,
 * 6 x filter of the fused steps on long lines */
int mhdgpu_profile_read(mhdgpu_ctx *ctx, int kclass, double *total_ms, long *count,
                        double *bytes);

#ifdef __cplusplus
}
#endif
#endif
