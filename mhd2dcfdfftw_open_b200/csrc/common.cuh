// Shared definitions of the sm_100a MHD hot path: the context that mirrors
// the reference's globals (initialize.h:11-69), the compact-scheme constants
// (parameter.h:23-56, initializeCFDSchemes at initialize.c:572-631) and the
// error plumbing of the C ABI.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mhd_gpu.h"

namespace mhd {

enum Var { RHO = 0, UX, UY, UZ, BX, BY, BZ, P, PSI };

// Operators of the x-direction line solver.
enum XOp { XOP_D1 = 0, XOP_D2 = 1, XOP_F = 2 };

// Stencil coefficients of one x operator.  Interior rows use
//   D1: (a/2 (f+1 - f-1) + b/4 (f+2 - f-2) + c/6 (f+3 - f-3)) * s
//   D2: (a (f+1 - 2f + f-1) + b/4 (...) + c/9 (...)) * s
//   F : a f + b/2 (f+1 + f-1) + c/2 (f+2 + f-2) + d/2 (f+3 + f-3)
// and the two edge rows the 5-point closure e0..e4 over f-2..f+2 (row 0) or
// its mirror f+2..f-2 (row N-1, times `edge_sign`), exactly as mathlib.c:46-85,
// 176-217 and 309-353 write them.
struct XStencil {
    double a, b, c, d;          // interior coefficients (pre-divided as above)
    double e0, e1, e2, e3, e4;  // closure coefficients
    double scale;               // 1/dx, 1/dx^2 or 1
    double edge_sign;           // -1 for the last row of D1, else +1
    int kind;                   // XOp
};

// Thomas factors of one x operator for a line of n rows (non-cyclic system,
// unit diagonal; mathlib.c:8-30): m[i] = A[i-1]/B'[i-1], invB[i] = 1/B'[i],
// g[i] = C[i]/B'[i]; plus the partition products used by the split solve.
struct XTables {
    double *m, *invB, *g;       // device, n each
    double *pfw, *qbw;          // device, n each (see xsolve.cu)
    int n, nsub_total;          // rows, sub-chunks of the partition
};

#define MHD_MAX_CLUSTER 16
#define MHD_PROF_MAX 8192

// kernel classes for the event-timing hooks (mhdgpu_profile_read)
enum KClass { KC_XSOLVE = 0, KC_YSPEC, KC_POINTWISE, KC_REDUCE, KC_FUSED_X, KC_FUSED_Y,
              KC_FUSED_XF, KC_NCLASS };

struct Ctx {
    mhdgpu_params p;
    int nvar;
    long nx, ny;
    double dx, dy, const_diff_divb;
    int device;
    int sm_count;
    cudaStream_t stream;
    // the reference's global arrays, on the device
    double *arr[MHDGPU_NARRAYS];
    int arr_fields[MHDGPU_NARRAYS];
    // x operator tables
    XStencil xs[3];
    XTables xt[3];
    int x_cluster, x_rows_per_cta, x_sub_rows;
    // y spectral tables
    double2 *tw;                 // exp(-2 pi i m / ny), m < ny
    double *ysym_d1, *ysym_d2, *ysym_f;  // per signed wavenumber, ny each
    // FP32 copies for the mixed-precision stage: twiddles, d/dy, d2/dy2 and
    // filter-minus-identity symbols, ny float2 each
    float2 *ytab32;
    int mixed;       // fused steps in mixed precision (FP32 operators, FP64 state)
    int deriv_fp32;  // the derivative arrays hold FP32 scratch of mixed steps
    // device step control of the fused steps: dt, Ch, Cp live in dscal and
    // the y pass forms its RK3 coefficients there; one step is captured as a
    // CUDA graph per (precision, CFL or fixed dt) and replayed
    int dev_dt;
    cudaGraphExec_t step_graph[2][2];
    long step_graph_launches[2][2];
    // scalars on the device: [0] dt, [1] Ch, [2] Cp, [3..] scratch
    double *dscal;
    double *dred;                // block partials of reductions
    int *dflag;                  // bounded-wait / status flags
    int nred;
    // time integration
    double cc[3], dd[3];
    double Ch, Cp;
    double dt;
    // fused path
    int fused_pending_filter;    // 1: uu still needs the x filter
    // instrumentation: launch counter and per-kernel-class event timing
    long launches;
    int prof_on;
    int prof_n;
    cudaEvent_t *prof_ev;        // 2 * MHD_PROF_MAX events (begin, end)
    int *prof_cls;
    double prof_bytes[8];        // algorithmic bytes of the profiled launches per class
    // fused x pass: Thomas factor edge tables and interior constants, tiling
    double *xf_edge;
    double xf_inner[2][3];
    int xf_W, xf_C, xf_R;
    int xf_hops;          // CTAs whose totals enter an inflow of the fused x pass
    double xf_pw[2][2];   // interior sub-chunk products (-m)^S, (-g)^S per matrix
    double xf_alphaF[2];  // filter matrix off-diagonal: interior, edge rows
    CUtensorMap xl_tmap_big, xl_tmap_unit;  // uu as [nvar*nx rows][ny] for the x pass
    // chunked x pass of long lines (xfir.cu): the x filter writes the filtered
    // state to xn_state, from which the derivatives and the y pass read it
    void *xn;                    // host side (parameter blocks, device tables)
    int xn_on;                   // the fused steps use it
    double *xn_state;            // nvar planes
    int state_in_S;              // the current, x-filtered state is in xn_state
    // streaming of independent states (mhdgpu_steps_fused_stream): device
    // staging copies of an incoming and an outgoing state, the copy streams
    // and their events (in ready, in free, out ready, out free)
    double *xfer_in, *xfer_out;
    cudaStream_t xfer_s[2];
    cudaEvent_t xfer_ev[4];
};

}  // namespace mhd

// --- error plumbing -------------------------------------------------------
int mhd_set_error(int status);

#define MHD_CUDA_TRY(expr)                                   \
    do {                                                     \
        cudaError_t e_ = (expr);                             \
        if (e_ != cudaSuccess) return mhd_set_error(MHDGPU_ERR_CUDA); \
    } while (0)

#define MHD_CHECK_LAUNCH() MHD_CUDA_TRY(cudaGetLastError())

// Bracket a launch with events when profiling is on; always count it.
void prof_begin(mhd::Ctx *c, int kclass, double bytes);
void prof_end(mhd::Ctx *c);

// kernels launched by api.cu, defined in the other translation units
namespace mhd {
const double *state_ptr(const Ctx *c);
int fused_settle_dev(Ctx *c);
int xsolve_setup(Ctx *c);
void xsolve_free(Ctx *c);
int launch_xsolve(Ctx *c, int op, int nv, const double *in, int in_start,
                  double *out, int src_kind);
int yspec_setup(Ctx *c);
void yspec_free(Ctx *c);
int launch_yspec(Ctx *c, int op, int nv, const double *in, int in_start,
                 double *out, int out_start);
int launch_efield(Ctx *c);
int launch_divb(Ctx *c, double *out);
int launch_rhs(Ctx *c);
int launch_rk(Ctx *c, int iRK);
int launch_calc_dt(Ctx *c, double dt0, double *dt_out);
int launch_calc_dt_dev(Ctx *c, int keep_dt);
int launch_max_divb(Ctx *c, double *out);
int launch_diagnostics(Ctx *c, double *energy, double *ch, long *nonfinite, long *nonpositive);
int xline_setup(Ctx *c);
void xline_free(Ctx *c);
int fused_setup(Ctx *c);
void fused_free(Ctx *c);
int fused_stage(Ctx *c, int iRK, int first_stage_of_run, int last_stage);
bool yrow_supported(const Ctx *c);
int xline_autotune(Ctx *c, int *w_out);
}  // namespace mhd
