// Fused RK3 stage: the reference's stage (mhd.c:154-199) regrouped into an x
// pass and a y pass.
//
// The x filter and the y filter act on different axes and commute, so the
// stage's closing filter F_y(F_x(u)) is applied as F_x(F_y(u)): the y filter
// closes the y pass of stage k, and the x filter opens the x pass of stage
// k+1, which reads each x-line once to filter it and differentiate the
// filtered line.  The state in HBM between two stages therefore lacks its x
// filter ("pending"); it is applied before anything outside the stage looks
// at the state (the end of a run, a CFL time step, a host read).
//
//   x pass:  per field, F_x (if pending) -> write state -> d/dx, d2/dx2
//            (xline.cu); then d/dx of Ey, Ez with E computed from the state.
//   y pass:  d/dy, d2/dy2, E, calcRHS, rkExecute, F_y (yrow.cu; with
//            diffusive cleaning split around calcDivB and the divB
//            derivatives; for rows the row kernel does not take, the
//            operator kernels in the same order).
#include <cstring>

#include "common.cuh"
#include "xcore.cuh"
#include "xfir.cuh"

namespace mhd {

bool yrow_supported(const Ctx *c);
int launch_yrow(Ctx *c, int iRK, int last_stage, int mode);

int fused_setup(Ctx *c)
{
    int rc = xline_setup(c);
    if (rc) return rc;
    return yrow_supported(c) ? xn_setup(c) : MHDGPU_OK;
}

void fused_free(Ctx *c)
{
    xline_free(c);
    xn_free(c);
}

static double planeb(const Ctx *c) { return (double)c->nx * c->ny * 8.0; }

// Where the current state is: the x-filtered copy the chunked x filter
// wrote, or the context's uu.
const double *state_ptr(const Ctx *c) { return c->state_in_S ? c->xn_state : c->arr[MHDGPU_UU]; }

// x pass of a stage: one launch for all fields and the electric field, or,
// on long lines, the chunked x filter into the state copy and the chunked
// derivatives of that copy (xfir.cu)
static int fused_x_pass(Ctx *c)
{
    if (c->xn_on) {
        if (c->fused_pending_filter) {
            int rc = launch_xf(c, c->arr[MHDGPU_UU], c->xn_state);
            if (rc) return rc;
            c->fused_pending_filter = 0;
            c->state_in_S = 1;
        }
        return launch_xd(c, state_ptr(c));
    }
    const mhdgpu_params &p = c->p;
    XFArgs a;
    std::memset(&a, 0, sizeof a);
    a.in = c->arr[MHDGPU_UU];
    a.in_start = 0;
    a.nfields = c->nvar;
    a.fout = c->fused_pending_filter ? c->arr[MHDGPU_UU] : nullptr;
    a.out1 = c->arr[MHDGPU_DUDX];
    a.out2a = p.viscosity > 0 ? c->arr[MHDGPU_D2UDX2] : nullptr;
    a.d2a_lo = UX;
    a.out2b = (p.resistivity > 0 || p.Hall == 1) ? c->arr[MHDGPU_D2BDX2] : nullptr;
    a.d2b_lo = BX;
    a.single_op = -1;
    // dEdx[1], dEdx[2]: one plane into the array, in the stored element type
    const size_t plane = (size_t)c->nx * c->ny;
    a.outE = c->mixed ? reinterpret_cast<double *>(reinterpret_cast<float *>(c->arr[MHDGPU_DEDX]) + plane)
                      : c->arr[MHDGPU_DEDX] + plane;
    int n2 = (a.out2a ? 3 : 0) + (a.out2b ? 3 : 0);
    double bytes = planeb(c) * (c->nvar + (a.fout ? c->nvar : 0) + c->nvar + n2 + 2);
    return launch_xline(c, a, bytes);
}

// y pass of a stage
static int fused_y_pass(Ctx *c, int iRK)
{
    const mhdgpu_params &p = c->p;
    double *uu = c->arr[MHDGPU_UU];
    int rc;
    if ((rc = launch_yspec(c, 0, c->nvar, uu, 0, c->arr[MHDGPU_DUDY], 0))) return rc;
    if (p.viscosity > 0 && (rc = launch_yspec(c, 1, 3, uu, UX, c->arr[MHDGPU_D2UDY2], 0))) return rc;
    if ((p.resistivity > 0 || p.Hall == 1) &&
        (rc = launch_yspec(c, 1, 3, uu, BX, c->arr[MHDGPU_D2BDY2], 0)))
        return rc;
    if ((rc = launch_efield(c))) return rc;
    if ((rc = launch_yspec(c, 0, 3, c->arr[MHDGPU_EFIELD], 0, c->arr[MHDGPU_DEDY], 0))) return rc;
    if ((rc = launch_rhs(c))) return rc;
    if ((rc = launch_rk(c, iRK))) return rc;
    return launch_yspec(c, 2, c->nvar, uu, 0, uu, 0);
}

// The x pass of a stage with no pending filter, for timing: it reads the
// state and writes only the x-derivative arrays.
int fused_x_timing_pass(Ctx *c)
{
    const int pending = c->fused_pending_filter;
    c->fused_pending_filter = 0;
    const int rc = fused_x_pass(c);
    c->fused_pending_filter = pending;
    return rc;
}

int fused_apply_pending_filter(Ctx *c);

// The pending x filter applied where the next device step reads the state
// (calcDt, the first stage): with the chunked x pass into the state copy,
// else in place.
int fused_settle_dev(Ctx *c)
{
    if (!c->xn_on) return fused_apply_pending_filter(c);
    if (!c->fused_pending_filter) return MHDGPU_OK;
    int rc = launch_xf(c, c->arr[MHDGPU_UU], c->xn_state);
    if (rc) return rc;
    c->fused_pending_filter = 0;
    c->state_in_S = 1;
    return MHDGPU_OK;
}

// The state filtered and in uu, as every entry point outside the fused steps
// expects it.
int fused_apply_pending_filter(Ctx *c)
{
    if (c->xn_on) {
        int rc = fused_settle_dev(c);
        if (rc) return rc;
        if (c->state_in_S) {
            MHD_CUDA_TRY(cudaMemcpyAsync(c->arr[MHDGPU_UU], c->xn_state,
                                         sizeof(double) * c->nvar * c->nx * c->ny,
                                         cudaMemcpyDeviceToDevice, c->stream));
            c->state_in_S = 0;
        }
        return MHDGPU_OK;
    }
    if (!c->fused_pending_filter) return MHDGPU_OK;
    XFArgs a;
    std::memset(&a, 0, sizeof a);
    a.in = c->arr[MHDGPU_UU];
    a.nfields = c->nvar;
    a.single_op = XOP_F;
    a.out1 = c->arr[MHDGPU_UU];
    int rc = launch_xline(c, a, planeb(c) * 2 * c->nvar);
    if (rc) return rc;
    c->fused_pending_filter = 0;
    return MHDGPU_OK;
}

int fused_stage(Ctx *c, int iRK, int first, int last)
{
    (void)first;
    int rc = fused_x_pass(c);
    if (rc) return rc;
    if (c->p.divBcleaning == 1 && yrow_supported(c)) {
        // diffusive cleaning (mhd.c:175-182): divB needs both passes'
        // derivatives, and its own derivatives the whole lines: the y pass
        // splits around calcDivB and the two operator derivatives of divB
        double *divb = c->arr[MHDGPU_DIVB];
        if ((rc = launch_yrow(c, iRK, last, 1))) return rc;
        if ((rc = launch_divb(c, divb))) return rc;
        if ((rc = launch_xsolve(c, XOP_D1, 1, divb, 0, c->arr[MHDGPU_DDIVBDX], 0))) return rc;
        if ((rc = launch_yspec(c, 0, 1, divb, 0, c->arr[MHDGPU_DDIVBDY], 0))) return rc;
        rc = launch_yrow(c, iRK, last, 2);
    } else {
        rc = yrow_supported(c) ? launch_yrow(c, iRK, last, 0) : fused_y_pass(c, iRK);
    }
    if (rc) return rc;
    c->fused_pending_filter = 1;
    c->state_in_S = 0;  // the y pass wrote the new state to uu
    return MHDGPU_OK;
}

}  // namespace mhd
