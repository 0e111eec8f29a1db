// C ABI of the sm_100a hot path (include/mhd_gpu.h): context lifetime, the
// reference's operators on the context's arrays, and whole RK3 stages/steps.
#include <cuda_runtime.h>

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>

#include "common.cuh"

using mhd::Ctx;

static thread_local int g_last_error = MHDGPU_OK;

int mhd_set_error(int status)
{
    g_last_error = status;
    return status;
}

extern "C" int mhdgpu_last_error(void) { return g_last_error; }

extern "C" const char *mhdgpu_error_string(int s)
{
    switch (s) {
    case MHDGPU_OK: return "ok";
    case MHDGPU_ERR_INVALID: return "invalid argument";
    case MHDGPU_ERR_UNSUPPORTED: return "configuration not supported by the GPU path";
    case MHDGPU_ERR_CUDA: return "CUDA runtime error";
    case MHDGPU_ERR_NOMEM: return "device memory exhausted";
    case MHDGPU_ERR_TIMEOUT: return "bounded device wait ran out";
    case MHDGPU_ERR_NONFINITE: return "state is not finite or not positive";
    default: return "unknown status";
    }
}

// readInput (initialize.c:442-525): 15 lines, the first 16 characters of
// each converted with atoi/atof.
extern "C" int mhdgpu_read_input(const char *path, mhdgpu_params *o)
{
    if (!path || !o) return mhd_set_error(MHDGPU_ERR_INVALID);
    FILE *fp = fopen(path, "r");
    if (!fp) return mhd_set_error(MHDGPU_ERR_INVALID);
    char line[256], v[17];
    double d[15];
    for (int k = 0; k < 15; k++) {
        if (!fgets(line, sizeof line, fp)) {
            fclose(fp);
            return mhd_set_error(MHDGPU_ERR_INVALID);
        }
        memcpy(v, line, 16);
        v[16] = 0;
        d[k] = (k == 0 || k == 4 || k == 5 || k == 9 || k == 13 || k == 14) ? (double)atoi(v) : atof(v);
    }
    fclose(fp);
    o->boundaryTypeX = (int)d[0];
    o->cfl = d[1];
    o->Tmax = d[2];
    o->dtOut = d[3];
    o->nx = (long)d[4];
    o->ny = (long)d[5];
    o->Lx = d[6];
    o->Ly = d[7];
    o->adiabaticIdx = d[8];
    o->Hall = (int)d[9];
    o->di = d[10];
    o->resistivity = d[11];
    o->viscosity = d[12];
    o->divBcleaning = (int)d[13];
    o->outDivB = (int)d[14];
    return MHDGPU_OK;
}

static int fields_of(const Ctx *c, int which)
{
    const mhdgpu_params &p = c->p;
    switch (which) {
    case MHDGPU_UU: case MHDGPU_DUDX: case MHDGPU_DUDY: case MHDGPU_DUDT: case MHDGPU_DUDTRK:
        return c->nvar;
    case MHDGPU_D2UDX2: case MHDGPU_D2UDY2:
        return p.viscosity > 0 ? 3 : 0;
    case MHDGPU_D2BDX2: case MHDGPU_D2BDY2:
        return (p.resistivity > 0 || p.Hall == 1) ? 3 : 0;
    case MHDGPU_DIVB:
        return 1;
    case MHDGPU_DDIVBDX: case MHDGPU_DDIVBDY:
        return p.divBcleaning == 1 ? 1 : 0;
    case MHDGPU_EFIELD: case MHDGPU_DEDX: case MHDGPU_DEDY:
        return 3;
    default:
        return -1;
    }
}

// Stream capture and the calls that synchronize the device (cudaFree) or
// allocate must not interleave across threads: a device-wide synchronization
// during another thread's capture invalidates that capture.  Contexts served
// from several threads therefore take this lock around capture, creation and
// destruction (all short, host-side).
static std::mutex g_device_mu;

static void destroy_locked(mhdgpu_ctx *h);

extern "C" void mhdgpu_destroy(mhdgpu_ctx *h)
{
    std::lock_guard<std::mutex> lock(g_device_mu);
    destroy_locked(h);
}

// mhdgpu_destroy with g_device_mu held
static void destroy_locked(mhdgpu_ctx *h)
{
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            if (c->step_graph[i][j]) cudaGraphExecDestroy(c->step_graph[i][j]);
    mhd::fused_free(c);
    mhd::xsolve_free(c);
    mhd::yspec_free(c);
    for (int k = 0; k < MHDGPU_NARRAYS; k++) cudaFree(c->arr[k]);
    cudaFree(c->dscal);
    cudaFree(c->dred);
    cudaFree(c->dflag);
    if (c->prof_ev) {
        for (int i = 0; i < 2 * MHD_PROF_MAX; i++) cudaEventDestroy(c->prof_ev[i]);
        free(c->prof_ev);
        free(c->prof_cls);
    }
    cudaFree(c->xfer_in);
    cudaFree(c->xfer_out);
    for (int i = 0; i < 2; i++)
        if (c->xfer_s[i]) {
            cudaStreamSynchronize(c->xfer_s[i]);
            cudaStreamDestroy(c->xfer_s[i]);
        }
    for (int i = 0; i < 4; i++)
        if (c->xfer_ev[i]) cudaEventDestroy(c->xfer_ev[i]);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

static bool valid_params(const mhdgpu_params *p)
{
    if (!p) return false;
    if (p->nx < 8 || p->ny < 8 || p->ny > 8192 || (p->ny & (p->ny - 1)) != 0) return false;
    if (!(p->Lx > 0) || !(p->Ly > 0) || !(p->adiabaticIdx > 1)) return false;
    if (p->divBcleaning < 0 || p->divBcleaning > 2) return false;
    return true;
}

extern "C" int mhdgpu_create(const mhdgpu_params *p, int device, mhdgpu_ctx **out)
{
    std::lock_guard<std::mutex> lock(g_device_mu);
    if (!out) return mhd_set_error(MHDGPU_ERR_INVALID);
    *out = nullptr;
    if (!valid_params(p)) return mhd_set_error(MHDGPU_ERR_INVALID);
    // The open x boundary (boundaryTypeX = 1) is not on the GPU path; the
    // reference's own single-rank open boundary is inconsistent
    // (parallel.c:34-61 fills only one halo side).
    if (p->boundaryTypeX != 0) return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
    Ctx *c = new (std::nothrow) Ctx();
    if (!c) return mhd_set_error(MHDGPU_ERR_NOMEM);
    memset(c, 0, sizeof *c);
    c->p = *p;
    c->device = device;
    c->nvar = p->divBcleaning == 2 ? 9 : 8;  // initialize.c:207-214
    c->nx = p->nx;
    c->ny = p->ny;
    c->dx = p->Lx / (double)p->nx;            // initialize.c:125-135
    c->dy = p->Ly / (double)p->ny;
    double mx = c->dx > c->dy ? c->dx : c->dy;
    c->const_diff_divb = 2.0 * mx * mx;       // initialize.c:17, 154
    c->Ch = c->Cp = 0.0;
    int rc = MHDGPU_OK;
    auto fail = [&](int s) {
        destroy_locked(reinterpret_cast<mhdgpu_ctx *>(c));
        return mhd_set_error(s);
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(MHDGPU_ERR_CUDA);
    if (cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return fail(MHDGPU_ERR_CUDA);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(MHDGPU_ERR_CUDA);
    const size_t plane = (size_t)c->nx * c->ny;
    for (int k = 0; k < MHDGPU_NARRAYS; k++) {
        int nf = fields_of(c, k);
        c->arr_fields[k] = nf;
        if (nf > 0) {
            if (cudaMalloc(&c->arr[k], sizeof(double) * plane * nf) != cudaSuccess)
                return fail(MHDGPU_ERR_NOMEM);
            if (cudaMemset(c->arr[k], 0, sizeof(double) * plane * nf) != cudaSuccess)
                return fail(MHDGPU_ERR_CUDA);
        }
    }
    c->nred = 8192;
    if (cudaMalloc(&c->dscal, sizeof(double) * 16) != cudaSuccess) return fail(MHDGPU_ERR_NOMEM);
    if (cudaMalloc(&c->dred, sizeof(double) * c->nred) != cudaSuccess) return fail(MHDGPU_ERR_NOMEM);
    if (cudaMalloc(&c->dflag, sizeof(int) * 4) != cudaSuccess) return fail(MHDGPU_ERR_NOMEM);
    cudaMemset(c->dscal, 0, sizeof(double) * 16);
    cudaMemset(c->dflag, 0, sizeof(int) * 4);
    if ((rc = mhd::xsolve_setup(c)) != MHDGPU_OK) return fail(rc);
    if ((rc = mhd::yspec_setup(c)) != MHDGPU_OK) return fail(rc);
    if ((rc = mhd::fused_setup(c)) != MHDGPU_OK) return fail(rc);
    // set-up work is on this context's stream and the legacy stream; other
    // contexts' streams keep running
    if (cudaStreamSynchronize(c->stream) != cudaSuccess ||
        cudaStreamSynchronize(cudaStreamLegacy) != cudaSuccess)
        return fail(MHDGPU_ERR_CUDA);
    *out = reinterpret_cast<mhdgpu_ctx *>(c);
    return MHDGPU_OK;
}

extern "C" int mhdgpu_nvar(const mhdgpu_ctx *h)
{
    return h ? reinterpret_cast<const Ctx *>(h)->nvar : -1;
}

#define CTX_OR_FAIL(h)                                          \
    Ctx *c = reinterpret_cast<Ctx *>(h);                        \
    if (!c) return mhd_set_error(MHDGPU_ERR_INVALID);           \
    if (cudaSetDevice(c->device) != cudaSuccess) return mhd_set_error(MHDGPU_ERR_CUDA)

namespace mhd {
int fused_apply_pending_filter(Ctx *c);
}

// Apply the x filter that the fused stage leaves pending (and bring a state
// settled into the x filter's copy back to uu), so that every public entry
// point sees the same state as the reference would hold.
static int settle(Ctx *c)
{
    return (c->fused_pending_filter || c->state_in_S) ? mhd::fused_apply_pending_filter(c)
                                                      : MHDGPU_OK;
}

extern "C" double *mhdgpu_device_array(mhdgpu_ctx *h, int which)
{
    Ctx *c = reinterpret_cast<Ctx *>(h);
    if (!c || which < 0 || which >= MHDGPU_NARRAYS) return nullptr;
    return c->arr[which];
}

extern "C" int mhdgpu_set_array(mhdgpu_ctx *h, int which, const double *host)
{
    CTX_OR_FAIL(h);
    if (which < 0 || which >= MHDGPU_NARRAYS || !host || !c->arr[which])
        return mhd_set_error(MHDGPU_ERR_INVALID);
    size_t n = (size_t)c->arr_fields[which] * c->nx * c->ny;
    MHD_CUDA_TRY(cudaMemcpyAsync(c->arr[which], host, n * sizeof(double), cudaMemcpyHostToDevice,
                                 c->stream));
    MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (which == MHDGPU_UU) {
        c->fused_pending_filter = 0;
        c->state_in_S = 0;
    }
    return MHDGPU_OK;
}

extern "C" int mhdgpu_get_array(mhdgpu_ctx *h, int which, double *host)
{
    CTX_OR_FAIL(h);
    if (which == MHDGPU_UU && settle(c)) return mhdgpu_last_error();
    if (which < 0 || which >= MHDGPU_NARRAYS || !host || !c->arr[which])
        return mhd_set_error(MHDGPU_ERR_INVALID);
    size_t n = (size_t)c->arr_fields[which] * c->nx * c->ny;
    MHD_CUDA_TRY(cudaMemcpyAsync(host, c->arr[which], n * sizeof(double), cudaMemcpyDeviceToHost,
                                 c->stream));
    MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return MHDGPU_OK;
}

int mhd_check_flag(Ctx *c);
static int check_flag(Ctx *c) { return mhd_check_flag(c); }

// status flag of the context's kernels: read, report and clear
int mhd_check_flag(Ctx *c)
{
    int f = 0;
    MHD_CUDA_TRY(cudaMemcpyAsync(&f, c->dflag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (f != 0) {
        cudaMemsetAsync(c->dflag, 0, sizeof(int), c->stream);
        return mhd_set_error(f);
    }
    return MHDGPU_OK;
}

extern "C" int mhdgpu_synchronize(mhdgpu_ctx *h)
{
    CTX_OR_FAIL(h);
    if (settle(c)) return mhdgpu_last_error();
    MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return check_flag(c);
}

// ---------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------
static bool arr_ok(const Ctx *c, int which, int first, int nv)
{
    return which >= 0 && which < MHDGPU_NARRAYS && c->arr[which] && first >= 0 &&
           first + nv <= c->arr_fields[which];
}

extern "C" int mhdgpu_deriv_x(mhdgpu_ctx *h, int nv, int in, int start, int out, int order)
{
    CTX_OR_FAIL(h);
    if (settle(c)) return mhdgpu_last_error();
    if (order != 1 && order != 2) return mhd_set_error(MHDGPU_ERR_INVALID);
    if (!arr_ok(c, in, start, nv) || !arr_ok(c, out, 0, nv)) return mhd_set_error(MHDGPU_ERR_INVALID);
    return mhd::launch_xsolve(c, order == 1 ? mhd::XOP_D1 : mhd::XOP_D2, nv, c->arr[in], start,
                              c->arr[out], 0);
}

extern "C" int mhdgpu_deriv_y(mhdgpu_ctx *h, int nv, int in, int start, int out, int order)
{
    CTX_OR_FAIL(h);
    if (settle(c)) return mhdgpu_last_error();
    if (order != 1 && order != 2) return mhd_set_error(MHDGPU_ERR_INVALID);
    if (!arr_ok(c, in, start, nv) || !arr_ok(c, out, 0, nv)) return mhd_set_error(MHDGPU_ERR_INVALID);
    return mhd::launch_yspec(c, order - 1, nv, c->arr[in], start, c->arr[out], 0);
}

extern "C" int mhdgpu_calc_efield(mhdgpu_ctx *h)
{
    CTX_OR_FAIL(h);
    if (settle(c)) return mhdgpu_last_error();
    return mhd::launch_efield(c);
}

extern "C" int mhdgpu_calc_divb(mhdgpu_ctx *h)
{
    CTX_OR_FAIL(h);
    return mhd::launch_divb(c, c->arr[MHDGPU_DIVB]);
}

extern "C" int mhdgpu_calc_rhs(mhdgpu_ctx *h)
{
    CTX_OR_FAIL(h);
    if (settle(c)) return mhdgpu_last_error();
    return mhd::launch_rhs(c);
}

// rkInit (timeAdvance.c:20-27): stage coefficients and dudtRK = 0
extern "C" int mhdgpu_rk_init(mhdgpu_ctx *h, double dt)
{
    CTX_OR_FAIL(h);
    c->dt = dt;
    c->cc[0] = 8.0 / 15.0 * dt;
    c->dd[0] = 0.0;
    c->cc[1] = 5.0 / 12.0 * dt;
    c->dd[1] = -17. / 60. * dt;
    c->cc[2] = 0.75 * dt;
    c->dd[2] = -5. / 12. * dt;
    MHD_CUDA_TRY(cudaMemsetAsync(c->arr[MHDGPU_DUDTRK], 0,
                                 sizeof(double) * c->nvar * c->nx * c->ny, c->stream));
    return MHDGPU_OK;
}

extern "C" int mhdgpu_rk_execute(mhdgpu_ctx *h, int iRK)
{
    CTX_OR_FAIL(h);
    if (settle(c)) return mhdgpu_last_error();
    if (iRK < 0 || iRK > 2) return mhd_set_error(MHDGPU_ERR_INVALID);
    return mhd::launch_rk(c, iRK);
}

// filtering (filtering.c:98-102): x filter of all NVAR fields, then y filter,
// both in place on uu
extern "C" int mhdgpu_filtering(mhdgpu_ctx *h)
{
    CTX_OR_FAIL(h);
    if (settle(c)) return mhdgpu_last_error();
    int rc = mhd::launch_xsolve(c, mhd::XOP_F, c->nvar, c->arr[MHDGPU_UU], 0, c->arr[MHDGPU_UU], 0);
    if (rc) return rc;
    return mhd::launch_yspec(c, 2, c->nvar, c->arr[MHDGPU_UU], 0, c->arr[MHDGPU_UU], 0);
}

extern "C" int mhdgpu_calc_dt(mhdgpu_ctx *h, double dt0, double *dt_out)
{
    CTX_OR_FAIL(h);
    if (settle(c)) return mhdgpu_last_error();
    return mhd::launch_calc_dt(c, dt0, dt_out);
}

extern "C" int mhdgpu_check_divb(mhdgpu_ctx *h, double *maxdivb)
{
    CTX_OR_FAIL(h);
    if (!maxdivb) return mhd_set_error(MHDGPU_ERR_INVALID);
    if (c->deriv_fp32) return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);  // FP32 scratch
    return mhd::launch_max_divb(c, maxdivb);
}

extern "C" int mhdgpu_get_cleaning_speeds(mhdgpu_ctx *h, double *Ch, double *Cp)
{
    CTX_OR_FAIL(h);
    if (Ch) *Ch = c->Ch;
    if (Cp) *Cp = c->Cp;
    return MHDGPU_OK;
}

// ---------------------------------------------------------------------------
// stages and steps
// ---------------------------------------------------------------------------
#define TRY(x)                  \
    do {                        \
        int r_ = (x);           \
        if (r_) return r_;      \
    } while (0)

// One RK3 stage with the reference's call order (mhd.c:154-199); the halo
// exchanges are index wrap-around inside the x kernels.
extern "C" int mhdgpu_stage(mhdgpu_ctx *h, int iRK)
{
    CTX_OR_FAIL(h);
    if (iRK < 0 || iRK > 2) return mhd_set_error(MHDGPU_ERR_INVALID);
    TRY(settle(c));
    const mhdgpu_params &p = c->p;
    TRY(mhdgpu_deriv_x(h, c->nvar, MHDGPU_UU, 0, MHDGPU_DUDX, 1));
    TRY(mhdgpu_deriv_y(h, c->nvar, MHDGPU_UU, 0, MHDGPU_DUDY, 1));
    if (p.viscosity > 0) {
        TRY(mhdgpu_deriv_x(h, 3, MHDGPU_UU, 1, MHDGPU_D2UDX2, 2));
        TRY(mhdgpu_deriv_y(h, 3, MHDGPU_UU, 1, MHDGPU_D2UDY2, 2));
    }
    if (p.Hall == 1 || p.resistivity > 0) {
        TRY(mhdgpu_deriv_x(h, 3, MHDGPU_UU, 4, MHDGPU_D2BDX2, 2));
        TRY(mhdgpu_deriv_y(h, 3, MHDGPU_UU, 4, MHDGPU_D2BDY2, 2));
    }
    if (p.divBcleaning == 1) {
        TRY(mhdgpu_calc_divb(h));
        TRY(mhdgpu_deriv_x(h, 1, MHDGPU_DIVB, 0, MHDGPU_DDIVBDX, 1));
        TRY(mhdgpu_deriv_y(h, 1, MHDGPU_DIVB, 0, MHDGPU_DDIVBDY, 1));
    }
    TRY(mhdgpu_calc_efield(h));
    TRY(mhdgpu_deriv_x(h, 3, MHDGPU_EFIELD, 0, MHDGPU_DEDX, 1));
    TRY(mhdgpu_deriv_y(h, 3, MHDGPU_EFIELD, 0, MHDGPU_DEDY, 1));
    TRY(mhdgpu_calc_rhs(h));
    TRY(mhdgpu_rk_execute(h, iRK));
    TRY(mhdgpu_filtering(h));
    return MHDGPU_OK;
}

// dt before the first step or after a step: fixed dt (with calcDt still run
// for Ch/Cp under hyperbolic cleaning) or the reference's CFL control
static int next_dt(mhdgpu_ctx *h, Ctx *c, double dt_fixed, double *dt)
{
    if (dt_fixed > 0) {
        if (c->p.divBcleaning == 2) TRY(mhd::launch_calc_dt(c, dt_fixed, nullptr));
        *dt = dt_fixed;
        return MHDGPU_OK;
    }
    return mhd::launch_calc_dt(c, *dt, dt);
}

extern "C" int mhdgpu_steps(mhdgpu_ctx *h, int nsteps, double dt_fixed, double *dt_io)
{
    CTX_OR_FAIL(h);
    if (nsteps < 0) return mhd_set_error(MHDGPU_ERR_INVALID);
    if (nsteps > 0) c->deriv_fp32 = 0;  // every stage rewrites the derivatives in FP64
    TRY(settle(c));
    double dt = dt_io ? *dt_io : 0.0;
    TRY(next_dt(h, c, dt_fixed, &dt));
    TRY(mhdgpu_rk_init(h, dt));
    for (int s = 0; s < nsteps; s++) {
        for (int k = 0; k < 3; k++) TRY(mhdgpu_stage(h, k));
        TRY(next_dt(h, c, dt_fixed, &dt));
        TRY(mhdgpu_rk_init(h, dt));
    }
    if (dt_io) *dt_io = dt;
    MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return check_flag(c);
}

// One fused RK3 step under device step control: the three fused stages and,
// with CFL control or hyperbolic cleaning, the x filter they leave pending
// and calcDt for the next step, all on the device.
static int fused_step_dev(Ctx *c, bool need_dt, bool keep_dt)
{
    for (int k = 0; k < 3; k++) TRY(mhd::fused_stage(c, k, 0, k == 2));
    if (need_dt) {
        TRY(mhd::fused_settle_dev(c));
        TRY(mhd::launch_calc_dt_dev(c, keep_dt));
    }
    return MHDGPU_OK;
}

// Steps through the fused stage (fused.cu).  Grids the fused x pass cannot
// tile (an odd nx with 8 columns), and diffusive cleaning (divBcleaning == 1)
// where the y row kernel does not apply, run through the operator stage.
//
// With the row kernel (16 <= ny <= 8192) the step control stays on the
// device: dt (and Ch, Cp) live in dscal, the y pass forms cc = c_k dt and
// dd = d_k dt there, calcDt runs on the device (the reference's arithmetic
// and hysteresis, timeAdvance.c:38-153), and dudtRK needs no clearing between
// steps (the first stage neither reads it nor needs it zero).  A step whose
// entry state is the steady one (CFL: filter settled; fixed dt: filter
// pending) is captured once per context, precision and dt mode as a CUDA graph
// and replayed; the host waits only at the end.  Profiling runs the same
// launches without the graph.
extern "C" int mhdgpu_steps_fused(mhdgpu_ctx *h, int nsteps, double dt_fixed, double *dt_io)
{
    CTX_OR_FAIL(h);
    if (nsteps < 0) return mhd_set_error(MHDGPU_ERR_INVALID);
    if (c->mixed && (c->p.divBcleaning == 1 || c->xf_W == 0 || !mhd::yrow_supported(c)))
        return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
    if (c->xf_W == 0 || (c->p.divBcleaning == 1 && !mhd::yrow_supported(c)))
        return mhdgpu_steps(h, nsteps, dt_fixed, dt_io);
    if (nsteps > 0) c->deriv_fp32 = c->mixed;
    const bool need_dt = dt_fixed <= 0 || c->p.divBcleaning == 2;
    double dt = dt_io ? *dt_io : 0.0;
    if (!mhd::yrow_supported(c)) {  // host step control (operator y sequence)
        if (need_dt) TRY(settle(c));
        TRY(next_dt(h, c, dt_fixed, &dt));
        TRY(mhdgpu_rk_init(h, dt));
        for (int s = 0; s < nsteps; s++) {
            for (int k = 0; k < 3; k++) TRY(mhd::fused_stage(c, k, s == 0 && k == 0, k == 2));
            if (need_dt) TRY(settle(c));
            TRY(next_dt(h, c, dt_fixed, &dt));
            TRY(mhdgpu_rk_init(h, dt));
        }
        TRY(settle(c));
        if (dt_io) *dt_io = dt;
        MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
        return check_flag(c);
    }

    // device step control
    const bool fixed = dt_fixed > 0;
    const double dt0 = fixed ? dt_fixed : dt;
    MHD_CUDA_TRY(cudaMemcpyAsync(c->dscal, &dt0, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (need_dt) {
        TRY(mhd::fused_settle_dev(c));
        TRY(mhd::launch_calc_dt_dev(c, fixed));
    }
    c->dev_dt = 1;
    const int gm = c->mixed ? 1 : 0, gd = fixed ? 1 : 0;
    int rc = MHDGPU_OK;
    for (int s = 0; s < nsteps && rc == MHDGPU_OK; s++) {
        // the steady entry state: filter settled with CFL control, pending otherwise
        const bool steady = need_dt ? !c->fused_pending_filter : c->fused_pending_filter != 0;
        if (!steady || c->prof_on || s == 0) {
            rc = fused_step_dev(c, need_dt, fixed);
            continue;
        }
        if (!c->step_graph[gm][gd]) {
            std::lock_guard<std::mutex> lock(g_device_mu);
            const long l0 = c->launches;
            cudaGraph_t g = nullptr;
            if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                rc = mhd_set_error(MHDGPU_ERR_CUDA);
                break;
            }
            const int rs = fused_step_dev(c, need_dt, fixed);
            const cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
            if (rs || ec != cudaSuccess ||
                cudaGraphInstantiate(&c->step_graph[gm][gd], g, 0) != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                c->step_graph[gm][gd] = nullptr;
                rc = rs ? rs : mhd_set_error(MHDGPU_ERR_CUDA);
                break;
            }
            cudaGraphDestroy(g);
            c->step_graph_launches[gm][gd] = c->launches - l0;
            c->launches = l0;  // captured, not yet run
        }
        if (cudaGraphLaunch(c->step_graph[gm][gd], c->stream) != cudaSuccess) {
            rc = mhd_set_error(MHDGPU_ERR_CUDA);
            break;
        }
        c->launches += c->step_graph_launches[gm][gd];
    }
    c->dev_dt = 0;
    TRY(rc);
    TRY(settle(c));
    double hs[3];
    MHD_CUDA_TRY(cudaMemcpyAsync(hs, c->dscal, sizeof hs, cudaMemcpyDeviceToHost, c->stream));
    MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (!fixed) dt = hs[0];
    else dt = dt_fixed;
    if (c->p.divBcleaning == 2) {
        c->Ch = hs[1];
        c->Cp = hs[2];
    }
    TRY(mhdgpu_rk_init(h, dt));  // the host coefficients and dudtRK = 0, as rkInit leaves them
    if (dt_io) *dt_io = dt;
    MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return check_flag(c);
}

extern "C" int mhdgpu_autotune(mhdgpu_ctx *h, int *columns_out)
{
    CTX_OR_FAIL(h);
    if (settle(c)) return mhdgpu_last_error();
    if (c->xn_on) {  // the chunked x pass: no tile width to choose
        if (columns_out) *columns_out = 0;
        return MHDGPU_OK;
    }
    TRY(mhd::xline_autotune(c, columns_out));
    // the captured steps hold the previous tiling
    std::lock_guard<std::mutex> lock(g_device_mu);
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            if (c->step_graph[i][j]) {
                cudaGraphExecDestroy(c->step_graph[i][j]);
                c->step_graph[i][j] = nullptr;
            }
    MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return check_flag(c);
}

// A stream of independent states through the fused steps (no counterpart
// in the reference, whose driver advances one state): state r is uploaded
// from h_in[r], advanced by nsteps steps exactly as mhdgpu_steps_fused
// advances a state set with mhdgpu_set_array, and downloaded to h_out[r].
// The upload of state r+1 (into a device staging copy, on its own stream)
// and the download of state r-1 (from a second staging copy, on a third
// stream) run while state r steps; with page-locked host buffers the
// transfers and the steps overlap.
extern "C" int mhdgpu_steps_fused_stream(mhdgpu_ctx *h, int nstates, const double *const *h_in,
                                         double *const *h_out, int nsteps, double dt_fixed,
                                         double *dt_io)
{
    CTX_OR_FAIL(h);
    if (nstates < 0 || nsteps < 0 || (nstates > 0 && (!h_in || !h_out)))
        return mhd_set_error(MHDGPU_ERR_INVALID);
    for (int r = 0; r < nstates; r++)
        if (!h_in[r] || !h_out[r]) return mhd_set_error(MHDGPU_ERR_INVALID);
    if (nstates == 0) return MHDGPU_OK;
    const size_t bytes = sizeof(double) * c->nvar * c->nx * c->ny;
    if (!c->xfer_in) {
        MHD_CUDA_TRY(cudaMalloc(&c->xfer_in, bytes));
        MHD_CUDA_TRY(cudaMalloc(&c->xfer_out, bytes));
        for (int i = 0; i < 2; i++)
            MHD_CUDA_TRY(cudaStreamCreateWithFlags(&c->xfer_s[i], cudaStreamNonBlocking));
        for (int i = 0; i < 4; i++)
            MHD_CUDA_TRY(cudaEventCreateWithFlags(&c->xfer_ev[i], cudaEventDisableTiming));
    }
    cudaStream_t sin = c->xfer_s[0], sout = c->xfer_s[1];
    cudaEvent_t in_ready = c->xfer_ev[0], in_free = c->xfer_ev[1];
    cudaEvent_t out_ready = c->xfer_ev[2], out_free = c->xfer_ev[3];
    double *uu = c->arr[MHDGPU_UU];
    const double dt0 = dt_io ? *dt_io : 0.0;
    double dt = dt0;
    // the copies and steps; every error path leaves through the
    // synchronisation below, so no copy of the caller's buffers is in flight
    // when the call returns
    auto run = [&]() -> int {
        MHD_CUDA_TRY(cudaMemcpyAsync(c->xfer_in, h_in[0], bytes, cudaMemcpyHostToDevice, sin));
        MHD_CUDA_TRY(cudaEventRecord(in_ready, sin));
        for (int r = 0; r < nstates; r++) {
            MHD_CUDA_TRY(cudaStreamWaitEvent(c->stream, in_ready, 0));
            MHD_CUDA_TRY(cudaMemcpyAsync(uu, c->xfer_in, bytes, cudaMemcpyDeviceToDevice, c->stream));
            MHD_CUDA_TRY(cudaEventRecord(in_free, c->stream));
            c->fused_pending_filter = 0;  // as mhdgpu_set_array(UU)
            c->state_in_S = 0;
            if (r + 1 < nstates) {
                MHD_CUDA_TRY(cudaStreamWaitEvent(sin, in_free, 0));
                MHD_CUDA_TRY(cudaMemcpyAsync(c->xfer_in, h_in[r + 1], bytes, cudaMemcpyHostToDevice, sin));
                MHD_CUDA_TRY(cudaEventRecord(in_ready, sin));
            }
            double d = dt0;
            const int rs = mhdgpu_steps_fused(h, nsteps, dt_fixed, &d);
            if (rs != MHDGPU_OK) return rs;
            dt = d;
            // the previous state's download has left the outgoing copy
            if (r > 0) MHD_CUDA_TRY(cudaStreamWaitEvent(c->stream, out_free, 0));
            MHD_CUDA_TRY(cudaMemcpyAsync(c->xfer_out, uu, bytes, cudaMemcpyDeviceToDevice, c->stream));
            MHD_CUDA_TRY(cudaEventRecord(out_ready, c->stream));
            MHD_CUDA_TRY(cudaStreamWaitEvent(sout, out_ready, 0));
            MHD_CUDA_TRY(cudaMemcpyAsync(h_out[r], c->xfer_out, bytes, cudaMemcpyDeviceToHost, sout));
            MHD_CUDA_TRY(cudaEventRecord(out_free, sout));
        }
        return MHDGPU_OK;
    };
    const int rc = run();
    // no copy of this call is left in flight, also after an error
    const cudaError_t e0 = cudaStreamSynchronize(sin), e1 = cudaStreamSynchronize(sout);
    if (rc != MHDGPU_OK) return rc;
    if (e0 != cudaSuccess || e1 != cudaSuccess) return mhd_set_error(MHDGPU_ERR_CUDA);
    if (dt_io) *dt_io = dt;
    return MHDGPU_OK;
}

extern "C" int mhdgpu_set_precision(mhdgpu_ctx *h, int precision)
{
    CTX_OR_FAIL(h);
    if (precision != MHDGPU_PRECISION_FP64 && precision != MHDGPU_PRECISION_MIXED)
        return mhd_set_error(MHDGPU_ERR_INVALID);
    if (precision == MHDGPU_PRECISION_MIXED &&
        (c->p.divBcleaning == 1 || c->xf_W == 0 || !mhd::yrow_supported(c)))
        return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
    c->mixed = precision == MHDGPU_PRECISION_MIXED;
    return MHDGPU_OK;
}

extern "C" int mhdgpu_diagnostics(mhdgpu_ctx *h, double *energy, double *cross_helicity, int *finite)
{
    CTX_OR_FAIL(h);
    if (settle(c)) return mhdgpu_last_error();
    long bad = 0;
    TRY(mhd::launch_diagnostics(c, energy, cross_helicity, &bad, nullptr));
    if (finite) *finite = bad == 0;
    return MHDGPU_OK;
}

extern "C" int mhdgpu_state_cells(mhdgpu_ctx *h, long *nonfinite, long *nonpositive)
{
    CTX_OR_FAIL(h);
    if (settle(c)) return mhdgpu_last_error();
    return mhd::launch_diagnostics(c, nullptr, nullptr, nonfinite, nonpositive);
}

// ---------------------------------------------------------------------------
// instrumentation
// ---------------------------------------------------------------------------
void prof_begin(Ctx *c, int kclass, double bytes)
{
    c->launches++;
    if (!c->prof_on || c->prof_n >= MHD_PROF_MAX) return;
    c->prof_bytes[kclass] += bytes;
    c->prof_cls[c->prof_n] = kclass;
    cudaEventRecord(c->prof_ev[2 * c->prof_n], c->stream);
}

void prof_end(Ctx *c)
{
    if (!c->prof_on || c->prof_n >= MHD_PROF_MAX) return;
    cudaEventRecord(c->prof_ev[2 * c->prof_n + 1], c->stream);
    c->prof_n++;
}

extern "C" void *mhdgpu_stream(mhdgpu_ctx *h)
{
    Ctx *c = reinterpret_cast<Ctx *>(h);
    return c ? (void *)c->stream : nullptr;
}

extern "C" long mhdgpu_launch_count(const mhdgpu_ctx *h)
{
    const Ctx *c = reinterpret_cast<const Ctx *>(h);
    return c ? c->launches : -1;
}

extern "C" int mhdgpu_profile(mhdgpu_ctx *h, int enable)
{
    CTX_OR_FAIL(h);
    if (enable && !c->prof_ev) {
        c->prof_ev = (cudaEvent_t *)calloc(2 * MHD_PROF_MAX, sizeof(cudaEvent_t));
        c->prof_cls = (int *)calloc(MHD_PROF_MAX, sizeof(int));
        if (!c->prof_ev || !c->prof_cls) return mhd_set_error(MHDGPU_ERR_NOMEM);
        for (int i = 0; i < 2 * MHD_PROF_MAX; i++)
            MHD_CUDA_TRY(cudaEventCreate(&c->prof_ev[i]));
    }
    c->prof_on = enable ? 1 : 0;
    if (enable) {
        c->prof_n = 0;
        for (int k = 0; k < 8; k++) c->prof_bytes[k] = 0.0;
    }
    return MHDGPU_OK;
}

extern "C" int mhdgpu_profile_read(mhdgpu_ctx *h, int kclass, double *total_ms, long *count,
                                   double *bytes)
{
    CTX_OR_FAIL(h);
    MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    double tot = 0.0;
    long n = 0;
    for (int i = 0; i < c->prof_n; i++) {
        if (c->prof_cls[i] != kclass) continue;
        float ms = 0.f;
        MHD_CUDA_TRY(cudaEventElapsedTime(&ms, c->prof_ev[2 * i], c->prof_ev[2 * i + 1]));
        tot += ms;
        n++;
    }
    if (total_ms) *total_ms = tot;
    if (count) *count = n;
    if (bytes) *bytes = (kclass >= 0 && kclass < 8) ? c->prof_bytes[kclass] : 0.0;
    return MHDGPU_OK;
}
