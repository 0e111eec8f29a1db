// Pointwise operators and reductions of the hot path:
//   calcEfield (calcRHS.c:24-43), calcDivB (calcRHS.c:13-22),
//   calcRHSInnerPoint + addSourceTerm (calcRHS.c:77-161, 498-544),
//   rkExecute (timeAdvance.c:29-36), calcDt (timeAdvance.c:38-153),
//   checkDivB (mhd.c:342-367) and the energy / cross-helicity diagnostics.
// All are HBM-streaming kernels over the [field][nx][ny] planes; the
// reductions write one partial per block and finish in a second, single-block
// pass in a fixed order, so their results do not depend on scheduling.
#include <cmath>

#include "common.cuh"
#include "dtcore.cuh"
#include "rhscore.cuh"

namespace mhd {

constexpr int PT = 256;

static int grid_for(const Ctx *c, long n)
{
    long b = (n + PT - 1) / PT;
    long cap = (long)c->sm_count * 8;
    return (int)(b < cap ? b : cap);
}

__global__ void efield_kernel(const double *__restrict__ uu, double *__restrict__ E, long plane)
{
    for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < plane;
         o += (long)gridDim.x * blockDim.x) {
        double ux = uu[UX * plane + o], uy = uu[UY * plane + o], uz = uu[UZ * plane + o];
        double bx = uu[BX * plane + o], by = uu[BY * plane + o], bz = uu[BZ * plane + o];
        E[o] = uz * by - uy * bz;
        E[plane + o] = ux * bz - uz * bx;
        E[2 * plane + o] = uy * bx - ux * by;
    }
}

__global__ void divb_kernel(const double *__restrict__ dudx, const double *__restrict__ dudy,
                            double *__restrict__ out, long plane)
{
    for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < plane;
         o += (long)gridDim.x * blockDim.x)
        out[o] = dudx[BX * plane + o] + dudy[BY * plane + o];
}

struct RhsArgs {
    const double *uu, *dudx, *dudy, *dEdx, *dEdy;
    const double *d2udx2, *d2udy2, *d2Bdx2, *d2Bdy2, *ddivBdx, *ddivBdy;
    double *dudt;
    long plane;
    double gamma, visc, resist, cdiff, Ch, Cp;
    int cleaning;
};

// calcRHSInnerPoint on the whole periodic domain, then addSourceTerm
// (rhs_point, rhscore.cuh)
__global__ void rhs_kernel(RhsArgs a)
{
    const long plane = a.plane;
    RhsCoef k{a.gamma, a.visc, a.resist, a.cdiff, a.Ch, a.Cp, a.cleaning};
    const int nv = a.cleaning == 2 ? 9 : 8;
    for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < plane;
         o += (long)gridDim.x * blockDim.x) {
        double u[9], dx[9], dy[9], d2x[6], d2y[6], r[9];
#pragma unroll
        for (int v = 0; v < 9; v++) {
            if (v < nv) {
                u[v] = a.uu[v * plane + o];
                dx[v] = a.dudx[v * plane + o];
                dy[v] = a.dudy[v * plane + o];
            } else {
                u[v] = dx[v] = dy[v] = 0.0;
            }
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            d2x[c] = a.visc > 0 ? a.d2udx2[c * plane + o] : 0.0;
            d2y[c] = a.visc > 0 ? a.d2udy2[c * plane + o] : 0.0;
            d2x[3 + c] = a.resist > 0 ? a.d2Bdx2[c * plane + o] : 0.0;
            d2y[3 + c] = a.resist > 0 ? a.d2Bdy2[c * plane + o] : 0.0;
        }
        double dbx = a.cleaning == 1 ? a.ddivBdx[o] : 0.0;
        double dby = a.cleaning == 1 ? a.ddivBdy[o] : 0.0;
        rhs_point(k, u, dx, dy, d2x, d2y, a.dEdx[plane + o], a.dEdx[2 * plane + o], a.dEdy[o],
                  a.dEdy[2 * plane + o], dbx, dby, r);
        for (int v = 0; v < nv; v++) a.dudt[v * plane + o] = r[v];
    }
}

__global__ void rk_kernel(double *__restrict__ uu, const double *__restrict__ dudt,
                          double *__restrict__ dudtRK, long n, double cc, double dd)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        double d = dudt[i];
        uu[i] = uu[i] + cc * d + dd * dudtRK[i];
        dudtRK[i] = d;
    }
}

// --- reductions ------------------------------------------------------------
__device__ __forceinline__ double warp_min(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// per block: the (mn, lastneg, nanflag) fold of dtcore.cuh at part[3 b ..]
__global__ void dt_partial_kernel(DtArgs a)
{
    DtFold f{INFINITY, -1.0, 0.0};
    for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < a.plane;
         o += (long)gridDim.x * blockDim.x)
        dt_cell_fold(a, o, f);
    __shared__ double sm[3][PT / 32];
    f.mn = warp_min(f.mn);
    f.lastneg = warp_max(f.lastneg);
    f.nanflag = warp_max(f.nanflag);
    if ((threadIdx.x & 31) == 0) {
        sm[0][threadIdx.x >> 5] = f.mn;
        sm[1][threadIdx.x >> 5] = f.lastneg;
        sm[2][threadIdx.x >> 5] = f.nanflag;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = INFINITY, l = -1.0, n = 0.0;
        for (int w = 0; w < (int)(blockDim.x / 32); w++) {
            m = fmin(m, sm[0][w]);
            l = fmax(l, sm[1][w]);
            n = fmax(n, sm[2][w]);
        }
        a.part[3 * blockIdx.x] = m;
        a.part[3 * blockIdx.x + 1] = l;
        a.part[3 * blockIdx.x + 2] = n;
    }
}

// scal[0] = the new dt: the reference's running minimum (dtcore.cuh) times
// cfl, with the 2% hysteresis of timeAdvance.c:144-151 around dt0 (dt0 is
// scal[0] itself with dev_dt; keep_dt leaves scal[0] alone); with hyperbolic
// cleaning scal[1] = Ch = MAX(cmaxx, cmaxy) of the LAST cell of the
// reference's loop (timeAdvance.c:107-112) and scal[2] = Cp = sqrt(Cr Ch)
// (divBcleaning.c:4-10).
__global__ void __launch_bounds__(256) dt_final_kernel(DtArgs a, int nparts, double cfl, double dt0, int cleaning,
                                double *scal, int dev_dt, int keep_dt)
{
    double mn = INFINITY, l = -1.0, n = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        mn = fmin(mn, a.part[3 * i]);
        l = fmax(l, a.part[3 * i + 1]);
        n = fmax(n, a.part[3 * i + 2]);
    }
    __shared__ double sm[3][32];
    mn = warp_min(mn);
    l = warp_max(l);
    n = warp_max(n);
    if ((threadIdx.x & 31) == 0) {
        sm[0][threadIdx.x >> 5] = mn;
        sm[1][threadIdx.x >> 5] = l;
        sm[2][threadIdx.x >> 5] = n;
    }
    __syncthreads();
    mn = INFINITY, l = -1.0, n = 0.0;
    for (int w = 0; w < (int)(blockDim.x / 32); w++) {
        mn = fmin(mn, sm[0][w]);
        l = fmax(l, sm[1][w]);
        n = fmax(n, sm[2][w]);
    }
    __shared__ double red[32];
    const double dmin = dt_resolve(a, mn, l, n, red);  // uniform across the block
    if (threadIdx.x == 0) {
        double dtmin = dmin * cfl;
        if (dev_dt) dt0 = scal[0];
        if (!keep_dt) scal[0] = (dt0 < 0.98 * dtmin || dt0 > 1.02 * dtmin) ? dtmin : dt0;
        if (cleaning == 2) {
            double cx, cy;
            cell_speeds(a, a.plane - 1, cx, cy);
            double ch = ref_max(cx, cy);
            scal[1] = ch;
            scal[2] = sqrt(0.18 * ch);
        }
    }
}

__global__ void maxdivb_kernel(const double *__restrict__ dudx, const double *__restrict__ dudy,
                               double *__restrict__ divb, long plane, double *part)
{
    double mx = 0.0;
    for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < plane;
         o += (long)gridDim.x * blockDim.x) {
        double v = dudx[BX * plane + o] + dudy[BY * plane + o];
        divb[o] = v;
        mx = fmax(mx, fabs(v));
    }
    __shared__ double sm[PT / 32];
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < blockDim.x / 32 ? sm[threadIdx.x] : 0.0;
        v = warp_max(v);
        if (threadIdx.x == 0) part[blockIdx.x] = v;
    }
}

__global__ void diag_kernel(const double *__restrict__ uu, long plane, double gamma, double *part)
{
    double e = 0.0, h = 0.0, bad = 0.0, neg = 0.0;
    for (long o = blockIdx.x * (long)blockDim.x + threadIdx.x; o < plane;
         o += (long)gridDim.x * blockDim.x) {
        double rho = uu[RHO * plane + o], ux = uu[UX * plane + o], uy = uu[UY * plane + o];
        double uz = uu[UZ * plane + o], bx = uu[BX * plane + o], by = uu[BY * plane + o];
        double bz = uu[BZ * plane + o], p = uu[P * plane + o];
        e += 0.5 * rho * (ux * ux + uy * uy + uz * uz) + 0.5 * (bx * bx + by * by + bz * bz) +
             p / (gamma - 1.0);
        h += ux * bx + uy * by + uz * bz;
        double s = rho + ux + uy + uz + bx + by + bz + p;
        if (!isfinite(s)) bad += 1.0;                          // a NaN or Inf in the cell
        else if (!(rho > 0) || !(p > 0)) neg += 1.0;           // finite, rho or p not positive
    }
    __shared__ double sm[4][PT / 32];
    e = warp_sum(e); h = warp_sum(h); bad = warp_sum(bad); neg = warp_sum(neg);
    if ((threadIdx.x & 31) == 0) {
        sm[0][threadIdx.x >> 5] = e; sm[1][threadIdx.x >> 5] = h;
        sm[2][threadIdx.x >> 5] = bad; sm[3][threadIdx.x >> 5] = neg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        for (int w = 0; w < (int)(blockDim.x / 32); w++) {
            s0 += sm[0][w]; s1 += sm[1][w]; s2 += sm[2][w]; s3 += sm[3][w];
        }
        part[4 * blockIdx.x] = s0; part[4 * blockIdx.x + 1] = s1;
        part[4 * blockIdx.x + 2] = s2; part[4 * blockIdx.x + 3] = s3;
    }
}

__global__ void reduce_final_kernel(const double *part, int nparts, int stride, int mode,
                                    double *out)
{
    // mode 0: max of part[i*stride]; mode 1: sums of each of `stride` columns
    if (threadIdx.x != 0) return;
    if (mode == 0) {
        double v = 0.0;
        for (int i = 0; i < nparts; i++) v = fmax(v, part[i * stride]);
        out[0] = v;
    } else {
        for (int k = 0; k < stride; k++) {
            double s = 0.0;
            for (int i = 0; i < nparts; i++) s += part[i * stride + k];
            out[k] = s;
        }
    }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
int launch_efield(Ctx *c)
{
    long plane = c->nx * c->ny;
    prof_begin(c, KC_POINTWISE, 9.0 * plane * 8.0);
    efield_kernel<<<grid_for(c, plane), PT, 0, c->stream>>>(c->arr[MHDGPU_UU],
                                                             c->arr[MHDGPU_EFIELD], plane);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    return MHDGPU_OK;
}

int launch_divb(Ctx *c, double *out)
{
    long plane = c->nx * c->ny;
    prof_begin(c, KC_POINTWISE, 3.0 * plane * 8.0);
    divb_kernel<<<grid_for(c, plane), PT, 0, c->stream>>>(c->arr[MHDGPU_DUDX], c->arr[MHDGPU_DUDY],
                                                           out, plane);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    return MHDGPU_OK;
}

// fields calcRHS reads and writes
static int rhs_fields(const Ctx *c)
{
    int n = 3 * c->nvar + 2 + 2 + c->nvar;  // uu, dudx, dudy, dEdx(Ey,Ez), dEdy(Ex,Ez), dudt
    if (c->p.viscosity > 0) n += 6;
    if (c->p.resistivity > 0) n += 6;
    if (c->p.divBcleaning == 1) n += 2;
    return n;
}

int launch_rhs(Ctx *c)
{
    RhsArgs a;
    a.uu = c->arr[MHDGPU_UU];
    a.dudx = c->arr[MHDGPU_DUDX];
    a.dudy = c->arr[MHDGPU_DUDY];
    a.dEdx = c->arr[MHDGPU_DEDX];
    a.dEdy = c->arr[MHDGPU_DEDY];
    a.d2udx2 = c->arr[MHDGPU_D2UDX2];
    a.d2udy2 = c->arr[MHDGPU_D2UDY2];
    a.d2Bdx2 = c->arr[MHDGPU_D2BDX2];
    a.d2Bdy2 = c->arr[MHDGPU_D2BDY2];
    a.ddivBdx = c->arr[MHDGPU_DDIVBDX];
    a.ddivBdy = c->arr[MHDGPU_DDIVBDY];
    a.dudt = c->arr[MHDGPU_DUDT];
    a.plane = c->nx * c->ny;
    a.gamma = c->p.adiabaticIdx;
    a.visc = c->p.viscosity;
    a.resist = c->p.resistivity;
    a.cdiff = c->const_diff_divb;
    a.Ch = c->Ch;
    a.Cp = c->Cp;
    a.cleaning = c->p.divBcleaning;
    prof_begin(c, KC_POINTWISE, (double)rhs_fields(c) * a.plane * 8.0);
    rhs_kernel<<<grid_for(c, a.plane), PT, 0, c->stream>>>(a);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    return MHDGPU_OK;
}

int launch_rk(Ctx *c, int iRK)
{
    long n = (long)c->nvar * c->nx * c->ny;
    prof_begin(c, KC_POINTWISE, 5.0 * n * 8.0);
    rk_kernel<<<grid_for(c, n), PT, 0, c->stream>>>(c->arr[MHDGPU_UU], c->arr[MHDGPU_DUDT],
                                                     c->arr[MHDGPU_DUDTRK], n, c->cc[iRK],
                                                     c->dd[iRK]);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    return MHDGPU_OK;
}

static DtArgs dt_args(Ctx *c)
{
    DtArgs a;
    a.uu = c->arr[MHDGPU_UU];
    a.plane = c->nx * c->ny;
    a.ny = c->ny;
    a.gamma = c->p.adiabaticIdx;
    a.dx = c->dx;
    a.dy = c->dy;
    a.di = c->p.di;
    a.resist = c->p.resistivity;
    a.visc = c->p.viscosity;
    a.hall = c->p.Hall;
    a.part = c->dred;
    return a;
}

// calcDt on the device only: dt stays in dscal[0] (the previous dt there is
// dt0 of the hysteresis; keep_dt leaves a fixed dt untouched), Ch and Cp in
// dscal[1..2]; nothing is read back, so it can run inside a captured step.
int launch_calc_dt_dev(Ctx *c, int keep_dt)
{
    DtArgs a = dt_args(c);
    a.uu = state_ptr(c);  // the settled state: in the x filter's copy on long lines
    int g = grid_for(c, a.plane);
    if (3 * g > c->nred) g = c->nred / 3;
    prof_begin(c, KC_REDUCE, 7.0 * a.plane * 8.0);
    dt_partial_kernel<<<g, PT, 0, c->stream>>>(a);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    prof_begin(c, KC_REDUCE, 0.0);
    dt_final_kernel<<<1, 256, 0, c->stream>>>(a, g, c->p.cfl, 0.0, c->p.divBcleaning, c->dscal, 1,
                                               keep_dt);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    return MHDGPU_OK;
}

int launch_calc_dt(Ctx *c, double dt0, double *dt_out)
{
    DtArgs a = dt_args(c);
    int g = grid_for(c, a.plane);
    if (3 * g > c->nred) g = c->nred / 3;
    prof_begin(c, KC_REDUCE, 7.0 * a.plane * 8.0);
    dt_partial_kernel<<<g, PT, 0, c->stream>>>(a);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    prof_begin(c, KC_REDUCE, 0.0);
    dt_final_kernel<<<1, 256, 0, c->stream>>>(a, g, c->p.cfl, dt0, c->p.divBcleaning, c->dscal, 0, 0);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    double h[3];
    MHD_CUDA_TRY(cudaMemcpyAsync(h, c->dscal, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->p.divBcleaning == 2) {
        c->Ch = h[1];
        c->Cp = h[2];
    }
    if (dt_out) *dt_out = h[0];
    return MHDGPU_OK;
}

int launch_max_divb(Ctx *c, double *out)
{
    long plane = c->nx * c->ny;
    int g = grid_for(c, plane);
    if (g > c->nred) g = c->nred;
    prof_begin(c, KC_REDUCE, 3.0 * plane * 8.0);
    maxdivb_kernel<<<g, PT, 0, c->stream>>>(c->arr[MHDGPU_DUDX], c->arr[MHDGPU_DUDY],
                                             c->arr[MHDGPU_DIVB], plane, c->dred);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    prof_begin(c, KC_REDUCE, 0.0);
    reduce_final_kernel<<<1, 32, 0, c->stream>>>(c->dred, g, 1, 0, c->dscal + 3);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    MHD_CUDA_TRY(cudaMemcpyAsync(out, c->dscal + 3, sizeof(double), cudaMemcpyDeviceToHost,
                                 c->stream));
    MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return MHDGPU_OK;
}

int launch_diagnostics(Ctx *c, double *energy, double *ch, long *nonfinite, long *nonpositive)
{
    long plane = c->nx * c->ny;
    int g = grid_for(c, plane);
    if (4 * g > c->nred) g = c->nred / 4;
    prof_begin(c, KC_REDUCE, 8.0 * plane * 8.0);
    diag_kernel<<<g, PT, 0, c->stream>>>(c->arr[MHDGPU_UU], plane, c->p.adiabaticIdx, c->dred);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    prof_begin(c, KC_REDUCE, 0.0);
    reduce_final_kernel<<<1, 32, 0, c->stream>>>(c->dred, g, 4, 1, c->dscal + 4);
    prof_end(c);
    MHD_CHECK_LAUNCH();
    double h[4];
    MHD_CUDA_TRY(cudaMemcpyAsync(h, c->dscal + 4, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    MHD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (energy) *energy = h[0] * c->dx * c->dy;
    if (ch) *ch = h[1] * c->dx * c->dy;
    if (nonfinite) *nonfinite = (long)h[2];
    if (nonpositive) *nonpositive = (long)h[3];
    return MHDGPU_OK;
}

}  // namespace mhd
