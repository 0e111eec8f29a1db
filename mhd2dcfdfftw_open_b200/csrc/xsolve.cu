// x-direction compact operators: first derivative (derivCFD1st,
// mathlib.c:33-86), second derivative (derivCFD2nd, mathlib.c:163-218) and
// the compact filter (filterCFD, mathlib.c:296-354), each a 7-point (5-point
// on the two edge rows) right-hand side followed by the non-cyclic
// tridiagonal solve of tridiagonalSolver (mathlib.c:8-30) along every x-line.
//
// B200 design.  x-lines have stride ny, so a CTA owns a tile of W = 32
// adjacent columns (one 256-byte segment per row) and a contiguous block of
// rows; a thread-block cluster of C CTAs covers a whole line, so the line is
// read once and never leaves the chip:
//   1. the tile (its rows plus a 3-row periodic halo on each side) is staged
//      into shared memory by the TMA engine (cp.async.bulk, one 256-byte copy
//      per row, completion counted on an mbarrier);
//   2. every thread runs the Thomas recurrences on a sub-chunk of one column
//      with zero inflow; the exact inflows follow from a scan of the
//      sub-chunk end values (first-order linear recurrences compose:
//      y_true = y_local + prod(-m) * y_in), first inside the CTA through
//      shared memory, then across the cluster through distributed shared
//      memory;
//   3. the backward recurrence is split the same way and the result is
//      written once.
// The result equals the serial Thomas solve up to rounding (no truncation,
// no cyclic correction: the reference's system is not cyclic).
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "xcore.cuh"

namespace cg = cooperative_groups;

namespace mhd {

constexpr int XW = 32;         // columns per CTA
constexpr int XT = 256;        // threads per CTA
constexpr int XSUB = XT / XW;  // sub-chunks per CTA
constexpr int X_SMEM_BUDGET = 200 * 1024;

struct XArgs {
    const double *in;      // field 0 of the source array
    double *out;           // field 0 of the destination array
    const double *m, *invB, *g;
    XStencil st;
    long nx, ny;
    int R;                 // rows per CTA
    int C;                 // CTAs per cluster (= per line)
    int in_start;          // first source field
    int src_kind;          // 0: field, 1: Ey = ux Bz - uz Bx, 2: Ez = uy Bx - ux By
    int *flag;
};

__global__ void __launch_bounds__(XT, 1) xsolve_kernel(XArgs a)
{
    extern __shared__ __align__(128) unsigned char xsm_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    const int C = a.C;
    const int crank = (int)cluster.block_rank();
    const int tile = blockIdx.x / C;
    const int field = blockIdx.z;
    const long nx = a.nx, ny = a.ny;
    const long j0 = (long)tile * XW;
    const int ncols = (int)min((long)XW, ny - j0);
    const long r0 = (long)crank * a.R;
    const int Rc = (int)max(0L, min((long)a.R, nx - r0));  // rows of this CTA

    double *t = reinterpret_cast<double *>(xsm_raw);       // (R+6) x XW
    double *agg = t + (size_t)(a.R + 6) * XW;               // aggregates
    double *fw_end = agg, *fw_P = agg + XSUB * XW;
    double *bw_st = agg + 2 * XSUB * XW, *bw_Q = agg + 3 * XSUB * XW;
    double *cta = agg + 4 * XSUB * XW;                      // 4 x XW: Y, P, X, Q
    uint64_t *bar = reinterpret_cast<uint64_t *>(cta + 4 * XW);

    const int tid = threadIdx.x;
    const int lane = tid % XW;
    const int sub = tid / XW;
    const size_t plane = (size_t)nx * ny;
    const int nrows_tile = Rc + 6;

    // ---- 1. stage the tile ------------------------------------------------
    if (a.src_kind == 0) {
        const double *src = a.in + (size_t)(a.in_start + field) * plane;
        const unsigned row_bytes = (unsigned)ncols * 8u;
        if (tid == 0) {
            mbar_init(bar, 1);
        }
        __syncthreads();
        if (tid == 0) mbar_expect_tx(bar, row_bytes * (unsigned)nrows_tile);
        if (tid < 32) {
            __syncwarp();
            for (int r = tid; r < nrows_tile; r += 32) {
                long gr = wrap(r0 - 3 + r, nx);
                bulk_g2s(t + (size_t)r * XW, src + gr * ny + j0, row_bytes, bar);
            }
        }
        mbar_wait_bounded(bar, 0, a.flag);
    } else {
        const double *u = a.in;
        for (int idx = tid; idx < nrows_tile * XW; idx += XT) {
            int r = idx / XW, c = idx % XW;
            if (c < ncols) {
                long gr = wrap(r0 - 3 + r, nx);
                size_t o = (size_t)gr * ny + j0 + c;
                double v;
                if (a.src_kind == 1)
                    v = u[UX * plane + o] * u[BZ * plane + o] - u[UZ * plane + o] * u[BX * plane + o];
                else
                    v = u[UY * plane + o] * u[BX * plane + o] - u[UX * plane + o] * u[BY * plane + o];
                t[(size_t)r * XW + c] = v;
            }
        }
    }
    __syncthreads();

    // ---- 2. halo values of this thread's sub-chunk -----------------------
    const int S = (Rc + XSUB - 1) / XSUB;
    const int la = min(sub * S, Rc), lb = min(la + S, Rc);  // local rows [la, lb)
    double pre0 = t[(size_t)(la + 0) * XW + lane], pre1 = t[(size_t)(la + 1) * XW + lane],
           pre2 = t[(size_t)(la + 2) * XW + lane];
    double post0 = t[(size_t)(lb + 3) * XW + lane], post1 = t[(size_t)(lb + 4) * XW + lane],
           post2 = t[(size_t)(lb + 5) * XW + lane];
    __syncthreads();

    auto val = [&](int l) -> double {  // input value of local row l (la-3 <= l < lb+3)
        if (l < la) return l == la - 3 ? pre0 : (l == la - 2 ? pre1 : pre2);
        if (l >= lb) return l == lb ? post0 : (l == lb + 1 ? post1 : post2);
        return t[(size_t)(l + 3) * XW + lane];
    };

    // ---- 3. forward recurrence, zero inflow ------------------------------
    double y = 0.0, Pp = 1.0;
    {
        double w0 = val(la - 3), w1 = val(la - 2), w2 = val(la - 1);
        double w3 = la < lb ? val(la) : 0.0, w4 = la < lb ? val(la + 1) : 0.0,
               w5 = la < lb ? val(la + 2) : 0.0;
        for (int l = la; l < lb; l++) {
            double w6 = val(l + 3);
            long gr = r0 + l;
            double rhs = stencil(a.st, w0, w1, w2, w3, w4, w5, w6, gr, nx);
            double mi = a.m[gr];
            y = rhs - mi * y;
            Pp *= -mi;
            t[(size_t)(l + 3) * XW + lane] = y;
            w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6;
        }
    }
    fw_end[sub * XW + lane] = y;
    fw_P[sub * XW + lane] = Pp;
    __syncthreads();
    if (sub == 0) {
        double Y = 0.0, PP = 1.0;
        for (int s = 0; s < XSUB; s++) {
            Y = fw_end[s * XW + lane] + fw_P[s * XW + lane] * Y;
            PP *= fw_P[s * XW + lane];
        }
        cta[0 * XW + lane] = Y;
        cta[1 * XW + lane] = PP;
    }
    cluster.sync();

    // ---- 4. forward inflow, fix-up, backward recurrence (zero inflow) ----
    double cin = 0.0;
    for (int c2 = 0; c2 < crank; c2++) {
        const double *rc = cluster.map_shared_rank(cta, c2);
        cin = rc[0 * XW + lane] + rc[1 * XW + lane] * cin;
    }
    for (int s = 0; s < sub; s++) cin = fw_end[s * XW + lane] + fw_P[s * XW + lane] * cin;
    {
        double d = cin;
        for (int l = la; l < lb; l++) {
            d *= -a.m[r0 + l];
            t[(size_t)(l + 3) * XW + lane] += d;
        }
    }
    double x = 0.0, Qq = 1.0;
    for (int l = lb - 1; l >= la; l--) {
        long gr = r0 + l;
        double gi = a.g[gr];
        x = t[(size_t)(l + 3) * XW + lane] * a.invB[gr] - gi * x;
        Qq *= -gi;
        t[(size_t)(l + 3) * XW + lane] = x;
    }
    bw_st[sub * XW + lane] = x;
    bw_Q[sub * XW + lane] = Qq;
    __syncthreads();
    if (sub == 0) {
        double X = 0.0, QQ = 1.0;
        for (int s = XSUB - 1; s >= 0; s--) {
            X = bw_st[s * XW + lane] + bw_Q[s * XW + lane] * X;
            QQ *= bw_Q[s * XW + lane];
        }
        cta[2 * XW + lane] = X;
        cta[3 * XW + lane] = QQ;
    }
    cluster.sync();

    // ---- 5. backward inflow, fix-up, store --------------------------------
    double cb = 0.0;
    for (int c2 = C - 1; c2 > crank; c2--) {
        const double *rc = cluster.map_shared_rank(cta, c2);
        cb = rc[2 * XW + lane] + rc[3 * XW + lane] * cb;
    }
    for (int s = XSUB - 1; s > sub; s--) cb = bw_st[s * XW + lane] + bw_Q[s * XW + lane] * cb;
    if (lane < ncols) {
        double *dst = a.out + (size_t)field * plane + j0 + lane;
        double d = cb;
        for (int l = lb - 1; l >= la; l--) {
            long gr = r0 + l;
            d *= -a.g[gr];
            dst[(size_t)gr * ny] = t[(size_t)(l + 3) * XW + lane] + d;
        }
    }
    cluster.sync();  // peers may still read this CTA's aggregates until here
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

// Scheme constants, computed with the same expressions as initializeCFDSchemes
// (initialize.c:572-631) from parameter.h:23-31.
static void scheme_constants(double dx, XStencil st[3], double alpha[3][2])
{
    const double alphaInner1 = 0.375, alphaSub1 = 0.0;
    const double alphaInner2 = 0.375, alphaSub2 = 0.0;  // initialize.c:33 uses ALPHASUB1
    const double alphaInnerF = 0.49, alphaSubF = 0.95;
    double aInner1 = (alphaInner1 + 9.) / 6.;
    double bInner1 = (32 * alphaInner1 - 9.) / 15.;
    double cInner1 = (-3. * alphaInner1 + 1) / 10.;
    double aInner2 = (6. - 9. * alphaInner2) / 4.;
    double bInner2 = (-3. + 24. * alphaInner2) / 5.;
    double cInner2 = (2. - 11. * alphaInner2) / 20.;
    double aSub1 = (1. - alphaSub1) / 12.;
    double bSub1 = (3. * alphaSub1 - 4.) / 6.;
    double cSub1 = -3. / 2. * alphaSub1;
    double dSub1 = (4. + 5. * alphaSub1) / 6.;
    double eSub1 = (3. * alphaSub1 - 1.) / 12.;
    double aSub2 = -(1. + alphaSub2) / 12.;
    double bSub2 = (alphaSub2 + 4.) / 3.;
    double cSub2 = (alphaSub2 - 5.) / 2.;
    double dSub2 = (4. - 5. * alphaSub2) / 3.;
    double eSub2 = (11. * alphaSub2 - 1.) / 12.;
    double aInnerF = (11. + 10. * alphaInnerF) / 16.;
    double bInnerF = (15. + 34. * alphaInnerF) / 32.;
    double cInnerF = (-3. + 6. * alphaInnerF) / 16.;
    double dInnerF = (1. - 2. * alphaInnerF) / 32.;
    double aSubF = (alphaSubF - 1.) / 16.;
    double bSubF = (1 - alphaSubF) / 4.;
    double cSubF = (3. * alphaSubF + 5.) / 8.;
    double dSubF = (3. * alphaSubF + 1.) / 4.;
    double eSubF = (alphaSubF - 1.) / 16.;

    st[XOP_D1] = XStencil{aInner1 / 2, bInner1 / 4, cInner1 / 6, 0.0, aSub1, bSub1, cSub1,
                          dSub1, eSub1, 1 / dx, -1.0, XOP_D1};
    double dx2 = dx * dx;
    st[XOP_D2] = XStencil{aInner2, bInner2 / 4, cInner2 / 9, 0.0, aSub2, bSub2, cSub2,
                          dSub2, eSub2, 1 / dx2, 1.0, XOP_D2};
    st[XOP_F] = XStencil{aInnerF, bInnerF / 2, cInnerF / 2, dInnerF / 2, aSubF, bSubF, cSubF,
                         dSubF, eSubF, 1.0, 1.0, XOP_F};
    alpha[XOP_D1][0] = alphaInner1; alpha[XOP_D1][1] = alphaSub1;
    alpha[XOP_D2][0] = alphaInner2; alpha[XOP_D2][1] = alphaSub2;
    alpha[XOP_F][0] = alphaInnerF;  alpha[XOP_F][1] = alphaSubF;
}

int xsolve_setup(Ctx *c)
{
    const long n = c->nx;
    double alpha[3][2];
    scheme_constants(c->dx, c->xs, alpha);
    c->xf_alphaF[0] = alpha[XOP_F][0];
    c->xf_alphaF[1] = alpha[XOP_F][1];
    for (int op = 0; op < 3; op++) {
        // initTriMatrixCFD* for a periodic boundary (initialize.c:636-654):
        // lower[i] (row i+1) = alpha_inner except lower[n-2] = alpha_sub,
        // upper[0] = alpha_sub, upper[i] = alpha_inner, unit diagonal.
        std::vector<double> low(n - 1, alpha[op][0]), up(n - 1, alpha[op][0]);
        low[n - 2] = alpha[op][1];
        up[0] = alpha[op][1];
        // Thomas forward factors, as tridiagonalSolver computes them
        std::vector<double> m(n, 0.0), Bp(n, 1.0), invB(n), g(n, 0.0);
        for (long i = 1; i < n; i++) {
            m[i] = low[i - 1] / Bp[i - 1];
            Bp[i] = Bp[i] - m[i] * up[i - 1];
        }
        for (long i = 0; i < n; i++) invB[i] = 1.0 / Bp[i];
        for (long i = 0; i < n - 1; i++) g[i] = up[i] / Bp[i];
        XTables &T = c->xt[op];
        T.n = (int)n;
        MHD_CUDA_TRY(cudaMalloc(&T.m, sizeof(double) * n));
        MHD_CUDA_TRY(cudaMalloc(&T.invB, sizeof(double) * n));
        MHD_CUDA_TRY(cudaMalloc(&T.g, sizeof(double) * n));
        T.pfw = T.qbw = nullptr;
        MHD_CUDA_TRY(cudaMemcpy(T.m, m.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        MHD_CUDA_TRY(cudaMemcpy(T.invB, invB.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        MHD_CUDA_TRY(cudaMemcpy(T.g, g.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
    }
    // cluster size: the fewest CTAs whose tiles fit the shared-memory budget
    const size_t fixed = (size_t)(4 * XSUB + 4) * XW * sizeof(double) + 16;
    const long rmax = (long)((X_SMEM_BUDGET - fixed) / (XW * sizeof(double))) - 6;
    int C = (int)((n + rmax - 1) / rmax);
    if (C < 1) C = 1;
    while (C > 1 && (long)(C - 1) * ((n + C - 1) / C) >= n) C--;
    if (C > MHD_MAX_CLUSTER) return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
    c->x_cluster = C;
    c->x_rows_per_cta = (int)((n + C - 1) / C);
    MHD_CUDA_TRY(cudaFuncSetAttribute(xsolve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      X_SMEM_BUDGET + 1024));
    if (C > 8)
        MHD_CUDA_TRY(cudaFuncSetAttribute(xsolve_kernel,
                                          cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    return MHDGPU_OK;
}

void xsolve_free(Ctx *c)
{
    for (int op = 0; op < 3; op++) {
        cudaFree(c->xt[op].m);
        cudaFree(c->xt[op].invB);
        cudaFree(c->xt[op].g);
        c->xt[op].m = c->xt[op].invB = c->xt[op].g = nullptr;
    }
}

// Solve operator `op` on nv fields: out[v] = op(in[in_start + v]).  With
// src_kind 1/2 the single source field is Ey/Ez computed from `in` = uu.
int launch_xsolve(Ctx *c, int op, int nv, const double *in, int in_start, double *out,
                  int src_kind)
{
    if (nv <= 0) return MHDGPU_OK;
    if (((uintptr_t)in & 15) || ((uintptr_t)out & 15)) return mhd_set_error(MHDGPU_ERR_INVALID);
    XArgs a;
    a.in = in;
    a.out = out;
    a.m = c->xt[op].m;
    a.invB = c->xt[op].invB;
    a.g = c->xt[op].g;
    a.st = c->xs[op];
    a.nx = c->nx;
    a.ny = c->ny;
    a.R = c->x_rows_per_cta;
    a.C = c->x_cluster;
    a.in_start = in_start;
    a.src_kind = src_kind;
    a.flag = c->dflag;
    const int ntiles = (int)((c->ny + XW - 1) / XW);
    size_t smem = (size_t)(a.R + 6) * XW * sizeof(double) +
                  (size_t)(4 * XSUB + 4) * XW * sizeof(double) + 16;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ntiles * a.C, 1, nv);
    cfg.blockDim = dim3(XT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    prof_begin(c, KC_XSOLVE, (double)c->nx * c->ny * 8.0 * (double)((src_kind ? 4 : nv) + nv));
    MHD_CUDA_TRY(cudaLaunchKernelEx(&cfg, xsolve_kernel, a));
    prof_end(c);
    return MHDGPU_OK;
}

}  // namespace mhd
