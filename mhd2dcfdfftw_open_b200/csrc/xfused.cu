// Fused x pass of an RK3 stage: for every field of the state, along every
// x-line, the compact filter (filterCFD, mathlib.c:296-354) when the field
// still needs it, then the first derivative (derivCFD1st, mathlib.c:33-86)
// and, for the velocity and magnetic components, the second derivative
// (derivCFD2nd, mathlib.c:163-218) of the filtered field; one launch also
// serves the electric-field derivatives (E computed from the state on load).
//
// One cluster of C CTAs owns W adjacent columns of one field over the whole
// line, as in xsolve.cu, but the line is read from HBM once for all three
// operators: the filtered values are written back into the staged tile, the
// three halo rows on each side come from the neighbouring CTAs' tiles through
// distributed shared memory, and the first and second derivatives run as two
// recurrences side by side over the same tile.  Every tridiagonal solve is the
// exact split Thomas solve (zero-inflow sweeps per sub-chunk, inflows from a
// scan of the sub-chunk end values inside the CTA and across the cluster).
//
// The Thomas factors of a line are constant away from its two ends; the
// factors of the first and last EDGE rows are staged in shared memory and the
// interior uses the constants (the host checks that the interior is constant
// to the last bit).
#include <cooperative_groups.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "xcore.cuh"

namespace cg = cooperative_groups;

namespace mhd {

constexpr int XF_T = 256;
constexpr int XF_SMEM_MAX = 226 * 1024;

template <int W>
struct XFSmem {
    double *t;     // (R+6) x W input tile
    double *y1;    // R x W
    double *y2;    // R x W
    double *tab;   // 2 x 3 x 2*EDGE
    double *agg;   // 2 ops x 2 x (T/W) x W
    double *cta;   // 2 ops x 4 x W
    uint64_t *bar;
};

template <int W>
__host__ __device__ inline size_t xf_smem_bytes(int R)
{
    return sizeof(double) * ((size_t)(R + 6) * W + 2 * (size_t)R * W + 2 * 3 * 2 * XF_EDGE +
                             2 * 2 * (size_t)XF_T + 2 * 4 * W) + 16;
}

template <int W>
__device__ __forceinline__ XFSmem<W> xf_carve(unsigned char *raw, int R)
{
    XFSmem<W> s;
    double *p = reinterpret_cast<double *>(raw);
    s.t = p; p += (size_t)(R + 6) * W;
    s.y1 = p; p += (size_t)R * W;
    s.y2 = p; p += (size_t)R * W;
    s.tab = p; p += 2 * 3 * 2 * XF_EDGE;
    s.agg = p; p += 2 * 2 * XF_T;
    s.cta = p; p += 2 * 4 * W;
    s.bar = reinterpret_cast<uint64_t *>(p);
    return s;
}

// Thomas factor `which` (0 m, 1 invB, 2 g) of matrix `mat` at global row gr.
__device__ __forceinline__ double xf_coef(const double *tab, const XFTables &tb, int mat,
                                          int which, long gr, long n)
{
    const double *t = tab + (mat * 3 + which) * 2 * XF_EDGE;
    if (gr < XF_EDGE) return t[gr];
    if (gr >= n - XF_EDGE) return t[XF_EDGE + (gr - (n - XF_EDGE))];
    return tb.inner[mat][which];
}

__device__ __forceinline__ int xf_mat(int op) { return op == XOP_F ? 1 : 0; }

// Exact split Thomas solve of up to two operators over the tile rows of this
// CTA (input s.t, rows [3, Rc+3)); results land in yA / yB and, when gA / gB
// are non-null, in global memory (column pointers, row stride ny).  Ends with
// a cluster barrier, so the aggregate arrays may be reused right after.
template <int W, bool TWO>
__device__ void xf_solve(const XFArgs &a, XFSmem<W> &s, cg::cluster_group &cluster, int opA,
                         double *yA, double *gA, int opB, double *yB, double *gB, int Rc,
                         long r0, int crank)
{
    constexpr int NSUB = XF_T / W;
    const int tid = threadIdx.x, lane = tid % W, sub = tid / W;
    const long nx = a.nx, ny = a.ny;
    const int C = a.C;
    const int S = (Rc + NSUB - 1) / NSUB;
    const int la = min(sub * S, Rc), lb = min(la + S, Rc);
    const int mA = xf_mat(opA), mB = xf_mat(opB);
    const XStencil &stA = a.st[opA];
    const XStencil &stB = a.st[opB];
    const double *t = s.t;
    double *aggA_e = s.agg, *aggA_p = s.agg + XF_T;
    double *aggB_e = s.agg + 2 * XF_T, *aggB_p = s.agg + 3 * XF_T;
    double *ctaA = s.cta, *ctaB = s.cta + 4 * W;  // [fwY, fwP, bwX, bwQ] x W

    // ---- forward recurrences, zero inflow --------------------------------
    double ya = 0.0, pa = 1.0, yb = 0.0, pb = 1.0;
    {
        double w0 = t[(la + 0) * W + lane], w1 = t[(la + 1) * W + lane], w2 = t[(la + 2) * W + lane];
        double w3 = t[(la + 3) * W + lane], w4 = t[(la + 4) * W + lane], w5 = t[(la + 5) * W + lane];
        for (int l = la; l < lb; l++) {
            double w6 = t[(l + 6) * W + lane];
            long gr = r0 + l;
            double m = xf_coef(s.tab, a.tb, mA, 0, gr, nx);
            ya = stencil(stA, w0, w1, w2, w3, w4, w5, w6, gr, nx) - m * ya;
            pa *= -m;
            yA[l * W + lane] = ya;
            if (TWO) {
                double mb = xf_coef(s.tab, a.tb, mB, 0, gr, nx);
                yb = stencil(stB, w0, w1, w2, w3, w4, w5, w6, gr, nx) - mb * yb;
                pb *= -mb;
                yB[l * W + lane] = yb;
            }
            w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6;
        }
    }
    aggA_e[sub * W + lane] = ya;
    aggA_p[sub * W + lane] = pa;
    if (TWO) {
        aggB_e[sub * W + lane] = yb;
        aggB_p[sub * W + lane] = pb;
    }
    __syncthreads();
    if (sub == 0) {
        double Y = 0.0, PP = 1.0, Yb = 0.0, PPb = 1.0;
        for (int q = 0; q < NSUB; q++) {
            Y = aggA_e[q * W + lane] + aggA_p[q * W + lane] * Y;
            PP *= aggA_p[q * W + lane];
            if (TWO) {
                Yb = aggB_e[q * W + lane] + aggB_p[q * W + lane] * Yb;
                PPb *= aggB_p[q * W + lane];
            }
        }
        ctaA[0 * W + lane] = Y;
        ctaA[1 * W + lane] = PP;
        if (TWO) {
            ctaB[0 * W + lane] = Yb;
            ctaB[1 * W + lane] = PPb;
        }
    }
    cluster.sync();

    // ---- forward inflows and fix-up; backward recurrences ----------------
    double ca = 0.0, cb = 0.0;
    for (int c2 = 0; c2 < crank; c2++) {
        const double *rA = cluster.map_shared_rank(ctaA, c2);
        ca = rA[lane] + rA[W + lane] * ca;
        if (TWO) {
            const double *rB = cluster.map_shared_rank(ctaB, c2);
            cb = rB[lane] + rB[W + lane] * cb;
        }
    }
    for (int q = 0; q < sub; q++) {
        ca = aggA_e[q * W + lane] + aggA_p[q * W + lane] * ca;
        if (TWO) cb = aggB_e[q * W + lane] + aggB_p[q * W + lane] * cb;
    }
    __syncthreads();  // sub aggregates are reused for the backward sweep
    double xa = 0.0, qa = 1.0, xb = 0.0, qb = 1.0;
    {
        double da = ca, db = cb;
        for (int l = la; l < lb; l++) {
            long gr = r0 + l;
            da *= -xf_coef(s.tab, a.tb, mA, 0, gr, nx);
            yA[l * W + lane] += da;
            if (TWO) {
                db *= -xf_coef(s.tab, a.tb, mB, 0, gr, nx);
                yB[l * W + lane] += db;
            }
        }
        for (int l = lb - 1; l >= la; l--) {
            long gr = r0 + l;
            double g = xf_coef(s.tab, a.tb, mA, 2, gr, nx);
            xa = yA[l * W + lane] * xf_coef(s.tab, a.tb, mA, 1, gr, nx) - g * xa;
            qa *= -g;
            yA[l * W + lane] = xa;
            if (TWO) {
                double gb = xf_coef(s.tab, a.tb, mB, 2, gr, nx);
                xb = yB[l * W + lane] * xf_coef(s.tab, a.tb, mB, 1, gr, nx) - gb * xb;
                qb *= -gb;
                yB[l * W + lane] = xb;
            }
        }
    }
    aggA_e[sub * W + lane] = xa;
    aggA_p[sub * W + lane] = qa;
    if (TWO) {
        aggB_e[sub * W + lane] = xb;
        aggB_p[sub * W + lane] = qb;
    }
    __syncthreads();
    if (sub == 0) {
        double X = 0.0, QQ = 1.0, Xb = 0.0, QQb = 1.0;
        for (int q = NSUB - 1; q >= 0; q--) {
            X = aggA_e[q * W + lane] + aggA_p[q * W + lane] * X;
            QQ *= aggA_p[q * W + lane];
            if (TWO) {
                Xb = aggB_e[q * W + lane] + aggB_p[q * W + lane] * Xb;
                QQb *= aggB_p[q * W + lane];
            }
        }
        ctaA[2 * W + lane] = X;
        ctaA[3 * W + lane] = QQ;
        if (TWO) {
            ctaB[2 * W + lane] = Xb;
            ctaB[3 * W + lane] = QQb;
        }
    }
    cluster.sync();

    // ---- backward inflows, fix-up, results ---------------------------------
    ca = 0.0;
    cb = 0.0;
    for (int c2 = C - 1; c2 > crank; c2--) {
        const double *rA = cluster.map_shared_rank(ctaA, c2);
        ca = rA[2 * W + lane] + rA[3 * W + lane] * ca;
        if (TWO) {
            const double *rB = cluster.map_shared_rank(ctaB, c2);
            cb = rB[2 * W + lane] + rB[3 * W + lane] * cb;
        }
    }
    for (int q = NSUB - 1; q > sub; q--) {
        ca = aggA_e[q * W + lane] + aggA_p[q * W + lane] * ca;
        if (TWO) cb = aggB_e[q * W + lane] + aggB_p[q * W + lane] * cb;
    }
    {
        double da = ca, db = cb;
        for (int l = lb - 1; l >= la; l--) {
            long gr = r0 + l;
            da *= -xf_coef(s.tab, a.tb, mA, 2, gr, nx);
            double va = yA[l * W + lane] + da;
            yA[l * W + lane] = va;
            if (gA) gA[gr * ny] = va;
            if (TWO) {
                db *= -xf_coef(s.tab, a.tb, mB, 2, gr, nx);
                double vb = yB[l * W + lane] + db;
                yB[l * W + lane] = vb;
                if (gB) gB[gr * ny] = vb;
            }
        }
    }
    cluster.sync();
}

template <int W>
__global__ void __launch_bounds__(XF_T, 1) xfused_kernel(XFArgs a)
{
    extern __shared__ __align__(128) unsigned char xf_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    const int C = a.C;
    const int crank = (int)cluster.block_rank();
    const int tile = blockIdx.x / C;
    const int field = blockIdx.z;
    const long nx = a.nx, ny = a.ny;
    const long j0 = (long)tile * W;
    const int ncols = (int)min((long)W, ny - j0);
    const long r0 = (long)crank * a.R;
    const int Rc = (int)min((long)a.R, nx - r0);
    const size_t plane = (size_t)nx * ny;
    const int tid = threadIdx.x, lane = tid % W;
    XFSmem<W> s = xf_carve<W>(xf_raw, a.R);

    for (int i = tid; i < 2 * 3 * 2 * XF_EDGE; i += XF_T) s.tab[i] = a.tb.edge[i];

    // ---- stage the tile: rows r0-3 .. r0+Rc+3 (periodic wrap) --------------
    const int nrows = Rc + 6;
    int kind = a.src_kind == 3 ? 1 + field : a.src_kind;
    if (kind == 0) {
        const double *src = a.in + (size_t)(a.in_start + field) * plane;
        const unsigned row_bytes = (unsigned)ncols * 8u;
        if (tid == 0) mbar_init(s.bar, 1);
        __syncthreads();
        if (tid == 0) mbar_expect_tx(s.bar, row_bytes * (unsigned)nrows);
        if (tid < 32) {
            __syncwarp();
            for (int r = tid; r < nrows; r += 32)
                bulk_g2s(s.t + (size_t)r * W, src + wrap(r0 - 3 + r, nx) * ny + j0, row_bytes, s.bar);
        }
        mbar_wait_bounded(s.bar, 0, a.flag);
    } else {
        const double *u = a.in;
        for (int idx = tid; idx < nrows * W; idx += XF_T) {
            int r = idx / W, c = idx % W;
            if (c < ncols) {
                size_t o = (size_t)wrap(r0 - 3 + r, nx) * ny + j0 + c;
                double v;
                if (kind == 1)
                    v = u[UX * plane + o] * u[BZ * plane + o] - u[UZ * plane + o] * u[BX * plane + o];
                else
                    v = u[UY * plane + o] * u[BX * plane + o] - u[UX * plane + o] * u[BY * plane + o];
                s.t[(size_t)r * W + c] = v;
            }
        }
    }
    __syncthreads();

    const bool col = lane < ncols;
    if (a.single_op >= 0) {
        double *g = (a.out1 && col) ? a.out1 + (size_t)field * plane + j0 + lane : nullptr;
        xf_solve<W, false>(a, s, cluster, a.single_op, s.y1, g, 0, nullptr, nullptr, Rc, r0, crank);
        return;
    }

    const int v = a.in_start + field;  // state variable
    if (a.fout) {
        double *g = col ? a.fout + (size_t)v * plane + j0 + lane : nullptr;
        xf_solve<W, false>(a, s, cluster, XOP_F, s.y1, g, 0, nullptr, nullptr, Rc, r0, crank);
        // filtered rows become the tile's core rows ...
        for (int idx = tid; idx < Rc * W; idx += XF_T) s.t[3 * W + idx] = s.y1[idx];
        cluster.sync();
        // ... and the three rows on each side come from the neighbouring CTAs
        const int prv = (crank - 1 + C) % C, nxt = (crank + 1) % C;
        const int Rp = (int)min((long)a.R, nx - (long)prv * a.R);
        const double *tp = cluster.map_shared_rank(s.t, prv);
        const double *tn = cluster.map_shared_rank(s.t, nxt);
        if (tid < 3 * W) {
            int r = tid / W, cc = tid % W;
            s.t[r * W + cc] = tp[(Rp + r) * W + cc];
        } else if (tid < 6 * W) {
            int r = (tid - 3 * W) / W, cc = tid % W;
            s.t[(Rc + 3 + r) * W + cc] = tn[(3 + r) * W + cc];
        }
        cluster.sync();
    }
    double *g1 = (a.out1 && col) ? a.out1 + (size_t)v * plane + j0 + lane : nullptr;
    double *g2 = nullptr;
    if (a.out2a && v >= a.d2a_lo && v < a.d2a_lo + 3)
        g2 = a.out2a + (size_t)(v - a.d2a_lo) * plane + j0 + lane;
    else if (a.out2b && v >= a.d2b_lo && v < a.d2b_lo + 3)
        g2 = a.out2b + (size_t)(v - a.d2b_lo) * plane + j0 + lane;
    if (g2) {
        xf_solve<W, true>(a, s, cluster, XOP_D1, s.y1, g1, XOP_D2, s.y2, col ? g2 : nullptr, Rc,
                          r0, crank);
    } else {
        xf_solve<W, false>(a, s, cluster, XOP_D1, s.y1, g1, 0, nullptr, nullptr, Rc, r0, crank);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static double *g_dummy = nullptr;

int xfused_setup(Ctx *c)
{
    const long n = c->nx;
    // x kernels need the tables of the two matrices, tabulated as xsolve.cu
    // builds them; copy them back from the device copies made there
    std::vector<double> edge(2 * 3 * 2 * XF_EDGE, 0.0);
    double inner[2][3];
    for (int mat = 0; mat < 2; mat++) {
        int op = mat == 0 ? XOP_D1 : XOP_F;
        std::vector<double> h[3];
        const double *dev[3] = {c->xt[op].m, c->xt[op].invB, c->xt[op].g};
        for (int w = 0; w < 3; w++) {
            h[w].resize(n);
            MHD_CUDA_TRY(cudaMemcpy(h[w].data(), dev[w], sizeof(double) * n, cudaMemcpyDeviceToHost));
        }
        for (int w = 0; w < 3; w++) {
            double *lo = edge.data() + (mat * 3 + w) * 2 * XF_EDGE;
            double *hi = lo + XF_EDGE;
            for (long i = 0; i < XF_EDGE; i++) {
                lo[i] = i < n ? h[w][i] : 0.0;
                long r = n - XF_EDGE + i;
                hi[i] = r >= 0 ? h[w][r] : 0.0;
            }
            inner[mat][w] = n > 2 * XF_EDGE ? h[w][XF_EDGE] : 0.0;
            for (long i = XF_EDGE; i < n - XF_EDGE; i++)
                if (std::memcmp(&h[w][i], &inner[mat][w], sizeof(double)) != 0)
                    return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);  // interior not constant
        }
    }
    MHD_CUDA_TRY(cudaMalloc(&c->xf_edge, sizeof(double) * edge.size()));
    MHD_CUDA_TRY(cudaMemcpy(c->xf_edge, edge.data(), sizeof(double) * edge.size(),
                            cudaMemcpyHostToDevice));
    std::memcpy(c->xf_inner, inner, sizeof inner);
    // tile width and cluster size
    int W, rmax;
    if (n <= 8 * 512) { W = 16; rmax = 512; }
    else if (n <= 8 * 1024) { W = 8; rmax = 1024; }
    else return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
    int C = (int)((n + rmax - 1) / rmax);
    long R = (n + C - 1) / C;
    if (R < 3 || n - (long)(C - 1) * R < 3) return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
    c->xf_W = W;
    c->xf_C = C;
    c->xf_R = (int)R;
    size_t smem = W == 16 ? xf_smem_bytes<16>((int)R) : xf_smem_bytes<8>((int)R);
    if (smem > (size_t)XF_SMEM_MAX) return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
    MHD_CUDA_TRY(cudaFuncSetAttribute(xfused_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      XF_SMEM_MAX));
    MHD_CUDA_TRY(cudaFuncSetAttribute(xfused_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      XF_SMEM_MAX));
    (void)g_dummy;
    return MHDGPU_OK;
}

void xfused_free(Ctx *c)
{
    cudaFree(c->xf_edge);
    c->xf_edge = nullptr;
}

// Fused program (single_op < 0) or one operator over nf fields.
int launch_xfused(Ctx *c, const XFArgs &proto, int nf, double bytes)
{
    if (nf <= 0) return MHDGPU_OK;
    XFArgs a = proto;
    for (int k = 0; k < 3; k++) a.st[k] = c->xs[k];
    a.tb.edge = c->xf_edge;
    std::memcpy(a.tb.inner, c->xf_inner, sizeof a.tb.inner);
    a.nx = c->nx;
    a.ny = c->ny;
    a.R = c->xf_R;
    a.C = c->xf_C;
    a.flag = c->dflag;
    const int W = c->xf_W;
    const int ntiles = (int)((c->ny + W - 1) / W);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ntiles * a.C, 1, nf);
    cfg.blockDim = dim3(XF_T, 1, 1);
    cfg.dynamicSmemBytes = W == 16 ? xf_smem_bytes<16>(a.R) : xf_smem_bytes<8>(a.R);
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    prof_begin(c, KC_FUSED_X, bytes);
    if (W == 16) {
        MHD_CUDA_TRY(cudaLaunchKernelEx(&cfg, xfused_kernel<16>, a));
    } else {
        MHD_CUDA_TRY(cudaLaunchKernelEx(&cfg, xfused_kernel<8>, a));
    }
    prof_end(c);
    return MHDGPU_OK;
}

}  // namespace mhd
