// x pass of the fused RK3 stage (see fused.cu): for every field of the state
// and every x-line, the compact filter (filterCFD, mathlib.c:296-354) when it
// is pending, then the first derivative (derivCFD1st, mathlib.c:33-86) and,
// for the velocity and magnetic components, the second derivative
// (derivCFD2nd, mathlib.c:163-218) of the filtered line; then d/dx of Ey and
// Ez computed from the filtered state.  Every solve is the non-cyclic Thomas
// solve of tridiagonalSolver (mathlib.c:8-30).
//
// Layout of the work.  A cluster of C CTAs owns W adjacent columns over the
// whole line and walks all fields of that column tile:
//   * field v+1 is staged into the second of two shared-memory tiles by the
//     TMA engine (2-D tensor-map boxes of W columns, mbarrier completion)
//     while field v is solved;
//   * 512 threads per CTA, two CTAs per SM (one CTA's barrier waits overlap
//     the other's sweeps): thread (column, sub-chunk) keeps its 8 rows of a
//     recurrence in registers; the exact inflows of each sub-chunk come from
//     a warp-shuffle scan of the sub-chunk (end value, product) pairs inside
//     the CTA and of the totals of at most two neighbouring CTAs, read
//     through distributed shared memory;
//   * d/dx and d2/dx2 of a field, and dEy/dx with dEz/dx, share their matrix
//     and run as one paired solve;
//   * the filtered line replaces the tile's core rows, and each CTA pushes its
//     first and last filtered rows into its neighbours' halo rows, so the
//     line is read from HBM once for all three operators.
// Rows away from the two line ends use the constant interior Thomas factors
// and a branch-free interior stencil; the few sub-chunks that touch the first
// or last XF_EDGE rows use the tabulated factors and the closure stencils.
// T is the type of the recurrences: double, or float in mixed precision
// (where the filter is solved for its change; see xl_solve).
#include <cooperative_groups.h>

#include <cudaTypedefs.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "xcore.cuh"

namespace cg = cooperative_groups;

namespace mhd {

#ifndef MHD_XLINE_THREADS
#define MHD_XLINE_THREADS 512
#endif
#ifndef MHD_XLINE_ROWS
#define MHD_XLINE_ROWS 8
#endif
#ifndef MHD_XLINE_MINB
#define MHD_XLINE_MINB 2  // CTAs per SM the registers are budgeted for
#endif
constexpr int XL_T = MHD_XLINE_THREADS;  // threads per CTA
constexpr int XL_S = MHD_XLINE_ROWS;     // rows of a recurrence per thread
// Halo rows kept on each side of a CTA's rows (the stencils use 3): with 4,
// every TMA copy starts on an even tile row, which keeps the shared-memory
// destination of a copy 128-byte aligned for 8-column (64-byte) rows.
constexpr int XL_H = 4;

template <int W>
struct XLGeom {
    static constexpr int NSUB = XL_T / W;
    static constexpr int RCAP = NSUB * XL_S;  // rows per CTA at most
    static constexpr int TROWS = RCAP + 2 * XL_H;
};

// aggregate arrays are stored column-major with one pad slot per column
// (index col * (NSUB + 1) + sub) so a scan warp reads consecutive sub-chunks
template <int W>
__host__ __device__ constexpr int xl_aggn() { return W * (XLGeom<W>::NSUB + 1); }

template <int W>
__host__ __device__ constexpr size_t xl_smem_bytes()
{
    return sizeof(double) * (2 * (size_t)XLGeom<W>::TROWS * W + 2 * 3 * 2 * XF_EDGE +
                             6 * (size_t)xl_aggn<W>() + 2 * 6 * W) + 2 * sizeof(uint64_t);
}

// Aggregates of the sub-chunk recurrences.  Up to two systems with the same
// matrix are solved side by side, so they share the products P and carry
// their own end values E[0], E[1].
// T is the type of the recurrences (double, or float in the mixed-precision
// pass); the arrays are sized for doubles either way.
template <typename T>
struct XLSmem {
    double *tile[2];
    double *tab;
    T *aggE[2], *aggP;  // sub-chunk end values and product (zero inflow)
    T *preE[2], *preP;  // composite of the preceding sub-chunks of the CTA
    T *cta[2];          // [fwE0, fwE1, fwP, bwE0, bwE1, bwP] x W, alternating between solves
    uint64_t *bar;
};

template <int W, typename T>
__device__ __forceinline__ XLSmem<T> xl_carve(unsigned char *raw)
{
    XLSmem<T> s;
    double *p = reinterpret_cast<double *>(raw);
    s.tile[0] = p; p += (size_t)XLGeom<W>::TROWS * W;
    s.tile[1] = p; p += (size_t)XLGeom<W>::TROWS * W;
    s.tab = p; p += 2 * 3 * 2 * XF_EDGE;
    s.aggE[0] = reinterpret_cast<T *>(p); p += xl_aggn<W>();
    s.aggE[1] = reinterpret_cast<T *>(p); p += xl_aggn<W>();
    s.aggP = reinterpret_cast<T *>(p); p += xl_aggn<W>();
    s.preE[0] = reinterpret_cast<T *>(p); p += xl_aggn<W>();
    s.preE[1] = reinterpret_cast<T *>(p); p += xl_aggn<W>();
    s.preP = reinterpret_cast<T *>(p); p += xl_aggn<W>();
    s.cta[0] = reinterpret_cast<T *>(p); p += 6 * W;
    s.cta[1] = reinterpret_cast<T *>(p); p += 6 * W;
    s.bar = reinterpret_cast<uint64_t *>(p);
    return s;
}

// Scan of first-order linear recurrences over the sub-chunks of each column:
// warp `col` (< W) combines the (end values, product) of the NSUB sub-chunks
// in order (reversed for the backward sweep), writes the CTA total to
// cta[off * W ..] and the composite of the preceding sub-chunks to preE/preP.
// Composition: segment A then B gives (E_B + P_B E_A, P_A P_B).
template <int W, int NR, typename T>
__device__ __forceinline__ void xl_scan(const XLSmem<T> &s, T *cta, int off, bool reverse)
{
    constexpr int NSUB = XLGeom<W>::NSUB;
    // sub-chunks per lane; with fewer sub-chunks than lanes the idle lanes
    // carry the identity pair (0, 1)
    constexpr int K = NSUB >= 32 ? NSUB / 32 : 1;
    static_assert(NSUB < 32 || NSUB % 32 == 0, "sub-chunks per column must fill whole warps");
    const int lane = threadIdx.x & 31;
    // warp w scans columns w, w + (warps per CTA), ...
    for (int warp = threadIdx.x >> 5; warp < W; warp += XL_T / 32) {
        const int base = warp * (NSUB + 1);
        T E[NR], P = (T)1;
#pragma unroll
        for (int r = 0; r < NR; r++) E[r] = (T)0;
#pragma unroll
        for (int jq = 0; jq < K; jq++) {
            int q = lane * K + jq;
            if (q >= NSUB) break;
            int sidx = reverse ? NSUB - 1 - q : q;
            const T p = s.aggP[base + sidx];
#pragma unroll
            for (int r = 0; r < NR; r++) E[r] = s.aggE[r][base + sidx] + p * E[r];
            P = p * P;
        }
        // every lane takes part in every shuffle (full mask)
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T Eo[NR];
#pragma unroll
            for (int r = 0; r < NR; r++) Eo[r] = __shfl_up_sync(0xffffffffu, E[r], o);
            const T Po = __shfl_up_sync(0xffffffffu, P, o);
            if (lane >= o) {
#pragma unroll
                for (int r = 0; r < NR; r++) E[r] = E[r] + P * Eo[r];
                P = P * Po;
            }
        }
        T Ex[NR];
#pragma unroll
        for (int r = 0; r < NR; r++) {
            const T e = __shfl_up_sync(0xffffffffu, E[r], 1);
            Ex[r] = lane == 0 ? (T)0 : e;
        }
        const T pxs = __shfl_up_sync(0xffffffffu, P, 1);
        T Px = lane == 0 ? (T)1 : pxs;
        if (lane == 31) {
#pragma unroll
            for (int r = 0; r < NR; r++) cta[(off + r) * W + warp] = E[r];
            cta[(off + 2) * W + warp] = P;
        }
#pragma unroll
        for (int jq = 0; jq < K; jq++) {
            int q = lane * K + jq;
            if (q >= NSUB) break;
            int sidx = reverse ? NSUB - 1 - q : q;
#pragma unroll
            for (int r = 0; r < NR; r++) s.preE[r][base + sidx] = Ex[r];
            s.preP[base + sidx] = Px;
            const T p = s.aggP[base + sidx];
#pragma unroll
            for (int r = 0; r < NR; r++) Ex[r] = s.aggE[r][base + sidx] + p * Ex[r];
            Px = p * Px;
        }
    }
}

// interior right-hand side of operator OP (rows 1..n-2 of the line)
template <int OP>
__device__ __forceinline__ double xl_rhs(const XStencil &s, double w0, double w1, double w2,
                                         double w3, double w4, double w5, double w6)
{
    if (OP == XOP_D1) return s.scale * (s.a * (w4 - w2) + s.b * (w5 - w1) + s.c * (w6 - w0));
    if (OP == XOP_D2)
        return s.scale * (s.a * (w4 - 2 * w3 + w2) + s.b * (w5 - 2 * w3 + w1) + s.c * (w6 - 2 * w3 + w0));
    return s.a * w3 + s.b * (w4 + w2) + s.c * (w5 + w1) + s.d * (w6 + w0);
}

// Thomas factor `which` (0 m, 1 invB, 2 g) of matrix `mat` at row gr < n:
// tabulated near the line ends, the interior constant elsewhere
__device__ __forceinline__ double xl_tab(const double *tab, const XFTables &tb, int mat, int which,
                                         long gr, long n)
{
    const double *t = tab + (mat * 3 + which) * 2 * XF_EDGE;
    if (gr < XF_EDGE) return t[gr];
    if (gr >= n - XF_EDGE) return t[XF_EDGE + (gr - (n - XF_EDGE))];
    return tb.inner[mat][which];
}

// Output element type of a solve: the filter writes the FP64 state, the
// derivatives are stored in the recurrence type.
template <int OP, typename T>
struct XLOut { using type = T; };
template <typename T>
struct XLOut<XOP_F, T> { using type = double; };

// Inflow of this CTA from the CTAs before it (forward, dir = 0) or after it
// (backward, dir = 1): their totals (E, P) composed over at most `hops`
// neighbours.  The omitted farther totals enter multiplied by the products
// of the `hops` nearer chunks, which the host keeps below 2^-60 (hops = C
// chains through the whole cluster when it cannot).  With hops <= 2 both
// remote loads are issued at once.
template <int W, int NR, typename T>
__device__ __forceinline__ void xl_inflow(const XFArgs &a, cg::cluster_group &cluster, T *cta,
                                          int crank, int dir, int lane, T cin[NR])
{
#pragma unroll
    for (int r = 0; r < NR; r++) cin[r] = (T)0;
    const int h = a.hops;
    if (h <= 2) {
        T e[2][NR], p[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {  // k = 0: nearest neighbour
            const int c2 = dir == 0 ? crank - 1 - k : crank + 1 + k;
            p[k] = (T)0;
#pragma unroll
            for (int r = 0; r < NR; r++) e[k][r] = (T)0;
            if (k < h && c2 >= 0 && c2 < a.C) {
                const T *rc = cluster.map_shared_rank(cta, c2);
                const int off = dir == 0 ? 0 : 3;
#pragma unroll
                for (int r = 0; r < NR; r++) e[k][r] = rc[(off + r) * W + lane];
                p[k] = rc[(off + 2) * W + lane];
            }
        }
#pragma unroll
        for (int r = 0; r < NR; r++) cin[r] = e[0][r] + p[0] * e[1][r];
        return;
    }
    // the whole chain, farthest first
    if (dir == 0) {
        for (int c2 = 0; c2 < crank; c2++) {
            const T *rc = cluster.map_shared_rank(cta, c2);
            const T pp = rc[2 * W + lane];
#pragma unroll
            for (int r = 0; r < NR; r++) cin[r] = rc[r * W + lane] + pp * cin[r];
        }
    } else {
        for (int c2 = a.C - 1; c2 > crank; c2--) {
            const T *rc = cluster.map_shared_rank(cta, c2);
            const T pp = rc[5 * W + lane];
#pragma unroll
            for (int r = 0; r < NR; r++) cin[r] = rc[(3 + r) * W + lane] + pp * cin[r];
        }
    }
}

// Exact split Thomas solve over the core rows of the tile(s), NR = 1 or 2
// systems with the same matrix: operator OP0 on tile t0 and (NR = 2)
// operator OP1 on tile t1.  The right-hand sides are formed in FP64 from the
// FP64 tiles; the recurrences run in T.  Results go to global memory (column
// pointers g0/g1 of type OT, row stride ny) and/or, for one system, back
// into the tile's core rows (tout).
//   T = double: the reference's solves.
//   T = float (mixed precision): derivatives are stored as floats; the
//   filter is solved for its change d = A^-1 (B - A) u, the right-hand side
//   (B - A) u formed in FP64, and u + d is accumulated in FP64.
// `par` alternates between calls so that consecutive solves exchange carries
// through different arrays; the caller issues a cluster barrier before
// reading results of other CTAs.
template <int W, int OP0, int OP1, int NR, typename T>
__device__ void xl_solve(const XFArgs &a, const XLSmem<T> &s, cg::cluster_group &cluster,
                         const double *t0, const double *t1,
                         typename XLOut<OP0, T>::type *g0, typename XLOut<OP0, T>::type *g1,
                         double *tout, int Rc, long r0, int crank, int par)
{
    using OT = typename XLOut<OP0, T>::type;
    constexpr bool DELTA = OP0 == XOP_F && sizeof(T) == 4;  // filter change in FP32
    constexpr int NSUB = XLGeom<W>::NSUB;
    constexpr int MAT = OP0 == XOP_F ? 1 : 0;
    static_assert(NR == 1 || (OP1 != XOP_F && MAT == 0), "paired systems share the matrix");
    const int tid = threadIdx.x, lane = tid % W, sub = tid / W;
    const int ai = lane * (NSUB + 1) + sub;  // this thread's aggregate slot
    const long nx = a.nx, ny = a.ny;
    const int la = sub * XL_S;
    // interior sub-chunk: constant factors, branch-free stencils, no row checks
    const bool fast = !((r0 + la < XF_EDGE) || (r0 + la + XL_S > nx - XF_EDGE)) && la + XL_S <= Rc;
    const T m_in = (T)a.tb.inner[MAT][0], ib_in = (T)a.tb.inner[MAT][1], g_in = (T)a.tb.inner[MAT][2];
    T *cta = s.cta[par];
    const bool same = NR == 2 && t1 == t0;
    T y[NR][XL_S];

    // ---- forward recurrence with zero inflow ------------------------------
    T yv[NR], P = (T)1;
#pragma unroll
    for (int r = 0; r < NR; r++) yv[r] = (T)0;
    if (fast) {
        const double *tw = t0 + (XL_H - 3) * W + lane;  // tw[r * W] = input of local row r - 3
        double w0 = tw[(la + 0) * W], w1 = tw[(la + 1) * W], w2 = tw[(la + 2) * W];
        double w3 = tw[(la + 3) * W], w4 = tw[(la + 4) * W], w5 = tw[(la + 5) * W];
        const double *tv = (NR == 2 ? t1 : t0) + (XL_H - 3) * W + lane;
        double v0 = 0, v1 = 0, v2 = 0, v3 = 0, v4 = 0, v5 = 0;
        if (NR == 2 && !same) {
            v0 = tv[(la + 0) * W]; v1 = tv[(la + 1) * W]; v2 = tv[(la + 2) * W];
            v3 = tv[(la + 3) * W]; v4 = tv[(la + 4) * W]; v5 = tv[(la + 5) * W];
        }
#pragma unroll
        for (int k = 0; k < XL_S; k++) {
            const int l = la + k;
            const double w6 = tw[(l + 6) * W];
            double rhs = xl_rhs<OP0>(a.st[OP0], w0, w1, w2, w3, w4, w5, w6);
            if constexpr (DELTA) rhs -= a.fa_in * (w2 + w4) + w3;  // (B - A) u
            yv[0] = (T)rhs - m_in * yv[0];
            y[0][k] = yv[0];
            if constexpr (NR == 2) {
                if (same) {
                    yv[1] = (T)xl_rhs<OP1>(a.st[OP1], w0, w1, w2, w3, w4, w5, w6) - m_in * yv[1];
                } else {
                    const double v6 = tv[(l + 6) * W];
                    yv[1] = (T)xl_rhs<OP1>(a.st[OP1], v0, v1, v2, v3, v4, v5, v6) - m_in * yv[1];
                    v0 = v1; v1 = v2; v2 = v3; v3 = v4; v4 = v5; v5 = v6;
                }
                y[NR - 1][k] = yv[NR - 1];
            }
            w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6;
        }
        P = (T)a.pw[MAT][0];  // (-m)^XL_S, formed on the host as the rows would form it
    } else {  // near a line end or past the last row: tabulated factors, closures
#pragma unroll
        for (int r = 0; r < NR; r++) {
            const double *tw = (r == 0 ? t0 : t1) + (XL_H - 3) * W + lane;
            double w0 = tw[(la + 0) * W], w1 = tw[(la + 1) * W], w2 = tw[(la + 2) * W];
            double w3 = tw[(la + 3) * W], w4 = tw[(la + 4) * W], w5 = tw[(la + 5) * W];
            const XStencil &st = a.st[r == 0 ? OP0 : OP1];
            T pp = (T)1;
#pragma unroll
            for (int k = 0; k < XL_S; k++) {
                const int l = la + k;
                const long gr = r0 + l;
                double w6 = tw[(l + 6) * W];
                if (l < Rc) {
                    double rhs = stencil(st, w0, w1, w2, w3, w4, w5, w6, gr, nx);
                    if constexpr (DELTA) {  // (B - A) u with the matrix rows of initTriMatrix
                        const double lo = gr == 0 ? 0.0 : (gr == nx - 1 ? a.fa_sub : a.fa_in);
                        const double up = gr == nx - 1 ? 0.0 : (gr == 0 ? a.fa_sub : a.fa_in);
                        rhs -= lo * w2 + w3 + up * w4;
                    }
                    T m = (T)xl_tab(s.tab, a.tb, MAT, 0, gr, nx);
                    yv[r] = (T)rhs - m * yv[r];
                    pp *= -m;
                }
                y[r][k] = yv[r];
                w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6;
            }
            P = pp;
        }
    }
#pragma unroll
    for (int r = 0; r < NR; r++) s.aggE[r][ai] = yv[r];
    s.aggP[ai] = P;
    __syncthreads();
    xl_scan<W, NR, T>(s, cta, 0, false);
    cluster.sync();

    // ---- forward inflow and fix-up; backward recurrence with zero inflow --
    T cin[NR];
    xl_inflow<W, NR, T>(a, cluster, cta, crank, 0, lane, cin);
    T xv[NR], Q = (T)1;
    {
        const T pP = s.preP[ai];
#pragma unroll
        for (int r = 0; r < NR; r++) {
            T d = s.preE[r][ai] + pP * cin[r];
            if (fast) {
#pragma unroll
                for (int k = 0; k < XL_S; k++) {
                    d *= -m_in;
                    y[r][k] += d;
                }
                T x = (T)0;
#pragma unroll
                for (int k = XL_S - 1; k >= 0; k--) {
                    x = y[r][k] * ib_in - g_in * x;
                    y[r][k] = x;
                }
                xv[r] = x;
                Q = (T)a.pw[MAT][1];  // (-g)^XL_S
            } else {
#pragma unroll
                for (int k = 0; k < XL_S; k++) {
                    const int l = la + k;
                    if (l < Rc) {
                        d *= -(T)xl_tab(s.tab, a.tb, MAT, 0, r0 + l, nx);
                        y[r][k] += d;
                    }
                }
                T x = (T)0, qq = (T)1;
#pragma unroll
                for (int k = XL_S - 1; k >= 0; k--) {
                    const int l = la + k;
                    if (l < Rc) {
                        T g = (T)xl_tab(s.tab, a.tb, MAT, 2, r0 + l, nx);
                        x = y[r][k] * (T)xl_tab(s.tab, a.tb, MAT, 1, r0 + l, nx) - g * x;
                        qq *= -g;
                        y[r][k] = x;
                    }
                }
                xv[r] = x;
                Q = qq;
            }
        }
    }
    // Each thread has read its own preE/preP above; the scan that rewrites
    // them runs only after the barrier below, which every thread reaches
    // after that read, so the backward aggregates need no barrier before.
#pragma unroll
    for (int r = 0; r < NR; r++) s.aggE[r][ai] = xv[r];
    s.aggP[ai] = Q;
    __syncthreads();
    xl_scan<W, NR, T>(s, cta, 3, true);
    cluster.sync();

    // ---- backward inflow, fix-up and results -------------------------------
    T cb[NR];
    xl_inflow<W, NR, T>(a, cluster, cta, crank, 1, lane, cb);
    const T pQ = s.preP[ai];
    // The filtered line's boundary rows also go straight into the halo rows
    // of the neighbouring CTAs' tiles (periodic: the first and last CTA are
    // neighbours).  The neighbours read their halos only in their forward
    // sweeps, which they finished before the cluster barriers above.
    double *hp = nullptr, *hn = nullptr;  // prv's right halo, nxt's left halo (row 0, this lane)
    if constexpr (NR == 1 && OP0 == XOP_F) {
        if (tout) {
            const int C = a.C, prv = (crank - 1 + C) % C, nxt = (crank + 1) % C;
            const int Rp = (int)min((long)a.R, nx - (long)prv * a.R);
            hp = cluster.map_shared_rank(tout, prv) + (Rp + XL_H) * W + lane;
            hn = cluster.map_shared_rank(tout, nxt) + lane;
        }
    }
#pragma unroll
    for (int r = 0; r < NR; r++) {
        T d = s.preE[r][ai] + pQ * cb[r];
        OT *g = r == 0 ? g0 : g1;
        if (g) g += (size_t)r0 * ny;
#pragma unroll
        for (int k = XL_S - 1; k >= 0; k--) {
            const int l = la + k;
            if (l < Rc) {
                d *= fast ? -g_in : -(T)xl_tab(s.tab, a.tb, MAT, 2, r0 + l, nx);
                const T x = y[r][k] + d;
                OT v;
                if constexpr (DELTA) v = t0[(l + XL_H) * W + lane] + (double)x;  // u + d in FP64
                else v = (OT)x;
                if (g) g[(size_t)l * ny] = v;
                if constexpr (NR == 1 && OP0 == XOP_F) {
                    if (tout) {
                        tout[(l + XL_H) * W + lane] = (double)v;
                        if (l < XL_H) hp[l * W] = (double)v;
                        if (l >= Rc - XL_H) hn[(l - (Rc - XL_H)) * W] = (double)v;
                    }
                }
            }
        }
    }
}

constexpr int XL_BOX = 256;  // rows of the large tensor-map box

// The rows of tile [0, Rc+2H) come from field rows r0-H .. r0+Rc+H-1 with
// periodic wrap: at most three contiguous runs.  Each run is copied with
// 256-row boxes (the last box ends exactly at the run's end and may overlap
// the previous one) or, when shorter than 256 rows, with U-row boxes, U = 2
// for 8-column tiles (a 128-byte copy) and 1 otherwise.
struct XLRun {
    int toff;  // first tile row
    long g;    // first field row
    int len;
};

__device__ __forceinline__ int xl_runs(long r0, int Rc, long nx, XLRun run[3])
{
    int n = 0, toff = 0, left = Rc + 2 * XL_H;
    long g = r0 - XL_H;
    while (left > 0 && n < 3) {
        long gw = g < 0 ? g + nx : (g >= nx ? g - nx : g);
        int len = (int)min((long)left, nx - gw);
        run[n++] = XLRun{toff, gw, len};
        toff += len;
        g += len;
        left -= len;
    }
    return n;
}

// Issue the TMA copies of field `v` into tile buffer `b`; warp 0 only.
template <int W, typename T>
__device__ __forceinline__ void xl_stage(const XFArgs &a, const XLSmem<T> &s, int b, int v, long r0,
                                         int Rc, long j0, const CUtensorMap *big,
                                         const CUtensorMap *unit)
{
    XLRun run[3];
    const int nrun = xl_runs(r0, Rc, a.nx, run);
    unsigned bytes = 0;
    constexpr int U = W == 8 ? 2 : 1;
    for (int q = 0; q < nrun; q++) {
        int len = run[q].len;
        int nbox = len >= XL_BOX ? (len + XL_BOX - 1) / XL_BOX : len / U;
        bytes += (unsigned)nbox * (len >= XL_BOX ? XL_BOX : U) * W * 8u;
    }
    if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&s.bar[b], bytes);
    }
    __syncwarp();
    const long frow = (long)v * a.nx;
    int k = 0;  // copy counter across runs, dealt round-robin to the lanes
    for (int q = 0; q < nrun; q++) {
        const int len = run[q].len;
        if (len >= XL_BOX) {
            const int nbox = (len + XL_BOX - 1) / XL_BOX;
            for (int i = 0; i < nbox; i++, k++) {
                if ((k & 31) != (int)threadIdx.x) continue;
                int off = min(i * XL_BOX, len - XL_BOX);
                double *dst = s.tile[b] + (size_t)(run[q].toff + off) * W;
                if (smem_u32(dst) & 127u) {  // never issue a misaligned copy
                    atomicExch(a.flag, MHDGPU_ERR_INVALID);
                    continue;
                }
                tma_load_2d(dst, big, (int)j0, (int)(frow + run[q].g + off), &s.bar[b]);
            }
        } else {
            for (int i = 0; i < len; i += U, k++) {
                if ((k & 31) != (int)threadIdx.x) continue;
                double *dst = s.tile[b] + (size_t)(run[q].toff + i) * W;
                if (smem_u32(dst) & 127u) {  // never issue a misaligned copy
                    atomicExch(a.flag, MHDGPU_ERR_INVALID);
                    continue;
                }
                tma_load_2d(dst, unit, (int)j0, (int)(frow + run[q].g + i), &s.bar[b]);
            }
        }
    }
}

template <int W, typename T>
__global__ void __launch_bounds__(XL_T, MHD_XLINE_MINB)
xline_kernel(XFArgs a, const __grid_constant__ CUtensorMap tm_big,
             const __grid_constant__ CUtensorMap tm_unit)
{
    extern __shared__ __align__(128) unsigned char xl_raw[];
    cg::cluster_group cluster = cg::this_cluster();
    const int C = a.C;
    const int crank = (int)cluster.block_rank();
    const int tile = blockIdx.x / C;
    const long nx = a.nx, ny = a.ny;
    const long j0 = (long)tile * W;
    const int ncols = (int)min((long)W, ny - j0);
    const long r0 = (long)crank * a.R;
    const int Rc = (int)min((long)a.R, nx - r0);
    const size_t plane = (size_t)nx * ny;
    const int tid = threadIdx.x, lane = tid % W;
    const bool col = lane < ncols;
    XLSmem<T> s = xl_carve<W, T>(xl_raw);
    T *const o1 = reinterpret_cast<T *>(a.out1);  // derivative outputs hold T
    T *const o2a = reinterpret_cast<T *>(a.out2a), *const o2b = reinterpret_cast<T *>(a.out2b);
    T *const oE = reinterpret_cast<T *>(a.outE);

    for (int i = tid; i < 2 * 3 * 2 * XF_EDGE; i += XL_T) s.tab[i] = a.tb.edge[i];
    if (tid == 0) {
        mbar_init(&s.bar[0], 1);
        mbar_init(&s.bar[1], 1);
    }
    __syncthreads();

    const int nf = a.nfields;  // state fields [in_start, in_start + nf)
    unsigned phase[2] = {0u, 0u};
    int par = 0;  // alternates the carry-exchange arrays between solves
    if (nf > 0 && tid < 32) xl_stage<W>(a, s, 0, a.in_start, r0, Rc, j0, &tm_big, &tm_unit);

    // Block-uniform: set once a tile wait of this CTA ran out.  From then on
    // the CTA issues no copy and waits on no barrier (the tile that never
    // landed may still be in flight, so its buffer is not reused); it keeps
    // solving on whatever the tiles hold so that every cluster barrier is
    // still reached by every CTA, and the host reports MHDGPU_ERR_TIMEOUT.
    int failed = 0;
    for (int f = 0; f < nf; f++) {
        const int b = f & 1;
        const int v = a.in_start + f;
        // the other tile is free: its last readers finished before the
        // cluster barriers of the previous field's solves
        if (!failed && f + 1 < nf && tid < 32)
            xl_stage<W>(a, s, b ^ 1, v + 1, r0, Rc, j0, &tm_big, &tm_unit);
        bool ok = true;
        if (!failed) ok = mbar_wait_bounded(&s.bar[b], phase[b], a.flag);
        phase[b] ^= 1u;
        failed = __syncthreads_or(failed || !ok);
        double *t = s.tile[b];
        if (a.single_op >= 0) {  // one operator per field
            const size_t off = (size_t)f * plane + j0 + lane;
            if (a.single_op == XOP_F)  // the filter writes FP64 state
                xl_solve<W, XOP_F, XOP_F, 1, T>(a, s, cluster, t, t, (a.out1 && col) ? a.out1 + off : nullptr,
                                                nullptr, nullptr, Rc, r0, crank, par);
            else if (a.single_op == XOP_D1)
                xl_solve<W, XOP_D1, XOP_D1, 1, T>(a, s, cluster, t, t, (o1 && col) ? o1 + off : nullptr,
                                                  nullptr, nullptr, Rc, r0, crank, par);
            else
                xl_solve<W, XOP_D2, XOP_D2, 1, T>(a, s, cluster, t, t, (o1 && col) ? o1 + off : nullptr,
                                                  nullptr, nullptr, Rc, r0, crank, par);
            par ^= 1;
            continue;
        }
        if (a.fout) {
            double *g = col ? a.fout + (size_t)v * plane + j0 + lane : nullptr;
            xl_solve<W, XOP_F, XOP_F, 1, T>(a, s, cluster, t, t, g, nullptr, t, Rc, r0, crank, par);
            par ^= 1;
            // every CTA's tile holds its filtered core rows and, pushed by
            // its neighbours, the filtered halo rows
            cluster.sync();
        }
        if (!a.out1) continue;
        T *g1 = col ? o1 + (size_t)v * plane + j0 + lane : nullptr;
        T *g2 = nullptr;
        if (o2a && v >= a.d2a_lo && v < a.d2a_lo + 3)
            g2 = o2a + (size_t)(v - a.d2a_lo) * plane + j0 + lane;
        else if (o2b && v >= a.d2b_lo && v < a.d2b_lo + 3)
            g2 = o2b + (size_t)(v - a.d2b_lo) * plane + j0 + lane;
        if (g2)  // d/dx and d2/dx2 share the matrix: one paired solve
            xl_solve<W, XOP_D1, XOP_D2, 2, T>(a, s, cluster, t, t, g1, col ? g2 : nullptr, nullptr, Rc,
                                              r0, crank, par);
        else
            xl_solve<W, XOP_D1, XOP_D1, 1, T>(a, s, cluster, t, t, g1, nullptr, nullptr, Rc, r0, crank,
                                              par);
        par ^= 1;
    }

    if (a.outE) {
        // d/dx of Ey = ux Bz - uz Bx and Ez = uy Bx - ux By from the
        // (filtered) state this cluster has just written
        __threadfence();
        cluster.sync();
        const double *u = a.in;
        for (int idx = tid; idx < (Rc + 2 * XL_H) * W; idx += XL_T) {
            const int r = idx / W, c = idx % W;
            if (c < ncols) {
                long gr = r0 - XL_H + r;  // within [-XL_H, nx + XL_H): one wrap at most
                gr = gr < 0 ? gr + nx : (gr >= nx ? gr - nx : gr);
                const size_t o = (size_t)gr * ny + j0 + c;
                const double ux = u[UX * plane + o], uy = u[UY * plane + o], uz = u[UZ * plane + o];
                const double bx = u[BX * plane + o], by = u[BY * plane + o], bz = u[BZ * plane + o];
                s.tile[0][idx] = ux * bz - uz * bx;
                s.tile[1][idx] = uy * bx - ux * by;
            }
        }
        __syncthreads();
        // Ey and Ez share the matrix: one paired solve
        xl_solve<W, XOP_D1, XOP_D1, 2, T>(a, s, cluster, s.tile[0], s.tile[1],
                                          col ? oE + j0 + lane : nullptr,
                                          col ? oE + plane + j0 + lane : nullptr, nullptr, Rc, r0,
                                          crank, par);
        par ^= 1;
    }
    cluster.sync();  // peers may still read this CTA's shared memory
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

// Thomas factors of the two matrices as xsolve.cu tabulates them: the first
// and last XF_EDGE rows, and the interior constant, checked bit for bit.
static int xline_tables(Ctx *c)
{
    const long n = c->nx;
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
    return MHDGPU_OK;
}

// Tensor map of a [rows][ny] double array with boxes of W columns x boxrows.
static int xl_tensor_map(CUtensorMap *map, const double *base, long rows, long ny, int W,
                         int boxrows)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return mhd_set_error(MHDGPU_ERR_CUDA);
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    cuuint64_t gdim[2] = {(cuuint64_t)ny, (cuuint64_t)rows};
    cuuint64_t gstride[1] = {(cuuint64_t)ny * sizeof(double)};
    cuuint32_t box[2] = {(cuuint32_t)W, (cuuint32_t)boxrows};
    cuuint32_t estride[2] = {1, 1};
    CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(base), gdim,
                        gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? MHDGPU_OK : mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
}

static long xl_rcap(int W)
{
    return W == 32 ? XLGeom<32>::RCAP : W == 16 ? XLGeom<16>::RCAP : XLGeom<8>::RCAP;
}

template <typename T>
static int xl_attrs(int C)
{
    MHD_CUDA_TRY(cudaFuncSetAttribute(xline_kernel<32, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)xl_smem_bytes<32>()));
    MHD_CUDA_TRY(cudaFuncSetAttribute(xline_kernel<16, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)xl_smem_bytes<16>()));
    MHD_CUDA_TRY(cudaFuncSetAttribute(xline_kernel<8, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)xl_smem_bytes<8>()));
    if (C > 8) {
        MHD_CUDA_TRY(cudaFuncSetAttribute(xline_kernel<32, T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        MHD_CUDA_TRY(cudaFuncSetAttribute(xline_kernel<16, T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        MHD_CUDA_TRY(cudaFuncSetAttribute(xline_kernel<8, T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    }
    return MHDGPU_OK;
}

// Tile widths picked by xline_autotune, per grid shape, for the contexts
// this process creates later.
struct XLTuneKey {
    long nx, ny;
    int nvar;
    bool operator<(const XLTuneKey &o) const
    {
        return std::tie(nx, ny, nvar) < std::tie(o.nx, o.ny, o.nvar);
    }
};
static std::map<XLTuneKey, int> g_xl_tuned;
static std::mutex g_xl_tuned_mu;

static int xl_configure(Ctx *c, int W);

int xline_setup(Ctx *c)
{
    int rc = xline_tables(c);
    if (rc) return rc;
    const long n = c->nx;
    // One CTA holds up to RCAP rows of W columns.  Short lines take W = 32 in
    // one CTA; longer lines take W = 8 (512 rows per CTA: clusters of 8 CTAs
    // for 4096 rows, 16 for 8192), which keeps the clusters' SM footprint
    // small so more of them fit on the GPU.
    // MHDGPU_XLINE_W (8, 16 or 32) overrides the choice.
    // A width picked by xline_autotune for this shape comes first.
    int W = n <= XLGeom<32>::RCAP ? 32 : 8;
    {
        std::lock_guard<std::mutex> lock(g_xl_tuned_mu);
        auto it = g_xl_tuned.find(XLTuneKey{c->nx, c->ny, c->nvar});
        if (it != g_xl_tuned.end()) W = it->second;
    }
    if (const char *e = getenv("MHDGPU_XLINE_W")) {
        int w = atoi(e);
        if (w == 8 || w == 16 || w == 32) W = w;
    }
    return xl_configure(c, W);
}

// Tiling, carries and tensor maps of the fused x pass for tile width W;
// xf_W = 0 when the grid cannot be tiled (the steps then run through the
// operator stage).
static int xl_configure(Ctx *c, int W)
{
    int rc;
    const long n = c->nx;
    while (W > 8 && W > c->ny) W /= 2;  // a tile never spans more columns than the grid
    const long rcap = xl_rcap(W);
    int C = (int)((n + rcap - 1) / rcap);
    long R = (n + C - 1) / C;
    if (W == 8 && (R % 2 || n % 2)) {  // 64-byte rows: copies must start on even rows
        W = 16;
        C = (int)((n + xl_rcap(W) - 1) / xl_rcap(W));
        R = (n + C - 1) / C;
    }
    // Grids the fused x pass cannot tile run their steps through the operator
    // stage instead (xf_W = 0; see mhdgpu_steps_fused).
    if (W > c->ny || C > MHD_MAX_CLUSTER || R < XL_H || n - (long)(C - 1) * R < XL_H) {
        c->xf_W = 0;
        return MHDGPU_OK;
    }
    c->xf_W = W;
    c->xf_C = C;
    c->xf_R = (int)R;
    // Interior products of a full sub-chunk, (-m)^XL_S and (-g)^XL_S, formed
    // in the order the device forms them row by row.
    for (int mat = 0; mat < 2; mat++) {
        double pm = 1.0, pg = 1.0;
        for (int k = 0; k < XL_S; k++) {
            pm *= -c->xf_inner[mat][0];
            pg *= -c->xf_inner[mat][2];
        }
        c->xf_pw[mat][0] = pm;
        c->xf_pw[mat][1] = pg;
    }
    // Carries between CTAs: the inflow of a CTA is composed over its `hops`
    // nearest neighbours; the totals beyond enter multiplied by the products
    // of those chunks' Thomas factors.  Take the fewest hops (at least 2)
    // that keep every such product below 2^-60 in both directions, else
    // chain through the whole cluster.
    {
        std::vector<double> h[2][2];
        const int ops[2] = {XOP_D1, XOP_F};
        for (int mat = 0; mat < 2; mat++) {
            const double *dev[2] = {c->xt[ops[mat]].m, c->xt[ops[mat]].g};
            for (int w = 0; w < 2; w++) {
                h[mat][w].resize(n);
                MHD_CUDA_TRY(cudaMemcpy(h[mat][w].data(), dev[w], sizeof(double) * n,
                                        cudaMemcpyDeviceToHost));
            }
        }
        std::vector<double> cp[2][2];  // |product| of the factors over each chunk
        for (int mat = 0; mat < 2; mat++)
            for (int w = 0; w < 2; w++) {
                cp[mat][w].assign(C, 1.0);
                for (long i = 0; i < n; i++) cp[mat][w][i / R] *= std::fabs(h[mat][w][i]);
            }
        int hops = 2;
        for (; hops < C; hops++) {
            bool ok = true;
            for (int mat = 0; mat < 2 && ok; mat++)
                for (int w = 0; w < 2 && ok; w++)
                    for (int cc = 0; cc < C && ok; cc++) {
                        // w = 0: forward inflow of cc from cc-1 .. cc-hops;
                        // w = 1: backward inflow from cc+1 .. cc+hops
                        const int far = w == 0 ? cc - hops - 1 : cc + hops + 1;
                        if (far < 0 || far >= C) continue;  // the chain is complete
                        double p = 1.0;
                        for (int k = 1; k <= hops; k++) p *= cp[mat][w][w == 0 ? cc - k : cc + k];
                        if (p >= std::ldexp(1.0, -60)) ok = false;
                    }
            if (ok) break;
        }
        c->xf_hops = hops >= C ? C : hops;
    }
    const long rows = (long)c->nvar * n;
    if ((rc = xl_tensor_map(&c->xl_tmap_big, c->arr[MHDGPU_UU], rows, c->ny, W, XL_BOX))) return rc;
    if ((rc = xl_tensor_map(&c->xl_tmap_unit, c->arr[MHDGPU_UU], rows, c->ny, W, W == 8 ? 2 : 1)))
        return rc;
    if ((rc = xl_attrs<double>(C))) return rc;
    if ((rc = xl_attrs<float>(C))) return rc;
    return MHDGPU_OK;
}

int fused_x_timing_pass(Ctx *c);

// Time the fused x pass (its full program without a pending filter: the
// state is only read) at the context's precision for each tile width the
// grid admits, keep the fastest and remember it for this shape.  *w_out: the
// width chosen.
int xline_autotune(Ctx *c, int *w_out)
{
    if (c->xf_W == 0) return mhd_set_error(MHDGPU_ERR_UNSUPPORTED);
    {   // a shape tuned before in this process keeps its width (runs repeat bit for bit)
        int known = 0;
        {
            std::lock_guard<std::mutex> lock(g_xl_tuned_mu);
            auto it = g_xl_tuned.find(XLTuneKey{c->nx, c->ny, c->nvar});
            if (it != g_xl_tuned.end()) known = it->second;
        }
        if (known) {
            int rc = known == c->xf_W ? MHDGPU_OK : xl_configure(c, known);
            if (rc) return rc;
            if (w_out) *w_out = c->xf_W;
            return MHDGPU_OK;
        }
    }
    cudaEvent_t e0, e1;
    MHD_CUDA_TRY(cudaEventCreate(&e0));
    MHD_CUDA_TRY(cudaEventCreate(&e1));
    int best = c->xf_W, rc = MHDGPU_OK;
    float best_ms = 0.0f;
    const int prev = c->xf_W;
    for (int W : {8, 16, 32}) {
        if (W > c->ny || (rc = xl_configure(c, W)) != MHDGPU_OK) break;
        if (c->xf_W != W) continue;  // not admissible here
        if ((rc = fused_x_timing_pass(c))) break;  // warm-up
        cudaEventRecord(e0, c->stream);
        for (int k = 0; k < 3 && !rc; k++) rc = fused_x_timing_pass(c);
        cudaEventRecord(e1, c->stream);
        if (rc || cudaEventSynchronize(e1) != cudaSuccess) {
            rc = rc ? rc : mhd_set_error(MHDGPU_ERR_CUDA);
            break;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (best_ms == 0.0f || ms < best_ms) {
            best_ms = ms;
            best = W;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) {
        xl_configure(c, prev);
        return rc;
    }
    if ((rc = xl_configure(c, best))) return rc;
    {
        std::lock_guard<std::mutex> lock(g_xl_tuned_mu);
        g_xl_tuned[XLTuneKey{c->nx, c->ny, c->nvar}] = c->xf_W;
    }
    if (w_out) *w_out = c->xf_W;
    return MHDGPU_OK;
}

void xline_free(Ctx *c)
{
    cudaFree(c->xf_edge);
    c->xf_edge = nullptr;
}

int launch_xline(Ctx *c, const XFArgs &proto, double bytes)
{
    if (proto.nfields > 0 && proto.in != c->arr[MHDGPU_UU]) return mhd_set_error(MHDGPU_ERR_INVALID);
    XFArgs a = proto;
    for (int k = 0; k < 3; k++) a.st[k] = c->xs[k];
    a.tb.edge = c->xf_edge;
    std::memcpy(a.tb.inner, c->xf_inner, sizeof a.tb.inner);
    a.nx = c->nx;
    a.ny = c->ny;
    a.R = c->xf_R;
    a.C = c->xf_C;
    a.hops = c->xf_hops;
    a.fa_in = c->xf_alphaF[0];
    a.fa_sub = c->xf_alphaF[1];
    std::memcpy(a.pw, c->xf_pw, sizeof a.pw);
    a.flag = c->dflag;
    const int W = c->xf_W;
    const int ntiles = (int)((c->ny + W - 1) / W);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ntiles * a.C, 1, 1);
    cfg.blockDim = dim3(XL_T, 1, 1);
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    prof_begin(c, KC_FUSED_X, bytes);
    if (c->mixed) {
        if (W == 32) {
            cfg.dynamicSmemBytes = xl_smem_bytes<32>();
            MHD_CUDA_TRY(cudaLaunchKernelEx(&cfg, xline_kernel<32, float>, a, c->xl_tmap_big, c->xl_tmap_unit));
        } else if (W == 16) {
            cfg.dynamicSmemBytes = xl_smem_bytes<16>();
            MHD_CUDA_TRY(cudaLaunchKernelEx(&cfg, xline_kernel<16, float>, a, c->xl_tmap_big, c->xl_tmap_unit));
        } else {
            cfg.dynamicSmemBytes = xl_smem_bytes<8>();
            MHD_CUDA_TRY(cudaLaunchKernelEx(&cfg, xline_kernel<8, float>, a, c->xl_tmap_big, c->xl_tmap_unit));
        }
    } else if (W == 32) {
        cfg.dynamicSmemBytes = xl_smem_bytes<32>();
        MHD_CUDA_TRY(cudaLaunchKernelEx(&cfg, xline_kernel<32, double>, a, c->xl_tmap_big, c->xl_tmap_unit));
    } else if (W == 16) {
        cfg.dynamicSmemBytes = xl_smem_bytes<16>();
        MHD_CUDA_TRY(cudaLaunchKernelEx(&cfg, xline_kernel<16, double>, a, c->xl_tmap_big, c->xl_tmap_unit));
    } else {
        cfg.dynamicSmemBytes = xl_smem_bytes<8>();
        MHD_CUDA_TRY(cudaLaunchKernelEx(&cfg, xline_kernel<8, double>, a, c->xl_tmap_big, c->xl_tmap_unit));
    }
    prof_end(c);
    return MHDGPU_OK;
}

}  // namespace mhd
